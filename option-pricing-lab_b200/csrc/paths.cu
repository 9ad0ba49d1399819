// ob_paths: the drop-in for optlab::api::paths(rq, 1, 0) (RC/include/optlab_cuda/requests.hpp:105-106,
// RC/src/paths_gpu.cu:76-167). One thread per antithetic pair, state in registers, the spot columns and window
// extremes written in the reference's layout (out[(a n_cols + c) 2 n_pairs + row], pair p at row p, its antithetic
// at n_pairs + p), in float or double. The request is checked as RC/src/requests.cpp:168-207 does.
//
// Baskets whose names share one model kind, without a mixer (one to five names in Black-Scholes or local vol, one to
// three in Heston or SLV: every single-model quote), run a specialised kernel, paths_staged_kernel: the fused kernels' step
// (per-step records, correlation root, Heston parameters and the table as (y, dy) pairs staged in shared memory,
// normals drawn in batches of whole Philox blocks in the generic engine's stream order: the spot normals, then the
// residuals, from stream 0 for Heston and from the aux stream for SLV), and per step end the observations taken
// there, read from a staged schedule. Columns and window extremes are the reference's S = F_j exp(x) at each
// observation (kept columns written, window extremes compared on S), so a window's extremes equal those of the full
// columns bit for bit. Other requests run the generic kernel, which follows RC/include/optlab_cuda/paths.hpp step for
// step.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "fused.cuh"
#include "host_copy.cuh"

namespace ob {

namespace {

template <typename R>
struct PathsDev {
    ModelDev<R> m;
    int n_obs, n_cols, n_keep, n_win;
    long long n_pairs, first_pair, rows;
    const int* obs_step;
    const int* col_of;
    const int* win_lo;
    const int* win_hi;
    const R* fwd;  // n x n_obs
    double* out;
};

template <typename R, int N>
__device__ __forceinline__ void record(const PathsDev<R>& s, long long p, int j, const PairDev<R, N>& st,
                                       R (&lo)[2][N][2], R (&hi)[2][N][2]) {
    const long long r0 = p, r1 = s.n_pairs + p;
    const int c = s.col_of[j];
#pragma unroll
    for (int a = 0; a < N; ++a) {
        if (a >= s.m.n_names) continue;
        const R f = s.fwd[a * s.n_obs + j];
        const R S0 = f * m_exp(st.x[0][a]), S1 = f * m_exp(st.x[1][a]);
        double* base = s.out + static_cast<long long>(a) * s.n_cols * s.rows;
        if (c >= 0) {
            base[c * s.rows + r0] = static_cast<double>(S0);
            base[c * s.rows + r1] = static_cast<double>(S1);
        }
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            if (w >= s.n_win || j < s.win_lo[w] || j > s.win_hi[w]) continue;
            if (j == s.win_lo[w]) {
                lo[0][a][w] = hi[0][a][w] = S0;
                lo[1][a][w] = hi[1][a][w] = S1;
            } else {
                lo[0][a][w] = m_min(lo[0][a][w], S0), hi[0][a][w] = m_max(hi[0][a][w], S0);
                lo[1][a][w] = m_min(lo[1][a][w], S1), hi[1][a][w] = m_max(hi[1][a][w], S1);
            }
            if (j == s.win_hi[w]) {
                const long long cl = s.n_keep + 2 * w, ch = cl + 1;
                base[cl * s.rows + r0] = static_cast<double>(lo[0][a][w]);
                base[ch * s.rows + r0] = static_cast<double>(hi[0][a][w]);
                base[cl * s.rows + r1] = static_cast<double>(lo[1][a][w]);
                base[ch * s.rows + r1] = static_cast<double>(hi[1][a][w]);
            }
        }
    }
}

template <typename R, int N>
__global__ void __launch_bounds__(256) paths_kernel(PathsDev<R> s) {
    const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= s.n_pairs) return;
    PairDev<R, N> st;
    pair_init<R, N>(s.m, st, static_cast<uint64_t>(s.first_pair + p));
    R lo[2][N][2], hi[2][N][2];
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
        for (int w = 0; w < 2; ++w) lo[0][a][w] = lo[1][a][w] = hi[0][a][w] = hi[1][a][w] = R(0);
    int j = 0;
    while (j < s.n_obs && s.obs_step[j] == 0) record<R, N>(s, p, j++, st, lo, hi);
    for (int i = 1; i <= s.m.n_steps; ++i) {
        pair_step<R, N>(s.m, st, i);
        while (j < s.n_obs && s.obs_step[j] == i) record<R, N>(s, p, j++, st, lo, hi);
    }
}

// Offsets of the staged blob of paths_staged_kernel (bytes).
struct PathsLvOffsets {
    int step, name_step, root, hes, table2, sched, col, fwd;
    int mix_den, low_root;  // local correlation: per step sigma sqrt(max(t0, 1/12)); the aligned low root
};

template <typename R>
struct PathsLvArgs {
    PathsLvOffsets off;
    const unsigned char* blob;
    int smem_blob;
    int n_steps, n_obs, n_cols, n_keep, n_win;
    int win_lo[2], win_hi[2];
    long long n_pairs, first_pair, rows;
    uint32_t k0, k1;
    R top;
    double* out;
    const Pair2<R>* tab;  // the table in global memory when it does not fit the stage (table_global), else unused
    int table_global;
    int kind, same;  // the names' model kind (0 Black-Scholes, 1 local vol, 2 Heston, 3 SLV); residuals through the root
    int mixer;       // local correlation (kernels with MIX): w0 + level, down, up, sign, cos, sin of the mixer
    R mix_base, mix_down, mix_up, mix_sign, mix_cos, mix_sin;
};

// Observation j of both legs: the kept column and the windows that hold it, on S = F_j exp(x) as the reference.
template <typename R, int N>
__device__ __forceinline__ void lv_record(const PathsLvArgs<R>& a, const int* s_col, const R* s_fwd, int j, long long p,
                                          bool active, const R (&x0)[N], const R (&x1)[N], R (&lo)[2][N][2],
                                          R (&hi)[2][N][2]) {
    const int c = s_col[j];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const R f = s_fwd[n * a.n_obs + j];
        const R S0 = f * m_exp(x0[n]), S1 = f * m_exp(x1[n]);
        double* base = a.out + static_cast<long long>(n) * a.n_cols * a.rows;
        if (c >= 0 && active) {
            base[c * a.rows + p] = static_cast<double>(S0);
            base[c * a.rows + a.n_pairs + p] = static_cast<double>(S1);
        }
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            if (w >= a.n_win || j < a.win_lo[w] || j > a.win_hi[w]) continue;
            if (j == a.win_lo[w]) {
                lo[0][n][w] = hi[0][n][w] = S0, lo[1][n][w] = hi[1][n][w] = S1;
            } else {
                lo[0][n][w] = m_min(lo[0][n][w], S0), hi[0][n][w] = m_max(hi[0][n][w], S0);
                lo[1][n][w] = m_min(lo[1][n][w], S1), hi[1][n][w] = m_max(hi[1][n][w], S1);
            }
            if (j == a.win_hi[w] && active) {
                const long long cl = a.n_keep + 2 * w, ch = cl + 1;
                base[cl * a.rows + p] = static_cast<double>(lo[0][n][w]);
                base[ch * a.rows + p] = static_cast<double>(hi[0][n][w]);
                base[cl * a.rows + a.n_pairs + p] = static_cast<double>(lo[1][n][w]);
                base[ch * a.rows + a.n_pairs + p] = static_cast<double>(hi[1][n][w]);
            }
        }
    }
}

// 512-thread blocks for one or two names, 256 for more (registers); one float name fits two blocks an SM (32 warps).
template <int N>
constexpr int lv_block() {
    return N <= 2 ? 512 : 256;
}

// KIND: 0 Black-Scholes (constant variance), 1 local vol (table), 2 Heston (Euler), 3 SLV (table x Heston, residuals
// on the aux stream). GT: the table is read from global memory (a.tab) instead of the stage. MIX (Black-Scholes or
// local vol, 2 to 5 names): the local-correlation mixer, one more normal a step after the names'.
template <typename R, int N, int KIND, bool GT, bool MIX = false>
__global__ void __launch_bounds__(lv_block<N>(), N == 1 && sizeof(R) == 4 ? 2 : 1)
    paths_staged_kernel(PathsLvArgs<R> a) {
    constexpr bool VAR = KIND == 2 || KIND == 3;
    constexpr bool TABLE = KIND == 1 || KIND == 3;
    static_assert(!MIX || (KIND <= 1 && N >= 2), "the staged mixer runs Black-Scholes and local-vol baskets");
    constexpr int C = KIND == 2 ? 2 * N : N + (MIX ? 1 : 0);  // normals per step, stream 0
    constexpr int CA = KIND == 3 ? N : 0;     // normals per step, aux stream
    constexpr int G = C % 4 == 0 ? 1 : (C % 2 == 0 ? 2 : 4);  // steps per batch of whole Philox blocks
    constexpr int NB = C * G / 4, NBA = CA * G / 4;
    extern __shared__ __align__(16) unsigned char sm[];
    {
        const int4* src = reinterpret_cast<const int4*>(a.blob);
        int4* dst = reinterpret_cast<int4*>(sm);
        for (int t = threadIdx.x; t < a.smem_blob / 16; t += blockDim.x) dst[t] = src[t];
    }
    __syncthreads();
    const StepRec<R>* s_step = reinterpret_cast<const StepRec<R>*>(sm + a.off.step);
    const NameStep<R>* s_ns = reinterpret_cast<const NameStep<R>*>(sm + a.off.name_step);
    const R* s_root = reinterpret_cast<const R*>(sm + a.off.root);
    // per name: v0, kappa, theta, xi, rho, sqrt(1 - rho^2), the constant variance (Black-Scholes)
    const R* s_hes = reinterpret_cast<const R*>(sm + a.off.hes);
    const Pair2<R>* tab = GT ? a.tab : reinterpret_cast<const Pair2<R>*>(sm + a.off.table2);
    const int2* s_sched = reinterpret_cast<const int2*>(sm + a.off.sched);  // observations [x, y) at each step end
    const int* s_col = reinterpret_cast<const int*>(sm + a.off.col);
    const R* s_fwd = reinterpret_cast<const R*>(sm + a.off.fwd);
    const int S = a.n_steps;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < a.n_pairs;
         base += stride) {
        const int lane = threadIdx.x & 31;
        const bool active = base + lane < a.n_pairs;
        const long long p = active ? base + lane : a.n_pairs - 1;
        const uint64_t pair = static_cast<uint64_t>(a.first_pair + p);
        R x0[N], x1[N], v0[N], v1[N], lo[2][N][2], hi[2][N][2];
#pragma unroll
        for (int n = 0; n < N; ++n) {
            x0[n] = x1[n] = R(0);
            v0[n] = v1[n] = VAR ? s_hes[8 * n] : R(0);
#pragma unroll
            for (int w = 0; w < 2; ++w) lo[0][n][w] = lo[1][n][w] = hi[0][n][w] = hi[1][n][w] = R(0);
        }
        for (int j = s_sched[0].x; j < s_sched[0].y; ++j) lv_record<R, N>(a, s_col, s_fwd, j, p, active, x0, x1, lo, hi);
        for (int i0 = 1, b = 0; i0 <= S; i0 += G, ++b) {
            R z[C * G];
            R za[CA > 0 ? CA * G : 1];
#pragma unroll
            for (int k = 0; k < NB; ++k)
                normals4<R>(pair, static_cast<uint64_t>(b) * NB + k, 0u, a.k0, a.k1, z[4 * k], z[4 * k + 1],
                            z[4 * k + 2], z[4 * k + 3]);
#pragma unroll
            for (int k = 0; k < NBA; ++k)
                normals4<R>(pair, static_cast<uint64_t>(b) * NBA + k, kAuxStream, a.k0, a.k1, za[4 * k],
                            za[4 * k + 1], za[4 * k + 2], za[4 * k + 3]);
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int i = i0 + g;
                if (G > 1 && i > S) break;
                const StepRec<R> st = s_step[i - 1];
                R zm0[MIX ? N : 1], zm1[MIX ? N : 1];  // with the mixer each leg's own normals (signs in)
                if (MIX) {
                    // paths.hpp:219-237: a common factor whose weight moves with the level of the basket (the log of
                    // the mean of S / F at the step's start), per leg
                    const R* zs = &z[g * C];
                    const R* s_low = reinterpret_cast<const R*>(sm + a.off.low_root);
                    const R den = reinterpret_cast<const R*>(sm + a.off.mix_den)[i - 1];
#pragma unroll
                    for (int leg = 0; leg < 2; ++leg) {
                        const R sg = leg ? R(-1) : R(1);
                        R mm = R(0);
#pragma unroll
                        for (int n = 0; n < N; ++n) mm += m_exp(leg ? x1[n] : x0[n]);
                        const R u = m_log(mm / static_cast<R>(N)) / den;
                        R wt = a.mix_base + a.mix_down * m_max(-u, R(0)) - a.mix_up * m_max(u, R(0));
                        wt = m_min(m_max(wt, R(0)), R(1));
                        const R market = a.mix_sign * sg * zs[N - 1], fr = sg * zs[N];
                        const R common = a.mix_cos * market + a.mix_sin * fr;
                        R other[N];
#pragma unroll
                        for (int n = 0; n < N - 1; ++n) other[n] = sg * zs[n];
                        other[N - 1] = a.mix_sin * market - a.mix_cos * fr;
                        const R sw = m_sqrt(wt), sl = m_sqrt(R(1) - wt);
#pragma unroll
                        for (int n = 0; n < N; ++n) {
                            R acc = R(0);
#pragma unroll
                            for (int b = 0; b < N; ++b) acc += s_low[n * N + b] * other[b];
                            (leg ? zm1 : zm0)[n] = sw * common + sl * acc;
                        }
                    }
                }
                R wc[N];  // the variance's residual normals (correlated through the root when `same`)
                if (VAR) {
                    const R* zr = KIND == 3 ? &za[g * CA] : &z[g * C + N];
#pragma unroll
                    for (int n = 0; n < N; ++n) {
                        R acc = R(0);
#pragma unroll
                        for (int m = 0; m < N; ++m) acc += s_root[n * N + m] * zr[m];
                        wc[n] = a.same ? acc : zr[n];
                    }
                }
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    R zc = R(0);
                    if (!MIX) {
#pragma unroll
                        for (int m = 0; m < N; ++m) zc += s_root[n * N + m] * z[g * C + m];
                    }
                    const NameStep<R> ns = s_ns[(i - 1) * N + n];
                    R var0, var1, vp0 = R(0), vp1 = R(0);
                    if (VAR) vp0 = m_max(v0[n], R(0)), vp1 = m_max(v1[n], R(0));
                    if (TABLE) {
                        int j0, j1;
                        R f0, f1;
                        table_cell(ns, a.top, x0[n], j0, f0), table_cell(ns, a.top, x1[n], j1, f1);
                        const Pair2<R> y0 = GT ? ldg_pair(tab + ns.row + j0) : tab[ns.row + j0];
                        const Pair2<R> y1 = GT ? ldg_pair(tab + ns.row + j1) : tab[ns.row + j1];
                        const R t0 = y0.a + f0 * y0.b, t1 = y1.a + f1 * y1.b;
                        var0 = KIND == 1 ? t0 : t0 * vp0, var1 = KIND == 1 ? t1 : t1 * vp1;
                    } else if (VAR) {
                        var0 = vp0, var1 = vp1;
                    } else {
                        var0 = var1 = s_hes[8 * n + 6];
                    }
                    if (VAR) {
                        const R* h = s_hes + 8 * n;
                        const R zv = h[4] * zc + h[5] * wc[n];
                        v0[n] += h[1] * (h[2] - vp0) * st.dt + h[3] * (m_sqrt(vp0) * st.sdt) * zv;
                        v1[n] += h[1] * (h[2] - vp1) * st.dt + h[3] * (m_sqrt(vp1) * st.sdt) * (-zv);
                    }
                    if (MIX) {
                        x0[n] = lv_advance(x0[n], var0, st.hdt, st.sdt * zm0[n]);
                        x1[n] = lv_advance(x1[n], var1, st.hdt, st.sdt * zm1[n]);
                    } else {
                        const R zd = st.sdt * zc;  // sqrt(dt) z, the legs' +-
                        x0[n] = lv_advance(x0[n], var0, st.hdt, zd);
                        x1[n] = lv_advance(x1[n], var1, st.hdt, -zd);
                    }
                }
                const int2 ob = s_sched[i];
                for (int j = ob.x; j < ob.y; ++j) lv_record<R, N>(a, s_col, s_fwd, j, p, active, x0, x1, lo, hi);
            }
        }
    }
}

void check_request(const ob_paths_request& c) {
    if (c.n_names < 1 || c.n_names > OB_MAX_NAMES) invalid("n_names must be 1 to 8");
    if (c.n_pairs < 1 || c.first_pair < 0) invalid("n_pairs must be >= 1 and first_pair >= 0");
    if (c.n_steps < 0 || c.n_obs < 0) invalid("n_steps and n_obs must be >= 0");
    if (!c.out && c.n_obs > 0) invalid("null output");
    if (c.n_steps > 0 && (!c.dt || !c.t0)) invalid("null time grid");
    if (!c.root || !c.kind || !c.cvar || !c.heston || !c.fwd || (c.n_obs && !c.obs_step)) invalid("null array");
    bool table = false;
    for (int a = 0; a < c.n_names; ++a) {
        const int k = c.kind[a];
        if (k < 0 || k > 3) invalid("kind must be 0 to 3");
        table |= k == 1 || k == 3;
        if ((k == 2 || k == 3) && !(c.heston[a * 5 + 1] > 0 && c.heston[a * 5 + 2] > 0 && c.heston[a * 5 + 3] >= 0 &&
                                    std::fabs(c.heston[a * 5 + 4]) <= 1))
            invalid("Heston parameters out of range");
    }
    if (table) {
        if (c.n_x < 2 || c.n_rows < 1 || !c.step_row || !c.row_lo || !c.row_inv_dx || !c.table)
            invalid("a tabulated variance needs n_x >= 2, rows and step_row");
        for (long long i = 0; i < static_cast<long long>(c.n_names) * c.n_steps; ++i) {
            const int k = c.kind[i / (c.n_steps ? c.n_steps : 1)];
            if ((k == 1 || k == 3) && (c.step_row[i] < 0 || c.step_row[i] >= c.n_rows)) invalid("step_row out of range");
        }
    }
    int prev = 0;
    for (int j = 0; j < c.n_obs; ++j) {
        if (c.obs_step[j] < prev || c.obs_step[j] > c.n_steps) invalid("obs_step must be nondecreasing in [0, n_steps]");
        prev = c.obs_step[j];
    }
    if (c.mixer && (c.mixer != 1 || !c.low_root || !(c.mix[4] > 0))) invalid("bad local correlation");
    if (c.n_windows < 0 || c.n_windows > OB_MAX_WINDOWS || (c.n_windows && (!c.win_lo || !c.win_hi)))
        invalid("n_windows must be 0 to 2, with win_lo and win_hi");
    if (c.n_obs && !c.col_of) invalid("null col_of");
    if (c.n_keep < 0 || c.n_cols != c.n_keep + 2 * c.n_windows) invalid("n_cols must be n_keep + 2 n_windows");
    for (int j = 0; j < c.n_obs; ++j)
        if (c.col_of[j] < -1 || c.col_of[j] >= c.n_keep) invalid("col_of out of range");
    for (int w = 0; w < c.n_windows; ++w)
        if (c.win_lo[w] < 0 || c.win_hi[w] < c.win_lo[w] || c.win_hi[w] >= c.n_obs) invalid("bad window");
}

// The staged blob of paths_staged_kernel, or false when the request is not for it (names of different kinds, a
// mixer, more than five Black-Scholes / local-vol or three Heston / SLV names, or a blob beyond the shared-memory
// budget: 110 KB in float, 200 KB in double, without the table). The table goes into the stage when it fits beside
// the rest, else into global memory: a plan's per-step rows (801 points for each of the 756 steps of three daily
// years, 4.8 MB in float) stay in L2 and are read through the read-only cache.
template <typename R>
bool pack_paths_staged(const ob_paths_request& h, DeviceArena& arena, PathsLvArgs<R>& a) {
    const int n = h.n_names, S = h.n_steps, kind = h.kind[0];
    if (S < 1 || kind < 0 || kind > 3 || n > (kind <= 1 ? 5 : 3)) return false;
    if (h.mixer && (kind > 1 || n < 2)) return false;  // the mixer beside Heston or SLV names: the generic kernel
    for (int k = 0; k < n; ++k)
        if (h.kind[k] != kind) return false;
    const bool table = kind == 1 || kind == 3;
    a.kind = kind, a.same = h.same;
    std::vector<unsigned char> blob;
    auto put = [&](const void* src, size_t bytes) {
        const size_t at = (blob.size() + 15) & ~static_cast<size_t>(15);
        blob.resize(at + ((bytes + 15) & ~static_cast<size_t>(15)), 0);
        if (bytes) std::memcpy(blob.data() + at, src, bytes);
        return static_cast<int>(at);
    };
    std::vector<StepRec<R>> steps(S);
    for (int i = 0; i < S; ++i) {
        std::memset(&steps[i], 0, sizeof steps[i]);
        steps[i].hdt = static_cast<R>(-0.5 * h.dt[i]), steps[i].sdt = static_cast<R>(std::sqrt(h.dt[i]));
        steps[i].dt = static_cast<R>(h.dt[i]), steps[i].obs = -1;
    }
    a.off.step = put(steps.data(), steps.size() * sizeof(StepRec<R>));
    a.top = static_cast<R>(h.n_x - 1) - static_cast<R>(1e-4);
    std::vector<NameStep<R>> ns(static_cast<size_t>(S) * n);
    for (int i = 0; i < S; ++i)
        for (int k = 0; k < n; ++k) {
            NameStep<R>& r = ns[static_cast<size_t>(i) * n + k];
            std::memset(&r, 0, sizeof r);
            if (!table) continue;
            const int row = h.step_row[static_cast<size_t>(k) * S + i];
            set_cell_row(r, h.row_lo[row], h.row_inv_dx[row], a.top);
            r.row = row * (h.n_x - 1);
        }
    a.off.name_step = put(ns.data(), ns.size() * sizeof(NameStep<R>));
    std::vector<R> root(static_cast<size_t>(n) * n);
    for (size_t k = 0; k < root.size(); ++k) root[k] = static_cast<R>(h.root[k]);
    a.off.root = put(root.data(), root.size() * sizeof(R));
    std::vector<R> hes(8 * static_cast<size_t>(n), R(0));
    for (int k = 0; k < n; ++k) {
        for (int f = 0; f < 5; ++f) hes[8 * k + f] = static_cast<R>(h.heston[5 * k + f]);
        hes[8 * k + 5] = static_cast<R>(std::sqrt(1.0 - h.heston[5 * k + 4] * h.heston[5 * k + 4]));
        hes[8 * k + 6] = static_cast<R>(h.cvar[k]);
    }
    a.off.hes = put(hes.data(), hes.size() * sizeof(R));
    a.mixer = h.mixer;
    if (h.mixer) {
        std::vector<R> den(S), low(static_cast<size_t>(n) * n);
        for (int i = 0; i < S; ++i)  // R arithmetic as the generic step: sigma sqrt(max(t0, 1/12))
            den[i] = static_cast<R>(h.mix[4]) * std::sqrt(std::max(static_cast<R>(h.t0[i]), R(1.0 / 12)));
        for (size_t k = 0; k < low.size(); ++k) low[k] = static_cast<R>(h.low_root[k]);
        a.off.mix_den = put(den.data(), den.size() * sizeof(R));
        a.off.low_root = put(low.data(), low.size() * sizeof(R));
        a.mix_base = static_cast<R>(h.mix[0]) + static_cast<R>(h.mix[1]);
        a.mix_down = static_cast<R>(h.mix[2]), a.mix_up = static_cast<R>(h.mix[3]);
        a.mix_sign = static_cast<R>(h.mix[5]), a.mix_cos = static_cast<R>(h.mix[6]), a.mix_sin = static_cast<R>(h.mix[7]);
    }
    std::vector<int2> sched(S + 1);
    for (int i = 0, j = 0; i <= S; ++i) {
        sched[i].x = j;
        while (j < h.n_obs && h.obs_step[j] == i) ++j;
        sched[i].y = j;
    }
    a.off.sched = put(sched.data(), sched.size() * sizeof(int2));
    a.off.col = put(h.col_of, static_cast<size_t>(h.n_obs) * sizeof(int));
    std::vector<R> fwd(static_cast<size_t>(n) * h.n_obs);
    for (size_t k = 0; k < fwd.size(); ++k) fwd[k] = static_cast<R>(h.fwd[k]);
    a.off.fwd = put(fwd.data(), fwd.size() * sizeof(R));
    std::vector<Pair2<R>> tab(table ? static_cast<size_t>(h.n_rows) * (h.n_x - 1) : 0);
    for (int r = 0; r < (table ? h.n_rows : 0); ++r)
        for (int k = 0; k + 1 < h.n_x; ++k) {
            const double y = h.table[static_cast<size_t>(r) * h.n_x + k], y1 = h.table[static_cast<size_t>(r) * h.n_x + k + 1];
            tab[static_cast<size_t>(r) * (h.n_x - 1) + k] = {static_cast<R>(y), static_cast<R>(y1 - y)};
        }
    const size_t budget = sizeof(R) == 4 ? (110u << 10) : (200u << 10);
    const size_t tab_bytes = tab.size() * sizeof(Pair2<R>);
    if (blob.size() > budget) return false;
    a.table_global = ((blob.size() + 15) & ~static_cast<size_t>(15)) + tab_bytes > budget;
    if (a.table_global) a.tab = arena.put_raw(tab.data(), tab.size());
    else a.off.table2 = put(tab.data(), tab_bytes);
    a.smem_blob = static_cast<int>(blob.size());
    a.blob = arena.put<unsigned char>(blob.data(), blob.size());
    a.n_steps = S, a.n_obs = h.n_obs, a.n_cols = h.n_cols, a.n_keep = h.n_keep, a.n_win = h.n_windows;
    for (int w = 0; w < 2; ++w) {
        a.win_lo[w] = w < h.n_windows ? h.win_lo[w] : 0;
        a.win_hi[w] = w < h.n_windows ? h.win_hi[w] : -1;
    }
    a.k0 = static_cast<uint32_t>(h.seed), a.k1 = static_cast<uint32_t>(h.seed >> 32);
    return true;
}

inline int lv_block_of(int n) { return n <= 2 ? lv_block<1>() : lv_block<3>(); }

template <typename R, int KIND, bool GT>
const void* pick_paths_n(int n) {
    switch (n) {
        case 1: return reinterpret_cast<const void*>(paths_staged_kernel<R, 1, KIND, GT>);
        case 2: return reinterpret_cast<const void*>(paths_staged_kernel<R, 2, KIND, GT>);
        case 3: return reinterpret_cast<const void*>(paths_staged_kernel<R, 3, KIND, GT>);
    }
    if constexpr (KIND <= 1) {
        if (n == 4) return reinterpret_cast<const void*>(paths_staged_kernel<R, 4, KIND, GT>);
        if (n == 5) return reinterpret_cast<const void*>(paths_staged_kernel<R, 5, KIND, GT>);
    }
    return nullptr;
}

template <typename R, int KIND, bool GT>
const void* pick_paths_mix(int n) {
    switch (n) {
        case 2: return reinterpret_cast<const void*>(paths_staged_kernel<R, 2, KIND, GT, true>);
        case 3: return reinterpret_cast<const void*>(paths_staged_kernel<R, 3, KIND, GT, true>);
        case 4: return reinterpret_cast<const void*>(paths_staged_kernel<R, 4, KIND, GT, true>);
        case 5: return reinterpret_cast<const void*>(paths_staged_kernel<R, 5, KIND, GT, true>);
        default: return nullptr;
    }
}

template <typename R>
const void* pick_paths_staged(int n, int kind, bool table_global, bool mixer) {
    if (mixer) {
        if (kind == 0) return pick_paths_mix<R, 0, false>(n);
        if (kind == 1) return table_global ? pick_paths_mix<R, 1, true>(n) : pick_paths_mix<R, 1, false>(n);
        return nullptr;
    }
    switch (kind) {
        case 0: return pick_paths_n<R, 0, false>(n);
        case 1: return table_global ? pick_paths_n<R, 1, true>(n) : pick_paths_n<R, 1, false>(n);
        case 2: return pick_paths_n<R, 2, false>(n);
        case 3: return table_global ? pick_paths_n<R, 3, true>(n) : pick_paths_n<R, 3, false>(n);
        default: return nullptr;
    }
}

template <typename R>
void run_paths(ob_paths_request& h) {
    const auto t_start = std::chrono::steady_clock::now();
    require_device();
    const int n = h.n_names;
    bool table = false, has_var = false, has_slv = false;
    for (int a = 0; a < n; ++a) {
        table |= h.kind[a] == 1 || h.kind[a] == 3;
        has_var |= h.kind[a] == 2 || h.kind[a] == 3;
        has_slv |= h.kind[a] == 3;
    }
    DeviceArena arena;
    arena.recycle = true;  // both streams are synchronised before the call returns
    PathsDev<R> s{};
    ModelDev<R>& m = s.m;
    m.n_names = n, m.n_steps = h.n_steps, m.n_x = h.n_x, m.same = h.same, m.mixer = h.mixer;
    m.has_var = has_var, m.has_slv = has_slv;
    m.k0 = static_cast<uint32_t>(h.seed), m.k1 = static_cast<uint32_t>(h.seed >> 32);
    Upload up;  // the inputs in one copy
    up.add<R>(m.dt, h.dt, h.n_steps);
    up.add<R>(m.t0, h.t0, h.n_steps);
    up.add<R>(m.root, h.root, static_cast<size_t>(n) * n);
    up.add<int>(m.kind, h.kind, n);
    up.add<R>(m.cvar, h.cvar, n);
    up.add<R>(m.hes, h.heston, 5 * static_cast<size_t>(n));
    if (table) {
        up.add<int>(m.step_row, h.step_row, static_cast<size_t>(n) * h.n_steps);
        up.add<R>(m.lo, h.row_lo, h.n_rows);
        up.add<R>(m.inv_dx, h.row_inv_dx, h.n_rows);
        up.add<R>(m.table, h.table, static_cast<size_t>(h.n_rows) * h.n_x);
    }
    if (h.mixer) up.add<R>(m.low_root, h.low_root, static_cast<size_t>(n) * n);
    for (int k = 0; k < 8; ++k) m.mix[k] = static_cast<R>(h.mix[k]);
    s.n_obs = h.n_obs, s.n_cols = h.n_cols, s.n_keep = h.n_keep, s.n_win = h.n_windows;
    up.add<int>(s.obs_step, h.obs_step, h.n_obs);
    up.add<int>(s.col_of, h.col_of, h.n_obs);
    up.add<int>(s.win_lo, h.win_lo, h.n_windows);
    up.add<int>(s.win_hi, h.win_hi, h.n_windows);
    up.add<R>(s.fwd, h.fwd, static_cast<size_t>(n) * h.n_obs);
    up.commit(arena);
    PathsLvArgs<R> lv{};
    const void* lv_fn = pack_paths_staged<R>(h, arena, lv)
                            ? pick_paths_staged<R>(n, lv.kind, lv.table_global != 0, h.mixer != 0)
                            : nullptr;
    const bool fast = lv_fn != nullptr;
    int lv_grid = 0;
    if (fast) {
        allow_smem(lv_fn, lv.smem_blob);
        lv_grid = require_device() * std::max(1, occupancy(lv_fn, lv_block_of(n), lv.smem_blob));
    }

    // Chunks of pairs, on two streams: the kernel of one chunk runs while the previous chunk's columns are copied to
    // the host. Large outputs go in four chunks at least; each chunk's output (two buffers) within an eighth of the
    // free memory, at most 2 GB. The caller's array is not pinned (pinning 117 MB took 12.5 ms on a B200 host, longer
    // than the pageable copy itself, 6.7 ms; pinned, 2.2 ms): a chunk is copied into the library's pinned staging
    // (PinnedStage, at most a slot a chunk), and host threads spread it into the caller's array while the next chunk
    // runs; without the staging, straight into the caller's array.
    const long long cols = static_cast<long long>(n) * h.n_cols;
    size_t free_mem = 0, total_mem = 0;
    check_cuda(cudaMemGetInfo(&free_mem, &total_mem), "cudaMemGetInfo");
    const long long budget = std::min<long long>(static_cast<long long>(free_mem) / 8, 2LL << 30);
    const long long row_bytes = cols * 2 * 8;  // one pair's output
    double* stage[2] = {nullptr, nullptr};
    if (cols > 0 && row_bytes <= static_cast<long long>(PinnedStage::kSlotBytes)) {
        stage[0] = PinnedStage::get().slot(0), stage[1] = PinnedStage::get().slot(1);
        if (!stage[0] || !stage[1]) stage[0] = stage[1] = nullptr;
    }
    long long chunk = h.n_pairs;
    if (cols > 0) {
        chunk = std::min(chunk, std::max<long long>(1024, budget / row_bytes));
        if (row_bytes * h.n_pairs >= (32LL << 20)) chunk = std::min(chunk, (h.n_pairs + 3) / 4);
        if (stage[0]) chunk = std::min(chunk, static_cast<long long>(PinnedStage::kSlotBytes) / row_bytes);
    }
    double* dbuf[2] = {arena.alloc<double>(std::max<long long>(1, cols * 2 * chunk)),
                       chunk < h.n_pairs ? arena.alloc<double>(std::max<long long>(1, cols * 2 * chunk)) : nullptr};
    Stream s0, s1;
    const cudaStream_t sts[2] = {s0.get(), s1.get()};
    std::vector<cudaEvent_t> evs;
    auto event = [&]() {
        cudaEvent_t e;
        check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        evs.push_back(e);
        return e;
    };
    struct Done {
        std::vector<cudaEvent_t>& v;
        ~Done() {
            for (cudaEvent_t e : v) cudaEventDestroy(e);
        }
    } done{evs};
    const long long n_chunks = (h.n_pairs + chunk - 1) / chunk;
    std::vector<cudaEvent_t> k0(n_chunks), k1(n_chunks), staged(n_chunks);
    // with the staging: chunk c's columns into slot c % 2 on its stream (after its kernel) ...
    auto stage_chunk = [&](long long c) {
        const long long mcount = std::min(chunk, h.n_pairs - c * chunk);
        check_cuda(cudaMemcpyAsync(stage[c % 2], dbuf[c % 2], static_cast<size_t>(cols * 2 * mcount) * sizeof(double),
                                   cudaMemcpyDeviceToHost, sts[c % 2]),
                   "cudaMemcpyAsync (columns)");
        staged[c] = event();
        check_cuda(cudaEventRecord(staged[c], sts[c % 2]), "cudaEventRecord");
    };
    // ... then spread by the host threads into the caller's array: column a of the chunk holds its rows of leg 0, then
    // those of leg 1; each leg's run is cut into pieces of kPiece doubles, the pool's items
    auto spread_chunk = [&](long long c) {
        check_cuda(cudaEventSynchronize(staged[c]), "cudaEventSynchronize");
        const long long c0 = c * chunk, mcount = std::min(chunk, h.n_pairs - c0);
        constexpr long long kPiece = 1 << 16;
        const long long pieces = (mcount + kPiece - 1) / kPiece;
        const double* src = stage[c % 2];
        double* out = h.out;
        const long long P = h.n_pairs;
        HostPool::get().run(static_cast<int>(cols * 2 * pieces), [&](int item) {
            const long long col = item / (2 * pieces), leg = (item / pieces) % 2, q = item % pieces;
            const long long r0 = q * kPiece, r1 = std::min(mcount, r0 + kPiece);
            std::memcpy(out + col * 2 * P + leg * P + c0 + r0, src + col * 2 * mcount + leg * mcount + r0,
                        static_cast<size_t>(r1 - r0) * sizeof(double));
        });
    };
    auto copy_back = [&](long long c) {
        if (cols <= 0) return;
        if (stage[0]) {
            spread_chunk(c);
            return;
        }
        const long long c0 = c * chunk, mcount = std::min(chunk, h.n_pairs - c0);
        const double* src = dbuf[c % 2];
        const size_t width = static_cast<size_t>(mcount) * sizeof(double);
        const size_t spitch = static_cast<size_t>(2 * mcount) * sizeof(double);
        const size_t dpitch = static_cast<size_t>(2 * h.n_pairs) * sizeof(double);
        check_cuda(cudaMemcpy2DAsync(h.out + c0, dpitch, src, spitch, width, cols, cudaMemcpyDeviceToHost, sts[c % 2]),
                   "cudaMemcpy2D (leg 0)");
        check_cuda(cudaMemcpy2DAsync(h.out + h.n_pairs + c0, dpitch, src + mcount, spitch, width, cols,
                                     cudaMemcpyDeviceToHost, sts[c % 2]),
                   "cudaMemcpy2D (leg 1)");
    };
    for (long long c = 0; c < n_chunks; ++c) {
        const long long c0 = c * chunk, mcount = std::min(chunk, h.n_pairs - c0);
        const cudaStream_t st = sts[c % 2];
        double* out = dbuf[c % 2];
        PathsDev<R> part = s;
        part.n_pairs = mcount, part.first_pair = h.first_pair + c0, part.rows = 2 * mcount, part.out = out;
        const int block = 256;
        const unsigned grid = static_cast<unsigned>((mcount + block - 1) / block);
        k0[c] = event(), k1[c] = event();
        // one kernel at a time (its timing is its own); only the copies overlap them
        if (c > 0) check_cuda(cudaStreamWaitEvent(st, k1[c - 1], 0), "cudaStreamWaitEvent");
        check_cuda(cudaEventRecord(k0[c], st), "cudaEventRecord");
        if (fast) {
            PathsLvArgs<R> la = lv;
            la.n_pairs = mcount, la.first_pair = h.first_pair + c0, la.rows = 2 * mcount, la.out = out;
            const int lb = lv_block_of(n);
            const unsigned g = static_cast<unsigned>(std::max<long long>(
                1, std::min<long long>(lv_grid, (mcount + lb - 1) / lb)));
            reinterpret_cast<void (*)(PathsLvArgs<R>)>(const_cast<void*>(lv_fn))<<<g, lb, la.smem_blob, st>>>(la);
        } else if (n <= 1) paths_kernel<R, 1><<<grid, block, 0, st>>>(part);
        else if (n <= 2) paths_kernel<R, 2><<<grid, block, 0, st>>>(part);
        else if (n <= 4) paths_kernel<R, 4><<<grid, block, 0, st>>>(part);
        else paths_kernel<R, 8><<<grid, block, 0, st>>>(part);
        check_cuda(cudaGetLastError(), "paths_kernel launch");
        check_cuda(cudaEventRecord(k1[c], st), "cudaEventRecord");
        if (cols > 0 && stage[0]) stage_chunk(c);
        if (c > 0) copy_back(c - 1);  // the host waits for it while chunk c runs on the other stream
    }
    copy_back(n_chunks - 1);
    check_cuda(cudaStreamSynchronize(sts[0]), "paths");
    check_cuda(cudaStreamSynchronize(sts[1]), "paths");
    float kernel_ms = 0.0f;
    for (long long c = 0; c < n_chunks; ++c) {
        float ms = 0.0f;
        check_cuda(cudaEventElapsedTime(&ms, k0[c], k1[c]), "cudaEventElapsedTime");
        kernel_ms += ms;
    }
    h.kernel_ms = kernel_ms;
    h.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
}

}  // namespace
}  // namespace ob

extern "C" int ob_paths(ob_paths_request* rq, int precision) {
    return ob::guarded([&] {
        if (!rq) ob::invalid("null request");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        ob::check_request(*rq);
        if (precision == OB_FP32) ob::run_paths<float>(*rq);
        else ob::run_paths<double>(*rq);
    });
}
