// Pathwise (adjoint) Greeks of an autocall under correlated local vol: delta per name and the gradient of the price
// with respect to every entry of the local-variance tables, from which node vegas follow by the chain rule.
//
// The payoff is the reference's autocall script evaluated with smoothed digitals, as its risk engine does for Greeks
// (packages/structured/src/optlab/structured/script/evaluator.py:93-107: a condition a >= b becomes the ramp
// clip((a - b) / (eps |b|) + 1/2, 0, 1); inside an `if` a payment is weighted by the mask and `terminate` multiplies
// `alive` by one minus it; packages/risk/src/optlab/risk/greeks.py:430 uses eps = 0.005), so that its pathwise
// derivative exists. The dynamics are the path engine's local-vol step (RC/include/optlab_cuda/paths.hpp:341-356).
//
// adj_forward   one thread per antithetic pair: simulates both legs (all names), keeps each observation's worst
//               log-performance and which name set it, the lowest worst log-performance over the step ends (the
//               daily knock-in) and where it was; stores the state every kCk steps (the checkpoints); at the end
//               runs the payoff and its reverse sweep, giving dV/d(log perf) at each observation and at the knock-in
//               minimum. Spot moves the whole path's log-performance (local vol in log-moneyness, the reference's
//               spot shocks scaling paths: packages/risk/src/optlab/risk/engine.py:563-598), so the deltas are the
//               sums of those sensitivities per name, divided by the spot.
// adj_backward  one thread per pair again, segments of kCk steps from the last to the first: restart from the
//               checkpoint, recompute the segment's states and normals, then walk it backwards carrying dV/dx per
//               name and leg, injecting the observation sensitivities where they were taken, and adding
//               dV/d(variance) x (1 - w, w) into the two table entries each step read. Each block adds into its own
//               copy of the whole table's gradient (every name's rows; float in the float build, double in the
//               double one) in global memory, small enough to stay in L2 (148 x 2 blocks x 120 x 200 floats =
//               28 MB), by reductions that return nothing: the float add of a shared-memory atomic is a
//               compare-and-swap loop, a global reduction is one instruction the warp does not wait for (the
//               backward took half the time with it). At the end the block adds its copy into the caller's
//               per-batch gradient.
// adj_backward_dense  the same reverse sweep, one leg a thread, when the forward stored the state after every step
//               (when those states fit in the dense budget): nothing is recomputed. A step from x to x' read the variance v at x
//               and moved by v (-dt/2) + sqrt(v dt) z, so its noise term is d = x' - x - v (-dt/2) and
//               dx'/dv = -dt/2 + d / (2 v): no normals are drawn again. Each segment's states are loaded while
//               the previous segment is swept (two register buffers).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "mc.cuh"

namespace ob {

namespace {

constexpr int kCk = 4;        // steps per checkpoint segment (a multiple of every normal batch: 4, 2 or 1 steps)
constexpr int kMaxObs = 64;   // observations of one product
constexpr int kAdjBatches = OB_ADJ_BATCHES;

template <typename R>
struct AdjArgs {
    int n_names, n_steps, n_obs, n_x, n_rows, n_seg;
    int n_ck;                  // states stored by the forward: every kCk-th step but the last segment's, or all
    long long n_pairs;
    uint32_t k0, k1;
    const StepRec<R>* steps;   // n_steps
    const NameStep<R>* ns;     // n_steps x n_names
    const R* root;             // n x n
    const Pair2<R>* table;     // n_rows x (n_x - 1): (y_i, y_i+1 - y_i)
    const R* trig;             // n_obs, in performance (<= 0: no call)
    const double* disc;        // n_obs
    R top, cb, ki, put_strike, eps;
    double coupon;
    int memory, has_coupon, ki_daily;
    // forward outputs, backward inputs
    R* ckpt;                   // n_ck x n x 2 x n_pairs: x at grid points CK, 2 CK, ... (CK = kCk, or 1 when dense)
    R* dobs;                   // n_obs x 2 x n_pairs: d(pair value) / d(log perf) at each observation
    unsigned char* who;        // n_obs x 2 x n_pairs: the name that was the worst there
    R* dki;                    // 2 x n_pairs: d(pair value) / d(lowest log perf)
    int* ki_step;              // 2 x n_pairs
    unsigned char* ki_name;    // 2 x n_pairs
    double* partial;           // per block: price sum and square, then per name delta sum and square
    double* grad;              // kAdjBatches x n_rows x n_x
    R* priv;                   // per backward block: (left, right) weights of each table interval, n_rows x (n_x - 1)
                               // pairs, zeroed before each backward
    unsigned long long* batch_pairs;  // kAdjBatches
};

// The reference's smoothed comparisons: (value, derivative with respect to a).
template <typename R>
__device__ __forceinline__ R ramp_ge(R a, R b, R eps, R& d) {
    if (eps <= R(0)) {
        d = R(0);
        return a >= b ? R(1) : R(0);
    }
    const R s = eps * fabs(b), t = (a - b) / s + R(0.5);
    d = (t > R(0) && t < R(1)) ? R(1) / s : R(0);
    return m_min(m_max(t, R(0)), R(1));
}
template <typename R>
__device__ __forceinline__ R ramp_lt(R a, R b, R eps, R& d) {
    if (eps <= R(0)) {
        d = R(0);
        return a < b ? R(1) : R(0);
    }
    const R s = eps * fabs(b), t = (b - a) / s + R(0.5);
    d = (t > R(0) && t < R(1)) ? -R(1) / s : R(0);
    return m_min(m_max(t, R(0)), R(1));
}

// The Phoenix script of packages/structured/src/optlab/structured/compiler.py:114-161,271-280 on one leg, smoothed:
// per observation j (performance p = exp(lp[j])) a coupon cpn (1 + missed) weighted by c = ramp(p >= cb) and the
// alive mass, missed = (1 - c)(missed + 1); then, before the last date, the call: N weighted by q = ramp(p >= trigger)
// and alive *= 1 - q; on the last date the redemption N (1 - k max(K - p, 0)) with k = ramp(low < ki) (the lowest
// daily performance, or p itself for a knock-in at maturity). Returns the value; with grad, lp[j] becomes dV/dlp[j]
// and dlow dV/d(lowest log perf).
template <typename R>
__device__ double smooth_autocall(const AdjArgs<R>& a, R* lp, R lowlp, bool grad, R& dlow) {
    const int J = a.n_obs;
    R alive_at[kMaxObs], missed_at[kMaxObs];
    double pv = 0.0;
    R al = R(1), mi = R(0), d;
    const R low = m_exp(lowlp);
    for (int j = 0; j < J; ++j) {
        alive_at[j] = al, missed_at[j] = mi;
        const R p = m_exp(lp[j]);
        const double D = a.disc[j];
        if (a.has_coupon) {
            const R c = ramp_ge(p, a.cb, a.eps, d);
            const R mult = a.memory ? R(1) + mi : R(1);
            pv += D * a.coupon * static_cast<double>(mult * c * al);
            mi = a.memory ? (R(1) - c) * (mi + R(1)) : R(0);
        }
        if (j < J - 1) {
            const R q = a.trig[j] > R(0) ? ramp_ge(p, a.trig[j], a.eps, d) : R(0);
            pv += D * static_cast<double>(q * al);
            al *= R(1) - q;
        } else {
            const R k = ramp_lt(a.ki_daily ? low : p, a.ki, a.eps, d);
            const R put = m_max(a.put_strike - p, R(0));
            pv += D * static_cast<double>(al * (R(1) - k * put));
        }
    }
    dlow = R(0);
    if (!grad) return pv;
    R abar = R(0), mbar = R(0);
    for (int j = J - 1; j >= 0; --j) {
        const R al_j = alive_at[j], mi_j = missed_at[j];
        const R p = m_exp(lp[j]);
        const R D = static_cast<R>(a.disc[j]);
        R pbar = R(0), abar_new = R(0), mbar_new = R(0);
        if (j < J - 1) {
            R dq = R(0);
            const R q = a.trig[j] > R(0) ? ramp_ge(p, a.trig[j], a.eps, dq) : R(0);
            const R qbar = D * al_j - abar * al_j;
            abar_new += D * q + abar * (R(1) - q);
            pbar += qbar * dq;
        } else {
            R dk;
            const R k = ramp_lt(a.ki_daily ? low : p, a.ki, a.eps, dk);
            const R put = m_max(a.put_strike - p, R(0));
            abar_new += D * (R(1) - k * put);
            const R kbar = -D * al_j * put;
            if (a.put_strike > p) pbar += D * al_j * k;  // d/dp of -k max(K - p, 0)
            if (a.ki_daily) dlow += kbar * dk * low;
            else pbar += kbar * dk;
        }
        if (a.has_coupon) {
            R dc;
            const R c = ramp_ge(p, a.cb, a.eps, dc);
            const R cpn = static_cast<R>(a.coupon);
            const R mult = a.memory ? R(1) + mi_j : R(1);
            const R cbar = D * cpn * mult * al_j - (a.memory ? mbar * (mi_j + R(1)) : R(0));
            abar_new += D * cpn * mult * c;
            mbar_new = a.memory ? D * cpn * c * al_j + mbar * (R(1) - c) : R(0);
            pbar += cbar * dc;
        }
        abar = abar_new, mbar = mbar_new;
        lp[j] = pbar * p;
    }
    return pv;
}

// One local-vol step of one leg of name n from x: the new x, with the interpolation kept for the adjoint.
template <typename R>
struct LvStep {
    R var;    // interpolated local variance
    R dvdx;   // its slope in x (0 where the interpolation is clamped)
    R w;      // weight of the right table point
    int idx;  // index of the (y_i, dy_i) pair: row offset + i
};

// GLOBAL: tab is the table in global memory, read through the read-only data cache (never a staged copy in shared
// memory).
template <bool GLOBAL, typename R>
__device__ __forceinline__ LvStep<R> lv_read(const AdjArgs<R>& a, const Pair2<R>* tab, const NameStep<R>& ns, R x) {
    LvStep<R> s;
    R u = table_u(ns, x);
    const bool inside = u > R(0) && u < a.top;
    u = m_min(m_max(u, R(0)), a.top);
    const int j = static_cast<int>(u);
    s.w = u - static_cast<R>(j);
    s.idx = ns.row + j;
    const Pair2<R> y = GLOBAL ? ldg_pair(tab + s.idx) : tab[s.idx];
    s.var = y.a + s.w * y.b;
    s.dvdx = inside ? y.b * ns.inv_dx : R(0);
    return s;
}

// ST (float tables up to kStageBytes): the whole table staged in the block's shared memory, read there by every step
// of the forward pass (1024-thread blocks, one an SM, so the warps stay as many); otherwise read from global memory
// through L1.
constexpr size_t kStageBytes = 200u << 10;

template <typename R, bool ST>
__device__ __forceinline__ const Pair2<R>* stage_table(const AdjArgs<R>& a, unsigned char* dyn) {
    if (!ST) return a.table;
    const int n16 = a.n_rows * (a.n_x - 1) * static_cast<int>(sizeof(Pair2<R>)) / 16;
    const int4* src = reinterpret_cast<const int4*>(a.table);
    int4* dst = reinterpret_cast<int4*>(dyn);
    for (int k = threadIdx.x; k < n16; k += blockDim.x) dst[k] = __ldg(src + k);
    if (threadIdx.x == 0 && (a.n_rows * (a.n_x - 1)) % 2)  // an odd count of 8-byte float pairs: the last one
        reinterpret_cast<Pair2<R>*>(dyn)[a.n_rows * (a.n_x - 1) - 1] = a.table[a.n_rows * (a.n_x - 1) - 1];
    __syncthreads();
    return reinterpret_cast<const Pair2<R>*>(dyn);
}

template <int N>
struct Batch {
    static constexpr int C = N;
    static constexpr int G = C % 4 == 0 ? 1 : (C % 2 == 0 ? 2 : 4);  // steps per batch of whole Philox blocks
    static constexpr int NB = C * G / 4;
};

// The correlated normals of the G steps of batch b: zc[g][n] (the first leg's; the second leg reads -zc).
template <typename R, int N>
__device__ __forceinline__ void batch_normals(const AdjArgs<R>& a, uint64_t pair, int b, R (&zc)[Batch<N>::G][N]) {
    constexpr int G = Batch<N>::G, NB = Batch<N>::NB;
    R z[N * G];
#pragma unroll
    for (int k = 0; k < NB; ++k)
        normals4<R>(pair, static_cast<uint64_t>(b) * NB + k, 0u, a.k0, a.k1, z[4 * k], z[4 * k + 1], z[4 * k + 2],
                    z[4 * k + 3]);
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int n = 0; n < N; ++n) {
            R acc = R(0);
#pragma unroll
            for (int m = 0; m < N; ++m) acc += a.root[n * N + m] * z[g * N + m];
            zc[g][n] = acc;
        }
}

template <typename R, int N, bool STORE, int CK, bool ST>
__global__ void __launch_bounds__(ST ? 1024 : 256) adj_forward(AdjArgs<R> a) {
    constexpr int G = Batch<N>::G;
    __shared__ double wacc[32][2 + 2 * N];
    extern __shared__ __align__(16) unsigned char dyn[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < 32 * (2 + 2 * N); t += blockDim.x) (&wacc[0][0])[t] = 0.0;
    const Pair2<R>* tab = stage_table<R, ST>(a, dyn);
    __syncthreads();
    const long long P = a.n_pairs;
    const R rtop = R(1) / a.top;  // (float rows scaled to the cell form)
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < P;
         base += stride) {
        const bool active = base + lane < P;
        const long long p = active ? base + lane : P - 1;
        const uint64_t pair = static_cast<uint64_t>(p);
        R x[2][N];
#pragma unroll
        for (int n = 0; n < N; ++n) x[0][n] = x[1][n] = R(0);
        R lpo[2][kMaxObs];
        unsigned char wo[2][kMaxObs];
        R low[2] = {R(0), R(0)};  // the worst log performance at t = 0 is 0
        int lstep[2] = {0, 0}, lname[2] = {0, 0};
        for (int i0 = 1, b = 0; i0 <= a.n_steps; i0 += G, ++b) {
            R zc[G][N];
            batch_normals<R, N>(a, pair, b, zc);
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int i = i0 + g;
                if (G > 1 && i > a.n_steps) break;
                const StepRec<R> st = ldg_rec(a.steps + i - 1);
                R wv[2] = {R(1e30), R(1e30)};
                int wn[2] = {0, 0};
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    const NameStep<R> ns = ldg_rec(a.ns + (i - 1) * N + n);
                    // float: the fused kernel's step (the row in the cell form, scaled here once for both legs; the
                    // log-spot step as two multiply-adds); double: the reference's grouping, as the backward reads it
                    R org_c = ns.org, inv_c = ns.inv_dx;
                    if constexpr (sizeof(R) == 4) org_c *= rtop, inv_c *= rtop;
                    const R zd = st.sdt * zc[g][n];
#pragma unroll
                    for (int leg = 0; leg < 2; ++leg) {
                        if constexpr (sizeof(R) == 4) {
                            int j;
                            R f;
                            table_cell(org_c, inv_c, a.top, x[leg][n], j, f);
                            const Pair2<R> y = !ST ? ldg_pair(tab + ns.row + j) : tab[ns.row + j];
                            x[leg][n] = lv_advance(x[leg][n], y.a + f * y.b, st.hdt, leg ? -zd : zd);
                        } else {
                            const R z = leg ? -zc[g][n] : zc[g][n];
                            const LvStep<R> s = lv_read<!ST>(a, tab, ns, x[leg][n]);
                            x[leg][n] += s.var * st.hdt + (m_sqrt(s.var) * st.sdt) * z;
                        }
                        const R lp = x[leg][n] + ns.lf;
                        if (lp < wv[leg]) wv[leg] = lp, wn[leg] = n;
                    }
                }
#pragma unroll
                for (int leg = 0; leg < 2; ++leg) {
                    if (wv[leg] < low[leg]) low[leg] = wv[leg], lstep[leg] = i, lname[leg] = wn[leg];
                    if (st.obs >= 0) lpo[leg][st.obs] = wv[leg], wo[leg][st.obs] = static_cast<unsigned char>(wn[leg]);
                }
                if (STORE && i % CK == 0 && i / CK <= a.n_ck && active) {
                    const long long c = i / CK - 1;
#pragma unroll
                    for (int n = 0; n < N; ++n)
#pragma unroll
                        for (int leg = 0; leg < 2; ++leg)
                            a.ckpt[((c * N + n) * 2 + leg) * P + p] = x[leg][n];
                }
            }
        }
        // payoff, its reverse sweep, the injections and the deltas
        double v[2], dl[2][N];
        for (int leg = 0; leg < 2; ++leg) {
            R dlow;
            v[leg] = smooth_autocall(a, lpo[leg], low[leg], true, dlow);
#pragma unroll
            for (int n = 0; n < N; ++n) dl[leg][n] = 0.0;
            for (int j = 0; j < a.n_obs; ++j) {
#pragma unroll
                for (int n = 0; n < N; ++n)
                    if (wo[leg][j] == n) dl[leg][n] += static_cast<double>(lpo[leg][j]);
                if (STORE && active) {
                    a.dobs[(static_cast<long long>(j) * 2 + leg) * P + p] = R(0.5) * lpo[leg][j];
                    a.who[(static_cast<long long>(j) * 2 + leg) * P + p] = wo[leg][j];
                }
            }
#pragma unroll
            for (int n = 0; n < N; ++n)
                if (lname[leg] == n) dl[leg][n] += static_cast<double>(dlow);
            if (STORE && active) {
                a.dki[static_cast<long long>(leg) * P + p] = R(0.5) * dlow;
                a.ki_step[static_cast<long long>(leg) * P + p] = lstep[leg];
                a.ki_name[static_cast<long long>(leg) * P + p] = static_cast<unsigned char>(lname[leg]);
            }
        }
        double y[2 + 2 * N];
        const double val = active ? 0.5 * (v[0] + v[1]) : 0.0;
        y[0] = val, y[1] = val * val;
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const double dn = active ? 0.5 * (dl[0][n] + dl[1][n]) : 0.0;
            y[2 + 2 * n] = dn, y[3 + 2 * n] = dn * dn;
        }
#pragma unroll
        for (int k = 0; k < 2 + 2 * N; ++k) {
            const double s = warp_sum(y[k]);
            if (lane == 0) wacc[warp][k] += s;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 + 2 * N; t += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += wacc[w][t];
        a.partial[static_cast<long long>(blockIdx.x) * (2 + 2 * N) + t] = s;
    }
}

// A step's gradient into the block's copy: interval idx of a row receives vb (1 - w) for its left point and vb w for
// its right one, as one 8-byte reduction in float (half the reduction operations of two scalar ones: the L2's atomic
// rate bounds the backward), two in double. The result is unused: no return value is waited for.
__device__ __forceinline__ void cell_add(float* cell, float left, float right) {
    atomicAdd(reinterpret_cast<float2*>(cell), make_float2(left, right));
}
__device__ __forceinline__ void cell_add(double* cell, double left, double right) {
    atomicAdd(cell, left);
    atomicAdd(cell + 1, right);
}

// The block's gradient copy added into the caller's gradient of batch blockIdx % kAdjBatches (entry k of a row: the
// left weight of interval k plus the right weight of interval k - 1), and its pair count.
template <typename R>
__device__ __forceinline__ void flush_gradient(const AdjArgs<R>& a, const R* sg, unsigned long long mine) {
    __syncthreads();
    const int nx = a.n_x, tab_n = a.n_rows * nx;
    const int batch = blockIdx.x % kAdjBatches;
    double* out = a.grad + static_cast<long long>(batch) * tab_n;
    for (int t = threadIdx.x; t < tab_n; t += blockDim.x) {
        const int row = t / nx, k = t - row * nx;
        const R* cells = sg + 2 * static_cast<long long>(row) * (nx - 1);  // from L2, where the reductions were made
        double v = 0.0;
        if (k < nx - 1) v += static_cast<double>(__ldcg(cells + 2 * k));
        if (k > 0) v += static_cast<double>(__ldcg(cells + 2 * (k - 1) + 1));
        if (v != 0.0) atomicAdd(out + t, v);
    }
    __shared__ unsigned long long s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    atomicAdd(&s_cnt, mine);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(a.batch_pairs + batch, s_cnt);
}

template <typename R, int N>
__global__ void __launch_bounds__(256) adj_backward(AdjArgs<R> a) {
    constexpr int G = Batch<N>::G;
    using GT = R;  // gradient accumulators: float in the float build, double in the double one
    GT* sg = a.priv + 2 * static_cast<long long>(blockIdx.x) * a.n_rows * (a.n_x - 1);
    const Pair2<R>* tab = a.table;
    const int lane = threadIdx.x & 31;
    const long long P = a.n_pairs;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    unsigned long long mine = 0;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < P;
         base += stride) {
        const bool active = base + lane < P;
        if (!active) continue;  // no block-wide synchronisation below: inactive lanes may leave
        const long long p = base + lane;
        ++mine;
        const uint64_t pair = static_cast<uint64_t>(p);
        const int kstep[2] = {__ldg(a.ki_step + p), __ldg(a.ki_step + P + p)};
        const int kname[2] = {__ldg(a.ki_name + p), __ldg(a.ki_name + P + p)};
        const R kd[2] = {__ldg(a.dki + p), __ldg(a.dki + P + p)};
        R xb[2][N];
#pragma unroll
        for (int n = 0; n < N; ++n) xb[0][n] = xb[1][n] = R(0);
        for (int s = a.n_seg - 1; s >= 0; --s) {
            const int i_first = s * kCk + 1;
            const int len = min(kCk, a.n_steps - s * kCk);
            R xs[kCk + 1][2][N];
#pragma unroll
            for (int n = 0; n < N; ++n)
#pragma unroll
                for (int leg = 0; leg < 2; ++leg)
                    xs[0][leg][n] =
                        s == 0 ? R(0) : __ldg(a.ckpt + ((static_cast<long long>(s - 1) * N + n) * 2 + leg) * P + p);
            R zc[kCk][N];
#pragma unroll
            for (int bb = 0; bb < kCk / G; ++bb) {
                R zb[G][N];
                batch_normals<R, N>(a, pair, (s * kCk) / G + bb, zb);
#pragma unroll
                for (int g = 0; g < G; ++g)
#pragma unroll
                    for (int n = 0; n < N; ++n) zc[bb * G + g][n] = zb[g][n];
            }
            // forward through the segment
#pragma unroll
            for (int g = 0; g < kCk; ++g) {
                if (g >= len) break;
                const StepRec<R> st = ldg_rec(a.steps + i_first + g - 1);
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    const NameStep<R> ns = ldg_rec(a.ns + (i_first + g - 1) * N + n);
#pragma unroll
                    for (int leg = 0; leg < 2; ++leg) {
                        const R z = leg ? -zc[g][n] : zc[g][n];
                        const LvStep<R> r = lv_read<true>(a, tab, ns, xs[g][leg][n]);
                        xs[g + 1][leg][n] = xs[g][leg][n] + r.var * st.hdt + (m_sqrt(r.var) * st.sdt) * z;
                    }
                }
            }
            // backwards through the segment: step i = i_first + g takes grid point i - 1 to grid point i
#pragma unroll
            for (int g = kCk - 1; g >= 0; --g) {
                if (g >= len) continue;
                const int i = i_first + g;
                const StepRec<R> st = ldg_rec(a.steps + i - 1);
                // the payoff's sensitivities at grid point i
                if (st.obs >= 0) {
#pragma unroll
                    for (int leg = 0; leg < 2; ++leg) {
                        const long long o = (static_cast<long long>(st.obs) * 2 + leg) * P + p;
                        const R d = __ldg(a.dobs + o);
                        const int w = __ldg(a.who + o);
#pragma unroll
                        for (int n = 0; n < N; ++n)
                            if (w == n) xb[leg][n] += d;
                    }
                }
#pragma unroll
                for (int leg = 0; leg < 2; ++leg)
                    if (kstep[leg] == i) {
#pragma unroll
                        for (int n = 0; n < N; ++n)
                            if (kname[leg] == n) xb[leg][n] += kd[leg];
                    }
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    const NameStep<R> ns = ldg_rec(a.ns + (i - 1) * N + n);
#pragma unroll
                    for (int leg = 0; leg < 2; ++leg) {
                        const R z = leg ? -zc[g][n] : zc[g][n];
                        const LvStep<R> r = lv_read<true>(a, tab, ns, xs[g][leg][n]);
                        const R sv = m_sqrt(r.var);
                        const R c = st.hdt + st.sdt * z / (R(2) * sv);  // d x_i / d var
                        const R vb = xb[leg][n] * c;
                        if (vb != R(0)) cell_add(sg + 2 * r.idx, vb * (R(1) - r.w), vb * r.w);
                        xb[leg][n] += vb * r.dvdx;
                    }
                }
            }
        }
    }
    flush_gradient(a, sg, mine);  // pairs of this block: the count of each batch makes its mean
}

template <typename R, int N>
__device__ __forceinline__ void dense_segment(const AdjArgs<R>& a, long long p, int leg, int s, R (&xs)[kCk + 1][N]) {
    const long long P = a.n_pairs;
#pragma unroll
    for (int g = 0; g <= kCk; ++g) {
        const int i = s * kCk + g;  // grid point
        if (i > a.n_steps) break;
#pragma unroll
        for (int n = 0; n < N; ++n)
            xs[g][n] = i == 0 ? R(0) : __ldg(a.ckpt + ((static_cast<long long>(i - 1) * N + n) * 2 + leg) * P + p);
    }
}

// One leg a warp: warps 2k and 2k + 1 of a block take the two legs of the same 32 pairs (so a pair's gradient stays
// in one block's batch). Half the state of a pair a thread, so more warps fit an SM to hide the states' loads.
template <typename R, int N>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 3 : 1) adj_backward_dense(AdjArgs<R> a) {
    using GT = R;
    GT* sg = a.priv + 2 * static_cast<long long>(blockIdx.x) * a.n_rows * (a.n_x - 1);
    const Pair2<R>* tab = a.table;  // (staging it in shared memory measured no faster: the state loads bound it)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, leg = warp & 1;
    const int chunks_per_block = blockDim.x >> 6;  // pairs of warps
    const long long P = a.n_pairs;
    const long long n_chunks = (P + 31) / 32;
    unsigned long long mine = 0;
    for (long long c = static_cast<long long>(blockIdx.x) * chunks_per_block + (warp >> 1); c < n_chunks;
         c += static_cast<long long>(gridDim.x) * chunks_per_block) {
        const long long p = c * 32 + lane;
        if (p >= P) continue;  // no block-wide synchronisation below: inactive lanes may leave
        if (leg == 0) ++mine;
        const int kstep = __ldg(a.ki_step + leg * P + p);
        const int kname = __ldg(a.ki_name + leg * P + p);
        const R kd = __ldg(a.dki + leg * P + p);
        R xb[N];
#pragma unroll
        for (int n = 0; n < N; ++n) xb[n] = R(0);
        R cur[kCk + 1][N], nxt[kCk + 1][N];
        dense_segment<R, N>(a, p, leg, a.n_seg - 1, cur);
        for (int s = a.n_seg - 1; s >= 0; --s) {
            if (s > 0) dense_segment<R, N>(a, p, leg, s - 1, nxt);
            const int i_first = s * kCk + 1;
            const int len = min(kCk, a.n_steps - s * kCk);
#pragma unroll
            for (int g = kCk - 1; g >= 0; --g) {
                if (g >= len) continue;
                const int i = i_first + g;
                const StepRec<R> st = ldg_rec(a.steps + i - 1);
                if (st.obs >= 0) {
                    const long long o = (static_cast<long long>(st.obs) * 2 + leg) * P + p;
                    const R d = __ldg(a.dobs + o);
                    const int w = __ldg(a.who + o);
#pragma unroll
                    for (int n = 0; n < N; ++n)
                        if (w == n) xb[n] += d;
                }
                if (kstep == i) {
#pragma unroll
                    for (int n = 0; n < N; ++n)
                        if (kname == n) xb[n] += kd;
                }
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    const NameStep<R> ns = ldg_rec(a.ns + (i - 1) * N + n);
                    const LvStep<R> r = lv_read<true>(a, tab, ns, cur[g][n]);
                    const R d = cur[g + 1][n] - cur[g][n] - r.var * st.hdt;  // sqrt(v dt) z
                    const R cc = st.hdt + d / (R(2) * r.var);               // d x_i / d var
                    const R vb = xb[n] * cc;
                    if (vb != R(0)) cell_add(sg + 2 * r.idx, vb * (R(1) - r.w), vb * r.w);
                    xb[n] += vb * r.dvdx;
                }
            }
#pragma unroll
            for (int g = 0; g <= kCk; ++g)
#pragma unroll
                for (int n = 0; n < N; ++n) cur[g][n] = nxt[g][n];
        }
    }
    flush_gradient(a, sg, mine);
}

// (y_i, y_i+1 - y_i) pairs of the caller's FP64 table.
template <typename R>
__global__ void adj_table(const double* __restrict__ t, int n_rows, int n_x, Pair2<R>* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_rows * (n_x - 1)) return;
    const int row = k / (n_x - 1), i = k - row * (n_x - 1);
    const double y0 = t[row * n_x + i], y1 = t[row * n_x + i + 1];
    out[k].a = static_cast<R>(y0);
    out[k].b = static_cast<R>(y1 - y0);
}

}  // namespace

struct AdjPlan {
    DeviceArena arena;
    int precision = OB_FP32, n = 1, sms = 0, n_out = 0;
    long long n_pairs = 0;
    int grid_f = 0, grid_b = 0;
    size_t priv_bytes = 0;
    AdjArgs<float> af{};
    AdjArgs<double> ad{};
    double spot[OB_MAX_NAMES] = {};
    const void *kf = nullptr, *kfs = nullptr, *kb = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
    bool backward = false;
    cudaStream_t last = nullptr;
    int tab_n = 0;
    bool dense = false;  // the forward stores every step's state and the backward recomputes nothing
    bool staged = false; // the table is staged in shared memory (float tables up to kStageBytes)
    int block_f = 256, block_b = 256;
    size_t smem = 0;     // dynamic shared memory of the staged forward kernels

    template <typename R>
    AdjArgs<R>& args();
    template <typename R>
    void build(const ob_adjoint_request& rq);
    void run(const double* d_table, double* d_grad, cudaStream_t st);
    void result(ob_adjoint_result& res, long long* batch_pairs);
    ~AdjPlan() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (e2) cudaEventDestroy(e2);
    }
};
template <>
AdjArgs<float>& AdjPlan::args<float>() {
    return af;
}
template <>
AdjArgs<double>& AdjPlan::args<double>() {
    return ad;
}

namespace {

template <typename R, int N, bool ST>
void pick_st(AdjPlan& p) {
    p.kf = reinterpret_cast<const void*>(adj_forward<R, N, false, kCk, ST>);
    p.kfs = p.dense ? reinterpret_cast<const void*>(adj_forward<R, N, true, 1, ST>)
                    : reinterpret_cast<const void*>(adj_forward<R, N, true, kCk, ST>);
    p.kb = p.dense ? reinterpret_cast<const void*>(adj_backward_dense<R, N>)
                   : reinterpret_cast<const void*>(adj_backward<R, N>);
}

// Staged tables for float only (double tables of the benchmark's size do not fit a block's shared memory).
template <typename R, int N>
void pick(AdjPlan& p) {
    if (sizeof(R) == 4 && p.staged) pick_st<R, N, true>(p);
    else pick_st<R, N, false>(p);
}

constexpr double kDenseBudget = 24.0 * (1ull << 30);  // bytes of stored states below which every step is stored

void check_adjoint(const ob_adjoint_request& r) {
    const ob_mc_request& rq = r.base;
    check_mc_request(rq);
    if (rq.model != OB_MODEL_PATHS || rq.product != OB_PRODUCT_AUTOCALL)
        invalid("the adjoint prices an autocall under the path engine's local vol");
    if (rq.n_names > 4) invalid("the adjoint takes 1 to 4 names");
    if (rq.mixer) invalid("the adjoint takes no local correlation");
    for (int a = 0; a < rq.n_names; ++a)
        if (rq.kind[a] != 1) invalid("the adjoint needs every name in local vol (kind 1)");
    if (rq.n_obs > kMaxObs) invalid("the adjoint takes at most 64 observations");
    if (rq.first_pair != 0) invalid("the adjoint runs pairs 0 .. n_pairs - 1");
    if (!(r.smoothing >= 0.0 && r.smoothing < 1.0)) invalid("smoothing must be in [0, 1)");
    if (r.checkpoint != 0 && r.checkpoint != 1 && r.checkpoint != kCk) invalid("checkpoint must be 0, 1 or 4");
    if (rq.ki_barrier <= 0 || rq.coupon_barrier < 0) invalid("the adjoint needs a knock-in barrier above 0");
}

}  // namespace

template <typename R>
void AdjPlan::build(const ob_adjoint_request& r) {
    const ob_mc_request& rq = r.base;
    n = rq.n_names;
    const int S = rq.n_steps;
    AdjArgs<R>& a = args<R>();
    a = AdjArgs<R>{};
    a.n_names = n, a.n_steps = S, a.n_obs = rq.n_obs, a.n_x = rq.n_x, a.n_rows = rq.n_rows;
    a.n_seg = (S + kCk - 1) / kCk;
    a.n_pairs = rq.n_pairs;
    a.k0 = static_cast<uint32_t>(rq.seed), a.k1 = static_cast<uint32_t>(rq.seed >> 32);
    a.top = static_cast<R>(rq.n_x - 1) - static_cast<R>(1e-4);
    a.cb = static_cast<R>(rq.coupon_barrier), a.ki = static_cast<R>(rq.ki_barrier);
    a.put_strike = static_cast<R>(rq.put_strike), a.eps = static_cast<R>(r.smoothing);
    a.coupon = rq.coupon, a.memory = rq.memory, a.ki_daily = rq.ki_daily;
    a.has_coupon = rq.coupon > 0.0 || rq.coupon_barrier > 0.0;
    std::vector<StepRec<R>> steps(S);
    for (int i = 0; i < S; ++i) {
        std::memset(&steps[i], 0, sizeof steps[i]);
        steps[i].dt = static_cast<R>(rq.dt[i]);
        steps[i].hdt = static_cast<R>(-0.5 * rq.dt[i]);
        steps[i].sdt = static_cast<R>(std::sqrt(rq.dt[i]));
        steps[i].obs = -1;
    }
    for (int j = 0; j < rq.n_obs; ++j) steps[rq.obs_step[j] - 1].obs = j;
    std::vector<NameStep<R>> ns(static_cast<size_t>(S) * n);
    for (int i = 1; i <= S; ++i)
        for (int k = 0; k < n; ++k) {
            NameStep<R>& e = ns[static_cast<size_t>(i - 1) * n + k];
            std::memset(&e, 0, sizeof e);
            const int row = rq.step_row[static_cast<size_t>(k) * S + (i - 1)];
            e.org = name_step_org<R>(rq.row_lo[row], rq.row_inv_dx[row]);
            e.inv_dx = static_cast<R>(rq.row_inv_dx[row]);
            e.lf = static_cast<R>(rq.log_fwd[static_cast<size_t>(k) * (S + 1) + i]);
            e.row = row * (rq.n_x - 1);
        }
    std::vector<R> root(static_cast<size_t>(n) * n), trig(rq.n_obs);
    for (size_t k = 0; k < root.size(); ++k) root[k] = static_cast<R>(rq.root[k]);
    for (int j = 0; j < rq.n_obs; ++j) trig[j] = rq.trigger[j] > 0 ? static_cast<R>(rq.trigger[j]) : R(0);
    a.steps = arena.put<StepRec<R>>(steps.data(), steps.size());
    a.ns = arena.put<NameStep<R>>(ns.data(), ns.size());
    a.root = arena.put<R>(root.data(), root.size());
    a.trig = arena.put<R>(trig.data(), trig.size());
    a.disc = arena.put<double>(rq.obs_discount, rq.n_obs);
    Pair2<R>* tab = arena.alloc<Pair2<R>>(static_cast<size_t>(rq.n_rows) * (rq.n_x - 1));
    double* t64 = arena.put<double>(rq.table, static_cast<size_t>(rq.n_rows) * rq.n_x);
    const int cells = rq.n_rows * (rq.n_x - 1);
    adj_table<R><<<(cells + 255) / 256, 256>>>(t64, rq.n_rows, rq.n_x, tab);
    check_cuda(cudaGetLastError(), "adj_table launch");
    a.table = tab;
    const long long P = rq.n_pairs;
    const double dense_bytes = static_cast<double>(S) * n * 2 * P * sizeof(R);
    dense = r.checkpoint == 1 || (r.checkpoint == 0 && dense_bytes <= kDenseBudget);
    a.n_ck = dense ? S : a.n_seg - 1;
    a.ckpt = arena.alloc<R>(static_cast<size_t>(std::max(1, a.n_ck)) * n * 2 * P);
    a.dobs = arena.alloc<R>(static_cast<size_t>(rq.n_obs) * 2 * P);
    a.who = arena.alloc<unsigned char>(static_cast<size_t>(rq.n_obs) * 2 * P);
    a.dki = arena.alloc<R>(2 * static_cast<size_t>(P));
    a.ki_step = arena.alloc<int>(2 * static_cast<size_t>(P));
    a.ki_name = arena.alloc<unsigned char>(2 * static_cast<size_t>(P));
    a.batch_pairs = arena.alloc<unsigned long long>(kAdjBatches);
    const size_t tab_bytes = static_cast<size_t>(rq.n_rows) * (rq.n_x - 1) * sizeof(Pair2<R>);
    staged = sizeof(R) == 4 && tab_bytes <= kStageBytes;
    smem = staged ? tab_bytes : 0;
    block_f = staged ? 1024 : 256;
    switch (n) {
        case 1: pick<R, 1>(*this); break;
        case 2: pick<R, 2>(*this); break;
        case 3: pick<R, 3>(*this); break;
        default: pick<R, 4>(*this); break;
    }
    const size_t smem_b = 0;
    if (staged) {
        check_cuda(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                   "cudaFuncSetAttribute");
        check_cuda(cudaFuncSetAttribute(kfs, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                   "cudaFuncSetAttribute");
    }
    tab_n = rq.n_rows * rq.n_x;
    int per_f = 0, per_b = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_f, kfs, block_f, smem), "occupancy");
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_b, kb, block_b, smem_b), "occupancy");
    grid_f = static_cast<int>(std::max<long long>(
        1, std::min<long long>((P + block_f - 1) / block_f, static_cast<long long>(sms) * std::max(1, per_f))));
    const long long pairs_b = dense ? block_b / 2 : block_b;  // the dense backward takes one leg a thread
    grid_b = static_cast<int>(std::max<long long>(
        1, std::min<long long>((P + pairs_b - 1) / pairs_b, static_cast<long long>(sms) * std::max(1, per_b))));
    a.partial = arena.alloc<double>(static_cast<size_t>(grid_f) * (2 + 2 * n));
    const size_t cells2 = 2 * static_cast<size_t>(rq.n_rows) * (rq.n_x - 1);
    priv_bytes = static_cast<size_t>(grid_b) * cells2 * sizeof(R);
    a.priv = arena.alloc<R>(static_cast<size_t>(grid_b) * cells2);
    for (int k = 0; k < n; ++k) spot[k] = rq.spot[k];
}

template void AdjPlan::build<float>(const ob_adjoint_request&);
template void AdjPlan::build<double>(const ob_adjoint_request&);

void AdjPlan::run(const double* d_table, double* d_grad, cudaStream_t st) {
    const bool grad = d_grad != nullptr;
    check_cuda(cudaEventRecord(e0, st), "cudaEventRecord");
    if (precision == OB_FP32) {
        if (d_table) {
            const int cells = af.n_rows * (af.n_x - 1);
            adj_table<float><<<(cells + 255) / 256, 256, 0, st>>>(d_table, af.n_rows, af.n_x,
                                                                   const_cast<Pair2<float>*>(af.table));
        }
        af.grad = d_grad;
        using F = void (*)(AdjArgs<float>);
        reinterpret_cast<F>(const_cast<void*>(grad ? kfs : kf))<<<grid_f, block_f, smem, st>>>(af);
    } else {
        if (d_table) {
            const int cells = ad.n_rows * (ad.n_x - 1);
            adj_table<double><<<(cells + 255) / 256, 256, 0, st>>>(d_table, ad.n_rows, ad.n_x,
                                                                    const_cast<Pair2<double>*>(ad.table));
        }
        ad.grad = d_grad;
        using F = void (*)(AdjArgs<double>);
        reinterpret_cast<F>(const_cast<void*>(grad ? kfs : kf))<<<grid_f, block_f, smem, st>>>(ad);
    }
    check_cuda(cudaGetLastError(), "adj_forward launch");
    check_cuda(cudaEventRecord(e1, st), "cudaEventRecord");
    if (grad) {
        const size_t gbytes = static_cast<size_t>(kAdjBatches) * tab_n * sizeof(double);
        check_cuda(cudaMemsetAsync(d_grad, 0, gbytes, st), "cudaMemsetAsync");
        if (precision == OB_FP32) {
            check_cuda(cudaMemsetAsync(af.batch_pairs, 0, kAdjBatches * sizeof(unsigned long long), st), "memset");
            check_cuda(cudaMemsetAsync(af.priv, 0, priv_bytes, st), "cudaMemsetAsync");
            using B = void (*)(AdjArgs<float>);
            reinterpret_cast<B>(const_cast<void*>(kb))<<<grid_b, block_b, 0, st>>>(af);
        } else {
            check_cuda(cudaMemsetAsync(ad.batch_pairs, 0, kAdjBatches * sizeof(unsigned long long), st), "memset");
            check_cuda(cudaMemsetAsync(ad.priv, 0, priv_bytes, st), "cudaMemsetAsync");
            using B = void (*)(AdjArgs<double>);
            reinterpret_cast<B>(const_cast<void*>(kb))<<<grid_b, block_b, 0, st>>>(ad);
        }
        check_cuda(cudaGetLastError(), "adj_backward launch");
    }
    check_cuda(cudaEventRecord(e2, st), "cudaEventRecord");
    backward = grad;
    last = st;
}

void AdjPlan::result(ob_adjoint_result& res, long long* batch_pairs) {
    check_cuda(cudaStreamSynchronize(last), "adjoint");
    const int k = 2 + 2 * n;
    std::vector<double> part(static_cast<size_t>(grid_f) * k);
    const double* dp = precision == OB_FP32 ? af.partial : ad.partial;
    check_cuda(cudaMemcpy(part.data(), dp, part.size() * sizeof(double), cudaMemcpyDeviceToHost), "copy partials");
    std::vector<double> tot(k, 0.0);
    for (int b = 0; b < grid_f; ++b)
        for (int t = 0; t < k; ++t) tot[t] += part[static_cast<size_t>(b) * k + t];
    std::memset(&res, 0, sizeof res);
    const double nn = static_cast<double>(n_pairs);
    auto est = [&](double s, double s2, double& m, double& se) {
        m = s / nn;
        const double var = s2 / nn - m * m;
        se = n_pairs > 1 ? std::sqrt(std::fmax(var, 0.0) / (nn - 1.0)) : 0.0;
    };
    est(tot[0], tot[1], res.price, res.price_se);
    for (int a = 0; a < n; ++a) {
        double m, se;
        est(tot[2 + 2 * a], tot[3 + 2 * a], m, se);
        res.delta[a] = m / spot[a], res.delta_se[a] = se / spot[a];
    }
    res.n_paths = 2 * n_pairs;
    res.n_batches = kAdjBatches;
    float f_ms = 0.0f, b_ms = 0.0f;
    check_cuda(cudaEventElapsedTime(&f_ms, e0, e1), "cudaEventElapsedTime");
    check_cuda(cudaEventElapsedTime(&b_ms, e1, e2), "cudaEventElapsedTime");
    res.forward_ms = f_ms, res.backward_ms = backward ? b_ms : 0.0;
    if (batch_pairs) {
        unsigned long long h[kAdjBatches];
        const unsigned long long* db = precision == OB_FP32 ? af.batch_pairs : ad.batch_pairs;
        check_cuda(cudaMemcpy(h, db, sizeof h, cudaMemcpyDeviceToHost), "copy batch counts");
        for (int b = 0; b < kAdjBatches; ++b) batch_pairs[b] = backward ? static_cast<long long>(h[b]) : 0;
    }
}

}  // namespace ob

struct ob_adjoint_plan {
    ob::AdjPlan impl;
};

extern "C" {

int ob_adjoint_plan_create(const ob_adjoint_request* rq, int precision, ob_adjoint_plan** plan) {
    return ob::guarded([&] {
        if (!rq || !plan) ob::invalid("null argument");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        *plan = nullptr;
        ob::check_adjoint(*rq);
        auto* p = new ob_adjoint_plan();
        try {
            p->impl.sms = ob::require_device();
            p->impl.precision = precision;
            p->impl.n_pairs = rq->base.n_pairs;
            ob::check_cuda(cudaEventCreate(&p->impl.e0), "cudaEventCreate");
            ob::check_cuda(cudaEventCreate(&p->impl.e1), "cudaEventCreate");
            ob::check_cuda(cudaEventCreate(&p->impl.e2), "cudaEventCreate");
            if (precision == OB_FP32) p->impl.build<float>(*rq);
            else p->impl.build<double>(*rq);
            ob::check_cuda(cudaDeviceSynchronize(), "adjoint plan");
        } catch (...) {
            delete p;
            throw;
        }
        *plan = p;
    });
}

int ob_adjoint_run(ob_adjoint_plan* plan, const double* d_table, double* d_grad, void* stream) {
    return ob::guarded([&] {
        if (!plan) ob::invalid("null plan");
        plan->impl.run(d_table, d_grad, static_cast<cudaStream_t>(stream));
    });
}

int ob_adjoint_result_get(ob_adjoint_plan* plan, ob_adjoint_result* res, long long* batch_pairs) {
    return ob::guarded([&] {
        if (!plan || !res) ob::invalid("null argument");
        plan->impl.result(*res, batch_pairs);
    });
}

int ob_adjoint_plan_destroy(ob_adjoint_plan* plan) {
    return ob::guarded([&] { delete plan; });
}

}  // extern "C"
