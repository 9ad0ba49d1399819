// ob_leverage: the drop-in for optlab::api::leverage(rq, 1, 0) (RC/include/optlab_cuda/requests.hpp:107-108), the SLV
// leverage by the particle method of Guyon and Henry-Labordere, as RC/src/leverage.cpp:97-152 (host algorithm) with
// the particle device of RC/src/leverage.cpp:156-214 / RC/src/leverage_gpu.cu:40-106.
//
// Per step i, everything stays on the device (the reference crosses PCIe three times a step):
//   lev_bin        one block an SM: its particles into a private fine histogram and regression bins in shared
//                  memory (u32 counts, the v sums in 64-bit fixed point, the local-linear moments in FP64), then its
//                  non-zero entries added into the step's global histogram and bins (integer atomics: the counts and v
//                  sums do not depend on the order)
//   lev_regress    one block per grid point g: the quantiles of the fine histogram bound the grid (the reference's
//                  first-match search, by a block scan), then the Gaussian-kernel regression E[v | x_g]
//                  (Nadaraya-Watson or local linear) over the bins in FP64, and L_g = clip(sqrt(sigma_loc^2 / E),
//                  lmin, lmax) with the local variance interpolated on its uniform row; the row and the grid go
//                  straight into the output tables
//   lev_step       one thread per antithetic pair (grid-stride): the SLV Euler step with the leverage row staged in
//                  shared memory, normals from Philox counter (pair, step + 1, 0, 0), each block's min and max of the
//                  new x stored for the next step (no atomics); it also clears the histogram and bins just read
// Particles are float (OB_FP32) or double (OB_FP64); bins, regression and the leverage ratio are FP64 in both (each v
// enters the sums rounded to 2^-37).
//
// The 3 x 504 launches are a few microseconds of GPU work each, so launching them one by one makes the host the
// bound on a slow CPU (measured: 54.8 us a step against 28.6 us of kernels). The kernels therefore take the step
// index from a device counter (set by lev_init, advanced by lev_bin once the previous step is done) rather than as
// an argument, so every step after the first is the same three launches: they are captured once as a CUDA graph of
// kGraphSteps steps (programmatic dependent launches inside it) and the graph is replayed, with one more graph for
// the remaining steps. The host then issues a few dozen graph launches instead of 1,500 kernel launches.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace ob {

namespace {

constexpr int kGraphSteps = 16;  // time steps per replayed graph

// Instantiated graphs, destroyed when the calibration ends (after its stream has been synchronised, or on an error).
struct GraphExecs {
    std::vector<cudaGraphExec_t> v;
    ~GraphExecs() {
        for (cudaGraphExec_t e : v) cudaGraphExecDestroy(e);
    }
};

constexpr int kMaxBins = 512;
constexpr int kMaxFine = 16384;
constexpr int kMaxX = 1024;

struct LevDev {
    long long n_pairs;
    int n_steps;
    int n_x, n_bins, n_fine, n_lv, local_linear, positive_part;
    uint32_t k0, k1;
    double v0, kappa, theta, xi, rho, atm_vol, bw_scale, l_min, l_max, q_lo, q_hi;
    const double* dt;
    const double* t0;
    const double* lv_lo;
    const double* lv_inv_dx;
    const double* lv_rows;
    const double* bw;          // n_steps: the kernel bandwidth of each step, computed on the host
    // the step's histogram and bins, added into by every binning block, cleared by the step kernel after use
    unsigned* fine;            // n_fine
    unsigned* chunk;           // (n_fine + 31) / 32: totals of 32-bin chunks of fine
    unsigned* cnt;             // n_bins
    unsigned long long* sv;    // n_bins + 1: v sums in fixed point, then the sum of all v
    double* acc_ll;            // 3 n_bins: x, x^2, x v sums (local linear only)
    int n_step_blocks;         // blocks of lev_step, each with its min and max of the new x
    double* part_range;        // n_step_blocks x 2
    double* x_eval;            // n_x, the current grid
    double* lev;               // n_x, the current leverage row
    double* x_grids;           // n_steps x n_x
    double* values;            // n_steps x n_x
    int* step;                 // the current step: 0 from lev_init, advanced by lev_bin before the step's regression
    // the persistent kernel's grid barrier: its arrival counter, and the status a barrier that gave up sets
    unsigned* bar_count;
    int* status;
    long long wait_limit;      // polls of a barrier's generation before it gives up (OB_ETIMEOUT)
};

// The v sums are 64-bit fixed point with 2^36 units per unit of v: integer additions, so the sums are the same
// whatever the order of the atomics (|v| may reach 2^27 / particles, far above any variance).
constexpr double kFix = 68719476736.0;

__device__ __forceinline__ long long warp_sum_i64(long long v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// Min and max of x over the last step's blocks, in every thread of the calling block (any multiple of 32 threads).
__device__ void range_of(const LevDev& d, double& lo, double& hi, double* s_mn, double* s_mx) {
    double mn = 1.0e300, mx = -1.0e300;
    const double2* pr = reinterpret_cast<const double2*>(d.part_range);
    for (int b0 = threadIdx.x; b0 < d.n_step_blocks; b0 += 4 * blockDim.x) {
        double2 r[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int b = b0 + j * blockDim.x;
            r[j] = b < d.n_step_blocks ? __ldcg(pr + b) : make_double2(1.0e300, -1.0e300);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) mn = fmin(mn, r[j].x), mx = fmax(mx, r[j].y);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, off));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_mn[warp] = mn, s_mx[warp] = mx;
    __syncthreads();
    lo = s_mn[0], hi = s_mx[0];
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) lo = fmin(lo, s_mn[w]), hi = fmax(hi, s_mx[w]);
    __syncthreads();
}

// Programmatic dependent launch: the step's kernels are launched while the previous one runs, and each waits here,
// before its first read of the previous kernel's output, until that kernel has finished and its writes are visible.
__device__ __forceinline__ void wait_previous() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename R>
__global__ void lev_init(R* x, R* v, long long n, R v0, int* step) {
    const long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j < n) x[j] = R(0), v[j] = v0;
    if (j == 0) *step = 0;
}

// The step index, read after the wait for the previous kernel (which may have advanced it), from L2.
__device__ __forceinline__ int current_step(const LevDev& d) { return __ldcg(d.step); }

// Bin edges and indices as the reference computes them: in double on the CPU, in float on its GPU. A block bins its
// particles in shared memory, then adds its non-zero entries into the step's global histogram and bins.
// The binning block's shared memory: v sums (nb + 1, fixed point), local-linear moments (3 nb), fine histogram (nf)
// and bin counts (nb).
struct BinShared {
    unsigned long long* sv;
    double* ll;
    unsigned* fine;
    unsigned* cnt;
};

__device__ __forceinline__ BinShared bin_shared(const LevDev& d, unsigned char* sm) {
    BinShared b;
    b.sv = reinterpret_cast<unsigned long long*>(sm);
    b.ll = reinterpret_cast<double*>(b.sv + d.n_bins + 1);
    b.fine = reinterpret_cast<unsigned*>(b.ll + (d.local_linear ? 3 * d.n_bins : 0));
    b.cnt = b.fine + d.n_fine;
    return b;
}

__device__ __forceinline__ void bin_clear_shared(const LevDev& d, const BinShared& b) {
    const int nb = d.n_bins, nf = d.n_fine;
    for (int k = threadIdx.x; k < nb + 1; k += blockDim.x) b.sv[k] = 0ull;
    if (d.local_linear)
        for (int k = threadIdx.x; k < 3 * nb; k += blockDim.x) b.ll[k] = 0.0;
    for (int k = threadIdx.x; k < nf + nb; k += blockDim.x) b.fine[k] = 0u;
}

// One block's share of a step's binning (the block's shared memory cleared by bin_clear_shared before): its particles
// into the shared histogram and bins, then the non-zero entries added into the step's global ones. Particles and the
// last step's ranges are read through L2: in the persistent kernel other blocks wrote them in the same launch.
// Particles a phase works on: arrays x, v of 2 n particles (leg 0 of pair c at c, leg 1 at n + c) whose pair c is
// global pair first + c, this thread taking pairs (or particles) start, start + stride, ... In global memory (SH false:
// every pair, the grid striding over them, read through L2) or in the block's shared memory (SH true: the block's own
// pairs, kept there from step to step by the persistent kernel).
template <typename R>
struct Particles {
    R* x;
    R* v;
    long long n, first, start, stride;
};

template <bool SH, typename R>
__device__ __forceinline__ R ld_part(const R* p) {
    if constexpr (SH) return *p;
    else return __ldcg(p);
}

template <typename R, bool SH = false>
__device__ void bin_phase(const LevDev& d, const Particles<R>& pt, const BinShared& b, double* s_mn, double* s_mx) {
    const R* __restrict__ x = pt.x;
    const R* __restrict__ v = pt.v;
    const int nb = d.n_bins, nf = d.n_fine, ll = d.local_linear;
    unsigned long long* s_sv = b.sv;
    double* s_ll = b.ll;
    unsigned* s_fine = b.fine;
    unsigned* s_cnt = b.cnt;
    double lo_d, hi_d;
    range_of(d, lo_d, hi_d, s_mn, s_mx);  // (its barrier also orders the clearing before)
    const R lo = static_cast<R>(lo_d), hi = static_cast<R>(hi_d);
    const R wf = (hi - lo) / static_cast<R>(nf), we = (hi + static_cast<R>(1e-12) - lo) / static_cast<R>(nb);
    const long long n = 2 * pt.n;
    long long tot = 0;
    const long long stride = pt.stride;
    for (long long j0 = pt.start; j0 < n; j0 += 4 * stride) {
        // four particles' loads in flight before their atomics
        R xr[4], vr[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long j = j0 + u * stride;
            xr[u] = j < n ? ld_part<SH>(x + j) : R(0), vr[u] = j < n ? ld_part<SH>(v + j) : R(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (j0 + u * stride >= n) break;
            const R xj = xr[u], vj = d.positive_part ? m_max(vr[u], R(0)) : vr[u];
            const int f = wf > R(0) ? static_cast<int>((xj - lo) / wf) : 0;
            atomicAdd(&s_fine[min(max(f, 0), nf - 1)], 1u);
            const int k = min(max(static_cast<int>((xj - lo) / we), 0), nb - 1);
            const double xd = static_cast<double>(xj), vd = static_cast<double>(vj);
            const long long q = __double2ll_rn(vd * kFix);
            atomicAdd(&s_cnt[k], 1u);
            atomicAdd(&s_sv[k], static_cast<unsigned long long>(q));
            if (ll) {
                atomicAdd(&s_ll[k], xd);
                atomicAdd(&s_ll[nb + k], xd * xd);
                atomicAdd(&s_ll[2 * nb + k], xd * vd);
            }
            tot += q;
        }
    }
    tot = warp_sum_i64(tot);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_sv[nb], static_cast<unsigned long long>(tot));
    __syncthreads();
    for (int k = threadIdx.x; k < nf; k += blockDim.x)
        if (s_fine[k]) atomicAdd(&d.fine[k], s_fine[k]);
    {
        // the block's 32-bin chunk totals: a warp a chunk, a lane a bin
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_ch = (nf + 31) / 32;
        for (int c = warp; c < n_ch; c += blockDim.x >> 5) {
            const int k = 32 * c + lane;
            unsigned u = k < nf ? s_fine[k] : 0u;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) u += __shfl_xor_sync(0xffffffffu, u, off);
            if (lane == 0 && u) atomicAdd(&d.chunk[c], u);
        }
    }
    for (int k = threadIdx.x; k < nb; k += blockDim.x)
        if (s_cnt[k]) atomicAdd(&d.cnt[k], s_cnt[k]), atomicAdd(&d.sv[k], s_sv[k]);
    if (threadIdx.x == 0) atomicAdd(&d.sv[nb], s_sv[nb]);
    if (ll)
        for (int k = threadIdx.x; k < 3 * nb; k += blockDim.x)
            if (s_ll[k] != 0.0) atomicAdd(&d.acc_ll[k], s_ll[k]);
}

template <typename R>
__global__ void __launch_bounds__(512) lev_bin(LevDev d, const R* __restrict__ x, const R* __restrict__ v) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ double s_mn[32], s_mx[32];
    const BinShared b = bin_shared(d, sm);
    bin_clear_shared(d, b);
    wait_previous();
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(d.step, 1);  // the previous step is done: this is the next
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    const Particles<R> pt{const_cast<R*>(x), const_cast<R*>(v), d.n_pairs, 0, blockIdx.x * (long long)blockDim.x + threadIdx.x,
                          stride};
    bin_phase<R>(d, pt, b, s_mn, s_mx);
}

// Exclusive prefix of x over the block and the block's total (any block size that is a multiple of 32, up to 1024).
__device__ unsigned long long block_scan(unsigned long long x, unsigned long long* s_warp, unsigned long long& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned long long inc = x;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    unsigned long long before = 0, tot = 0;
    for (int w = 0; w < nw; ++w) {
        const unsigned long long c = s_warp[w];
        before += w < warp ? c : 0ull;
        tot += c;
    }
    __syncthreads();
    total = tot;
    return before + inc - x;
}

__device__ __forceinline__ double interp_uniform(double x, double a, double b, const double* y, int n) {
    const double u = (x - a) / (b - a) * (n - 1);
    if (!(u > 0)) return y[0];
    if (u >= n - 1) return y[n - 1];
    const int i = static_cast<int>(u);
    const double w = u - i;
    return y[i] * (1 - w) + y[i + 1] * w;
}

// Grid, regression and leverage of step i; block g computes grid point g. Step 0 uses the reference's initial grid
// and E[v | x] = v0. The grid's bounds are the quantiles of the fine histogram (RC/src/leverage.cpp:26-38: the first
// fine bin k with a count and (counts before k) + count >= q total, at lo + (k + (q total - before) / count) width),
// computed in every block from the chunk totals and, for the chunk that holds each quantile, its 32 bins.
// Shared memory of the regression (blocks of at most 512 threads).
struct RegressShared {
    unsigned long long warp[32];
    double cum[2][512];
    int best[2];
    double q[2];
    double red[5][32];
    double mn[32], mx[32];
};

__device__ void regress_phase(const LevDev& d, double n_particles, int g, int i, RegressShared& sh) {
    unsigned long long* s_warp = sh.warp;
    double(*s_cum)[512] = sh.cum;
    int* s_best = sh.best;
    double* s_q = sh.q;
    double(*s_red)[32] = sh.red;
    double *s_mn = sh.mn, *s_mx = sh.mx;
    const int nx = d.n_x, nb = d.n_bins, nf = d.n_fine, t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5, nw = blockDim.x >> 5;
    const double h = d.dt[i];
    double x0, cond;
    if (i == 0) {
        x0 = (-6.0 + 12.0 * g / (nx - 1)) * d.atm_vol * sqrt(h > 1e-4 ? h : 1e-4);
        cond = d.v0;
    } else {
        // Two levels: each thread owns a run of 32-bin chunks and their totals (kept by lev_bin); a block scan of the
        // runs gives the counts before every chunk; the first chunk with a count that reaches the target holds the
        // quantile's bin, and the thread owning it scans that chunk's 32 bins.
        const int n_ch = (nf + 31) / 32, cpt = (n_ch + blockDim.x - 1) / blockDim.x;
        const int ca = min(t * cpt, n_ch), cb = min(ca + cpt, n_ch);
        unsigned mine_c[2] = {0u, 0u};  // cpt <= 2 (n_fine <= 16384)
        unsigned long long mine = 0;
        for (int c = ca; c < cb; ++c) mine_c[c - ca] = __ldcg(d.chunk + c), mine += mine_c[c - ca];
        if (t < 2) s_best[t] = n_ch;
        double lo, hi;
        range_of(d, lo, hi, s_mn, s_mx);  // (its barriers also publish s_best)
        unsigned long long total_u;
        const unsigned long long before = block_scan(mine, s_warp, total_u);
        const double total = static_cast<double>(total_u);
        const double q2[2] = {d.q_lo, d.q_hi};
#pragma unroll
        for (int qi = 0; qi < 2; ++qi) {
            const double target = q2[qi] * total;
            double cum = static_cast<double>(before);
            for (int c = ca; c < cb; ++c) {
                const unsigned tc = mine_c[c - ca];
                if (tc > 0 && cum + static_cast<double>(tc) >= target) {
                    atomicMin(&s_best[qi], c);
                    s_cum[qi][t] = cum;
                    break;
                }
                cum += static_cast<double>(tc);
            }
        }
        __syncthreads();
        const double width = (hi - lo) / static_cast<double>(nf);
#pragma unroll
        for (int qi = 0; qi < 2; ++qi) {
            const int cw = s_best[qi];
            if (cw < n_ch && t == cw / cpt) {
                // the bins of chunk cw: the first with a count and (counts before it) + count >= target
                const double target = q2[qi] * total;
                unsigned cc[32];  // the 32 loads issued together, then the search
#pragma unroll
                for (int j = 0; j < 32; ++j) cc[j] = 32 * cw + j < nf ? __ldcg(d.fine + 32 * cw + j) : 0u;
                double cum = s_cum[qi][t];
                int kb = nf;
                unsigned cb_count = 0u;
                double before_kb = 0.0;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const unsigned c = cc[j];
                    if (kb == nf && c > 0 && cum + static_cast<double>(c) >= target)
                        kb = 32 * cw + j, cb_count = c, before_kb = cum;
                    cum += static_cast<double>(c);
                }
                s_q[qi] = kb >= nf ? hi
                                   : lo + (static_cast<double>(kb) + (target - before_kb) /
                                                                         static_cast<double>(cb_count)) *
                                              width;
            } else if (cw >= n_ch && t == 0) {
                s_q[qi] = hi;
            }
        }
        __syncthreads();
        const double qv[2] = {s_q[0], s_q[1]};
        x0 = qv[0] + (qv[1] - qv[0]) * g / (nx - 1);
        const double bw = d.bw[i];
        const double wc = (hi + 1e-12 - lo) / nb;
        const double *sx = d.acc_ll, *sxx = sx + nb, *sxv = sxx + nb;
        double r[5] = {0, 0, 0, 0, 0};
        // n_bins <= 512: at most two bins a thread, their loads issued together
        unsigned cn[2];
        unsigned long long sq[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int k = t + u * static_cast<int>(blockDim.x);
            cn[u] = k < nb ? __ldcg(d.cnt + k) : 0u, sq[u] = k < nb ? __ldcg(d.sv + k) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int k = t + u * static_cast<int>(blockDim.x);
            if (k >= nb) break;
            const double c = lo + (k + 0.5) * wc;
            const double dd = (x0 - c) / bw, w = exp(-0.5 * dd * dd);
            const double sv = static_cast<double>(static_cast<long long>(sq[u])) / kFix;
            r[0] += w * static_cast<double>(cn[u]), r[1] += w * sv;
            if (d.local_linear) r[2] += w * __ldcg(sx + k), r[3] += w * __ldcg(sxx + k), r[4] += w * __ldcg(sxv + k);
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            r[q] = warp_sum(r[q]);
            if (lane == 0) s_red[q][warp] = r[q];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            r[q] = 0.0;
            for (int w = 0; w < nw; ++w) r[q] += s_red[q][w];
        }
        const double S0 = r[0], T0 = r[1], Ax = r[2], Axx = r[3], Axv = r[4];
        const double fallback = static_cast<double>(static_cast<long long>(__ldcg(d.sv + nb))) / kFix / n_particles;
        const double nw_e = S0 > 1e-8 ? T0 / (S0 > 1e-300 ? S0 : 1e-300) : fallback;
        cond = nw_e;
        if (d.local_linear) {
            const double S1 = Ax - x0 * S0, S2 = Axx - 2 * x0 * Ax + x0 * x0 * S0, T1 = Axv - x0 * T0;
            const double det = S0 * S2 - S1 * S1;
            const bool ok = S0 >= 50 && det > 1e-12 * S0 * fabs(S2);
            const double lle = ok ? (S2 * T0 - S1 * T1) / det : nw_e;
            cond = lle > 1e-8 ? lle : 1e-8;
        }
    }
    if (t == 0) {
        const double* row = d.lv_rows + static_cast<long long>(i) * d.n_lv;
        const double lv_lo = d.lv_lo[i], lv_hi = lv_lo + (d.n_lv - 1) / d.lv_inv_dx[i];
        const double loc = interp_uniform(x0, lv_lo, lv_hi, row, d.n_lv);
        double L = sqrt(loc / (cond > 1e-8 ? cond : 1e-8));
        L = L > d.l_min ? L : d.l_min;
        L = L < d.l_max ? L : d.l_max;
        d.x_eval[g] = x0, d.lev[g] = L;
        d.x_grids[static_cast<long long>(i) * nx + g] = x0;
        d.values[static_cast<long long>(i) * nx + g] = L;
    }
    __syncthreads();  // the block's shared memory is free for its next grid point
}

__global__ void __launch_bounds__(256) lev_regress(LevDev d, double n_particles) {
    __shared__ RegressShared sh;
    wait_previous();
    regress_phase(d, n_particles, blockIdx.x, current_step(d), sh);
}

// The SLV Euler step of every pair (grid-stride), and the block's min and max of the new x into part_range. The step's
// histogram and bins are read (lev_regress is done): the blocks clear them for the next step's binning.
template <typename R, bool SH = false>
__device__ void step_phase(const LevDev& d, const Particles<R>& pt, int i, R* s_lev, R* s_min, R* s_max) {
    R* __restrict__ x = pt.x;
    R* __restrict__ v = pt.v;
    {
        const int nb = d.n_bins, nf = d.n_fine, n_ll = d.local_linear ? 3 * nb : 0, n_ch = (nf + 31) / 32;
        const int stride = gridDim.x * blockDim.x;
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nf + nb + nb + 1 + n_ll + n_ch; k += stride) {
            if (k < nf) d.fine[k] = 0u;
            else if (k < nf + nb) d.cnt[k - nf] = 0u;
            else if (k < nf + 2 * nb + 1) d.sv[k - nf - nb] = 0ull;
            else if (k < nf + 2 * nb + 1 + n_ll) d.acc_ll[k - nf - 2 * nb - 1] = 0.0;
            else d.chunk[k - nf - 2 * nb - 1 - n_ll] = 0u;
        }
    }
    for (int g = threadIdx.x; g < d.n_x; g += blockDim.x) s_lev[g] = static_cast<R>(__ldcg(d.lev + g));
    __syncthreads();
    const int nx = d.n_x;
    const R h = static_cast<R>(d.dt[i]);
    const R a = static_cast<R>(__ldcg(d.x_eval)), b = static_cast<R>(__ldcg(d.x_eval + nx - 1));
    const R rho = static_cast<R>(d.rho), kappa = static_cast<R>(d.kappa), theta = static_cast<R>(d.theta);
    const R xi = static_cast<R>(d.xi);
    const R rc = m_sqrt(R(1) - rho * rho);
    R mn = sizeof(R) == 4 ? R(3.0e38f) : R(1.0e300), mx = -mn;
    for (long long p = pt.start; p < pt.n; p += pt.stride) {
        R z0, z1, z2, z3;
        normals4<R>(static_cast<uint64_t>(pt.first + p), static_cast<uint64_t>(i + 1), 0u, d.k0, d.k1, z0, z1, z2, z3);
#pragma unroll
        for (int leg = 0; leg < 2; ++leg) {
            const long long j = leg ? pt.n + p : p;
            const R sg = leg ? R(-1) : R(1), zz1 = sg * z0, zz2 = sg * z1;
            const R xj = ld_part<SH>(x + j);
            R L;
            // interpolation on the uniform grid [a, b]: the CPU's form in double, the reference GPU's in float
            const R u = sizeof(R) == 8 ? (xj - a) / (b - a) * static_cast<R>(nx - 1)
                                       : (xj - a) * (static_cast<R>(nx - 1) / (b - a));
            if (!(u > R(0))) L = s_lev[0];
            else if (u >= static_cast<R>(nx - 1)) L = s_lev[nx - 1];
            else {
                const int k = static_cast<int>(u);
                const R w = u - static_cast<R>(k);
                L = s_lev[k] * (R(1) - w) + s_lev[k + 1] * w;
            }
            const R vp = m_max(ld_part<SH>(v + j), R(0)), var = L * L * vp;
            const R zx = rho * zz2 + rc * zz1;
            v[j] += kappa * (theta - vp) * h + xi * m_sqrt(vp * h) * zz2;
            const R xn = xj + R(-0.5) * var * h + m_sqrt(var * h) * zx;
            x[j] = xn;
            mn = m_min(mn, xn), mx = m_max(mx, xn);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        mn = m_min(mn, __shfl_down_sync(0xffffffffu, mn, off));
        mx = m_max(mx, __shfl_down_sync(0xffffffffu, mx, off));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_min[warp] = mn, s_max[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) mn = m_min(mn, s_min[w]), mx = m_max(mx, s_max[w]);
        d.part_range[2 * blockIdx.x] = static_cast<double>(mn);
        d.part_range[2 * blockIdx.x + 1] = static_cast<double>(mx);
    }
}

template <typename R>
__global__ void __launch_bounds__(256) lev_step(LevDev d, R* __restrict__ x, R* __restrict__ v) {
    __shared__ R s_lev[kMaxX];
    __shared__ R s_min[32], s_max[32];
    wait_previous();
    const Particles<R> pt{x, v, d.n_pairs, 0, blockIdx.x * (long long)blockDim.x + threadIdx.x,
                          static_cast<long long>(gridDim.x) * blockDim.x};
    step_phase<R>(d, pt, current_step(d), s_lev, s_min, s_max);
}

// ------------------------------------------------------------------------------------------------ persistent
//
// The whole calibration as one cooperative launch (every block resident at once): per step the three phases above,
// separated by grid barriers, with the step index a loop variable. One block of 512 threads per SM. The barrier is a
// counter and a generation word in global memory; a block that waits polls the generation at most d.wait_limit times,
// then records OB_ETIMEOUT in d.status and returns, and every other block leaves at its next barrier on seeing the
// status, so a calibration whose barrier cannot complete ends with an error instead of holding the GPU.

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int status_of(const LevDev& d) { return *reinterpret_cast<volatile int*>(d.status); }

__device__ __forceinline__ void red_release_gpu(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Every block's writes before the barrier are visible to every block after it. The barrier is one arrival counter
// that only grows: a block adds one (a release) and waits until the count reaches every block's arrivals so far
// (`arrived`, advanced by gridDim.x at each barrier, the same in every thread). A block polls at most d.wait_limit
// times (with a limit of zero it gives up at once), then records OB_ETIMEOUT; a block that sees the status leaves.
// False: the calibration has failed and the caller returns.
__device__ bool grid_barrier(const LevDev& d, unsigned& arrived) {
    __shared__ int s_ok;
    arrived += gridDim.x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        red_release_gpu(d.bar_count, 1u);
        for (long long polls = 0;; ++polls) {
            if (polls >= d.wait_limit) {
                atomicCAS(d.status, 0, OB_ETIMEOUT);
                ok = 0;
                break;
            }
            if (ld_acquire_gpu(d.bar_count) >= arrived) break;
            if (status_of(d) != 0) {
                ok = 0;
                break;
            }
            if (polls > 256) __nanosleep(32);
        }
        __threadfence();
        if (status_of(d) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

constexpr int kPersistentThreads = 512;

// Block b owns pairs [b chunk, (b + 1) chunk) and keeps their particles in its shared memory (after the binning
// arrays, at part_off) for the whole calibration: the binning and the step read them there, not through L2.
template <typename R>
__global__ void __launch_bounds__(kPersistentThreads, 1)
    lev_persistent(LevDev d, long long chunk, int part_off, double n_particles) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ RegressShared rs;
    __shared__ R s_lev[kMaxX];
    __shared__ R s_min[32], s_max[32];
    __shared__ double s_mn[32], s_mx[32];
    const BinShared b = bin_shared(d, sm);
    const long long first = static_cast<long long>(blockIdx.x) * chunk;
    const long long count = first < d.n_pairs ? (d.n_pairs - first < chunk ? d.n_pairs - first : chunk) : 0;
    R* sx = reinterpret_cast<R*>(sm + part_off);
    R* sv = sx + 2 * chunk;
    const Particles<R> pt{sx, sv, count, first, threadIdx.x, blockDim.x};
    for (long long j = threadIdx.x; j < 2 * count; j += blockDim.x) sx[j] = R(0), sv[j] = static_cast<R>(d.v0);
    unsigned arrived = 0;
    // (step 0's regression reads no particle; its barrier orders these stores before the first step)
    for (int i = 0; i < d.n_steps; ++i) {
        if (i > 0) {
            bin_clear_shared(d, b);
            bin_phase<R, true>(d, pt, b, s_mn, s_mx);
            if (!grid_barrier(d, arrived)) return;
        }
        for (int g = blockIdx.x; g < d.n_x; g += gridDim.x) regress_phase(d, n_particles, g, i, rs);
        if (!grid_barrier(d, arrived)) return;
        step_phase<R, true>(d, pt, i, s_lev, s_min, s_max);
        if (i + 1 < d.n_steps && !grid_barrier(d, arrived)) return;
    }
}

// Polls of a grid barrier before it gives up (ob_set_wait_limit): a barrier completes within one phase, microseconds;
// the default, 2^22 polls with a short sleep between them, is about a second.
constexpr long long kDefaultWaitLimit = 1LL << 22;
long long g_wait_limit = kDefaultWaitLimit;

// Dynamic shared memory of a persistent block at most: the binning arrays and the block's particles.
constexpr size_t kPersistentSmemMax = size_t(200) << 10;

// The persistent calibration on stream st; false (nothing launched) when a block's particles do not fit its shared
// memory or the device cannot hold every block at once.
template <typename R>
bool run_persistent(LevDev& d, double n_particles, size_t bin_smem, int sms, cudaStream_t st) {
    const long long chunk = (d.n_pairs + sms - 1) / sms;
    const size_t part_off = (bin_smem + 15) & ~static_cast<size_t>(15);
    const size_t smem = part_off + 4 * static_cast<size_t>(chunk) * sizeof(R);
    if (smem > kPersistentSmemMax) return false;
    check_cuda(cudaFuncSetAttribute(lev_persistent<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)),
               "cudaFuncSetAttribute");
    int occ = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, lev_persistent<R>, kPersistentThreads, smem),
               "occupancy");
    int coop = 0, dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "cudaDeviceGetAttribute");
    if (occ < 1 || !coop || d.n_step_blocks != sms) return false;
    int off = static_cast<int>(part_off);
    long long ch = chunk;
    void* args[] = {&d, &ch, &off, &n_particles};
    const cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(lev_persistent<R>), dim3(sms),
                                                      dim3(kPersistentThreads), args, smem, st);
    if (e == cudaErrorCooperativeLaunchTooLarge) {
        cudaGetLastError();
        return false;
    }
    check_cuda(e, "lev_persistent launch");
    return true;
}

void check_request(const ob_leverage_request& rq) {
    if (!rq.dt || !rq.t0 || !rq.lv_lo || !rq.lv_inv_dx || !rq.lv_rows || !rq.x_grids || !rq.values)
        invalid("null pointer");
    if (rq.n_steps < 1 || rq.n_pairs < 2 || rq.n_x < 2 || rq.n_bins < 2 || rq.n_fine < 16 || rq.n_lv < 2)
        invalid("n_steps, n_pairs, n_x, n_bins, n_fine or n_lv too small");
    if (!(rq.kappa > 0 && rq.theta > 0 && rq.xi >= 0 && std::fabs(rq.rho) <= 1 && rq.v0 >= 0))
        invalid("Heston parameters out of range");
    if (rq.n_bins > kMaxBins) invalid("n_bins must be <= 512");
    if (rq.n_fine > kMaxFine) invalid("n_fine must be <= 16384");
    if (rq.n_x > kMaxX) invalid("n_x must be <= 1024");
}

template <typename R>
void run_leverage(ob_leverage_request& rq) {
    const auto t_start = std::chrono::steady_clock::now();
    const int sms = require_device();
    DeviceArena arena;
    arena.recycle = true;  // the stream is synchronised before the call returns
    LevDev d{};
    const long long n = 2 * rq.n_pairs;
    const int S = rq.n_steps;
    d.n_pairs = rq.n_pairs, d.n_x = rq.n_x, d.n_bins = rq.n_bins, d.n_fine = rq.n_fine, d.n_lv = rq.n_lv;
    d.local_linear = rq.local_linear, d.positive_part = rq.positive_part;
    d.k0 = static_cast<uint32_t>(rq.seed), d.k1 = static_cast<uint32_t>(rq.seed >> 32);
    d.v0 = rq.v0, d.kappa = rq.kappa, d.theta = rq.theta, d.xi = rq.xi, d.rho = rq.rho;
    d.atm_vol = rq.atm_vol, d.bw_scale = rq.bandwidth_scale, d.l_min = rq.l_min, d.l_max = rq.l_max;
    d.q_lo = rq.q_lo, d.q_hi = rq.q_hi;
    d.dt = arena.put<double>(rq.dt, S);
    d.t0 = arena.put<double>(rq.t0, S);
    d.lv_lo = arena.put<double>(rq.lv_lo, S);
    d.lv_inv_dx = arena.put<double>(rq.lv_inv_dx, S);
    d.lv_rows = arena.put<double>(rq.lv_rows, static_cast<size_t>(S) * rq.n_lv);
    const int nb = rq.n_bins, nf = rq.n_fine, ll = rq.local_linear;
    d.fine = arena.alloc<unsigned>(nf);
    d.chunk = arena.alloc<unsigned>((nf + 31) / 32);
    check_cuda(cudaMemset(d.chunk, 0, (nf + 31) / 32 * sizeof(unsigned)), "cudaMemset");
    d.cnt = arena.alloc<unsigned>(nb);
    d.sv = arena.alloc<unsigned long long>(nb + 1);
    d.acc_ll = arena.alloc<double>(3 * static_cast<size_t>(nb));
    check_cuda(cudaMemset(d.fine, 0, nf * sizeof(unsigned)), "cudaMemset");
    check_cuda(cudaMemset(d.cnt, 0, nb * sizeof(unsigned)), "cudaMemset");
    check_cuda(cudaMemset(d.sv, 0, (nb + 1) * sizeof(unsigned long long)), "cudaMemset");
    check_cuda(cudaMemset(d.acc_ll, 0, 3 * nb * sizeof(double)), "cudaMemset");
    d.x_eval = arena.alloc<double>(rq.n_x);
    d.lev = arena.alloc<double>(rq.n_x);
    d.x_grids = arena.alloc<double>(static_cast<size_t>(S) * rq.n_x);
    d.values = arena.alloc<double>(static_cast<size_t>(S) * rq.n_x);
    R* x = arena.alloc<R>(n);
    R* v = arena.alloc<R>(n);
    d.step = arena.alloc<int>(1);
    const size_t bin_smem = (static_cast<size_t>(nb) + 1) * sizeof(unsigned long long) +
                            (ll ? 3 * static_cast<size_t>(nb) * sizeof(double) : 0) +
                            (static_cast<size_t>(nf) + nb) * sizeof(unsigned);
    check_cuda(cudaFuncSetAttribute(lev_bin<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(bin_smem)),
               "cudaFuncSetAttribute");
    // one binning block an SM (fewer for small particle counts): each block bins many particles before it adds
    const int n_bin_blocks = static_cast<int>(std::max<long long>(1, std::min<long long>(sms, (n + 511) / 512)));
    // the persistent kernel's blocks (one an SM) each write their range; the graph path's lev_step uses up to 4 an SM
    d.n_step_blocks = sms;
    d.part_range = arena.alloc<double>(2 * static_cast<size_t>(4 * sms));
    d.n_steps = S;
    d.bar_count = arena.alloc<unsigned>(4);
    d.status = reinterpret_cast<int*>(d.bar_count + 2);
    check_cuda(cudaMemset(d.bar_count, 0, 4 * sizeof(unsigned)), "cudaMemset");
    d.wait_limit = g_wait_limit;
    const double n_particles = 2.0 * static_cast<double>(rq.n_pairs);
    // the kernel bandwidth of each step, as RC/src/leverage.cpp:63 computes it
    std::vector<double> bw(S);
    for (int i = 0; i < S; ++i)
        bw[i] = rq.bandwidth_scale * rq.atm_vol * std::sqrt(std::max(rq.t0[i], 0.15)) * std::pow(n_particles, -0.2);
    d.bw = arena.put<double>(bw.data(), S);
    Stream stream;
    cudaStream_t st = stream.get();
    cudaLaunchAttribute pdl[1];
    pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    pdl[0].val.programmaticStreamSerializationAllowed = 1;
    auto config = [&](unsigned grid, unsigned block, size_t smem) {
        cudaLaunchConfig_t c{};
        c.gridDim = dim3(grid), c.blockDim = dim3(block), c.dynamicSmemBytes = smem, c.stream = st;
        c.attrs = pdl, c.numAttrs = 1;
        return c;
    };
    // OPTLAB_B200_LEVERAGE=graphs runs the three-kernel schedule below instead (to compare the two; same results)
    const char* mode = std::getenv("OPTLAB_B200_LEVERAGE");
    const bool graphs_only = mode && std::strcmp(mode, "graphs") == 0;
    if (!graphs_only && run_persistent<R>(d, n_particles, bin_smem, sms, st)) {
        int status = 0;
        check_cuda(cudaMemcpyAsync(&status, d.status, sizeof status, cudaMemcpyDeviceToHost, st), "copy status");
        check_cuda(cudaMemcpyAsync(rq.x_grids, d.x_grids, static_cast<size_t>(S) * rq.n_x * sizeof(double),
                                   cudaMemcpyDeviceToHost, st),
                   "copy x_grids");
        check_cuda(cudaMemcpyAsync(rq.values, d.values, static_cast<size_t>(S) * rq.n_x * sizeof(double),
                                   cudaMemcpyDeviceToHost, st),
                   "copy values");
        check_cuda(cudaStreamSynchronize(st), "leverage");
        if (status == OB_ETIMEOUT)
            throw Error(OB_ETIMEOUT, "leverage: a grid barrier of the calibration gave up waiting for the other blocks");
        if (status != 0) throw Error(OB_ECUDA, "leverage: the calibration kernel reported a failure");
        rq.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        return;
    }
    // the device cannot hold the persistent kernel: three kernels a step, replayed as graphs
    d.n_step_blocks = static_cast<int>(std::max<long long>(1, std::min<long long>(4LL * sms, (rq.n_pairs + 255) / 256)));
    lev_init<R><<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(x, v, n, static_cast<R>(rq.v0), d.step);
    check_cuda(cudaGetLastError(), "lev_init launch");
    const R* cx = x;
    const R* cv = v;
    // step 0 (no binning: the particles all start at x = 0), launched directly
    const cudaLaunchConfig_t c_reg0 = config(rq.n_x, 256, 0), c_step0 = config(d.n_step_blocks, 256, 0);
    check_cuda(cudaLaunchKernelEx(&c_reg0, lev_regress, d, n_particles), "lev_regress launch");
    check_cuda(cudaLaunchKernelEx(&c_step0, lev_step<R>, d, x, v), "lev_step launch");
    // the other steps: graphs of kGraphSteps steps, replayed, and one of the remainder
    Stream capture;
    const cudaStream_t cs = capture.get();
    auto on = [&](cudaLaunchConfig_t c) {
        c.stream = cs;
        return c;
    };
    const cudaLaunchConfig_t c_bin = on(config(n_bin_blocks, 512, bin_smem));
    const cudaLaunchConfig_t c_step = on(config(d.n_step_blocks, 256, 0));
    const cudaLaunchConfig_t c_reg = on(config(rq.n_x, 256, 0));
    GraphExecs execs;
    auto make_graph = [&](int steps) {
        check_cuda(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < steps && e == cudaSuccess; ++k) {
            e = cudaLaunchKernelEx(&c_bin, lev_bin<R>, d, cx, cv);
            if (e == cudaSuccess) e = cudaLaunchKernelEx(&c_reg, lev_regress, d, n_particles);
            if (e == cudaSuccess) e = cudaLaunchKernelEx(&c_step, lev_step<R>, d, x, v);
        }
        cudaGraph_t g = nullptr;
        const cudaError_t e_end = cudaStreamEndCapture(cs, &g);
        if (e != cudaSuccess || e_end != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            check_cuda(e != cudaSuccess ? e : e_end, "leverage capture");
        }
        cudaGraphExec_t ge = nullptr;
        const cudaError_t e_inst = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        check_cuda(e_inst, "cudaGraphInstantiate (leverage)");
        execs.v.push_back(ge);
        return ge;
    };
    const int rest = S - 1, full = rest / kGraphSteps, tail = rest % kGraphSteps;
    if (full) {
        const cudaGraphExec_t ge = make_graph(kGraphSteps);
        for (int r = 0; r < full; ++r) check_cuda(cudaGraphLaunch(ge, st), "cudaGraphLaunch (leverage)");
    }
    if (tail) check_cuda(cudaGraphLaunch(make_graph(tail), st), "cudaGraphLaunch (leverage)");
    check_cuda(cudaMemcpyAsync(rq.x_grids, d.x_grids, static_cast<size_t>(S) * rq.n_x * sizeof(double),
                               cudaMemcpyDeviceToHost, st),
               "copy x_grids");
    check_cuda(cudaMemcpyAsync(rq.values, d.values, static_cast<size_t>(S) * rq.n_x * sizeof(double),
                               cudaMemcpyDeviceToHost, st),
               "copy values");
    check_cuda(cudaStreamSynchronize(st), "leverage");
    rq.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
}

}  // namespace
}  // namespace ob

extern "C" int ob_leverage(ob_leverage_request* rq, int precision) {
    return ob::guarded([&] {
        if (!rq) ob::invalid("null request");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        ob::check_request(*rq);
        if (precision == OB_FP32) ob::run_leverage<float>(*rq);
        else ob::run_leverage<double>(*rq);
    });
}

extern "C" long long ob_set_wait_limit(long long polls) {
    std::lock_guard<std::mutex> lock(ob::api_mutex());
    const long long prev = ob::g_wait_limit;
    ob::g_wait_limit = polls < 0 ? ob::kDefaultWaitLimit : polls;
    return prev;
}
