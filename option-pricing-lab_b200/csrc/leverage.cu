// ob_leverage: the drop-in for optlab::api::leverage(rq, 1, 0) (RC/include/optlab_cuda/requests.hpp:107-108), the SLV
// leverage by the particle method of Guyon and Henry-Labordere, as RC/src/leverage.cpp:97-152 (host algorithm) with
// the particle device of RC/src/leverage.cpp:156-214 / RC/src/leverage_gpu.cu:40-106.
//
// Per step i, everything stays on the device (the reference crosses PCIe three times a step), in three phases:
//   bin       each block's particles into a fine histogram and regression bins in its shared memory (u32 counts, the
//             v sums in 64-bit fixed point, the local-linear moments in FP64), then added into the step's global
//             histogram and bins (integer additions: the sums do not depend on their order)
//   regress   one block per grid point g: the quantiles of the fine histogram bound the grid (the reference's
//             first-match search, by a block scan), then the Gaussian-kernel regression E[v | x_g] (Nadaraya-Watson
//             or local linear) over the bins in FP64, and L_g = clip(sqrt(sigma_loc^2 / E), lmin, lmax) with the local
//             variance interpolated on its uniform row; the row and the grid go straight into the output tables
//   step      the SLV Euler step of every pair with the leverage row staged in shared memory, normals from Philox
//             counter (pair, step + 1, 0, 0), the new range of x kept for the next step's bins; the step's histogram
//             and bins are cleared for the next step
// Particles are float (OB_FP32) or double (OB_FP64); bins, regression and the leverage ratio are FP64 in both (each v
// enters the sums rounded to 2^-36).
//
// The calibration runs as one persistent cooperative kernel, lev_persistent: one block of 512 threads per SM holds its
// particles in shared memory for the whole calibration, the phases are separated by grid barriers with bounded waits
// (OB_ETIMEOUT), the range of x travels as two order-key atomics, and the histogram and bins are added into global
// memory by TMA bulk reductions (the fine histogram packed two 16-bit counts to a word). When the device cannot hold
// it (particles beyond a block's shared memory, no cooperative launch), the phases run as three kernels a step
// (lev_bin, lev_regress, lev_step) that take the step index from a device counter, captured as CUDA graphs of
// kGraphSteps steps with programmatic dependent launches, and replayed.
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
// The fine histogram's arrays (global and shared) are padded with zero bins to a multiple of 8 x 512, so that a block
// of 256 or 512 threads splits them, packed or not, into equal runs of whole 16-byte words.
constexpr int kFinePad = 4096;
// The persistent kernel packs the fine histogram two bins to a 32-bit word (16-bit counts, the even bin in the low
// half): a block's own counts fit (it bins fewer than 2^16 particles), and a step whose global count of one bin passes
// 2^16 - 1 shows as a total other than the number of particles (a carry moves 2^16 - 1, a lost one 2^16): the kernel
// then records kPackOverflow and the calibration is run again unpacked.
constexpr int kPackOverflow = -2;
// Local-variance rows of up to this many points are staged in the regression block's shared memory.
constexpr int kMaxRowSmem = 4096;

struct LevDev {
    long long n_pairs;
    int n_steps;
    int n_x, n_bins, n_fine, n_lv, local_linear, positive_part;
    int nfp;                   // n_fine padded to a multiple of kFinePad
    int nbq;                   // n_bins + 1 padded to a multiple of 4: the length of cnt and sv
    int packed;                // the fine histogram two bins to a word (persistent kernel)
    uint32_t k0, k1;
    double v0, kappa, theta, xi, rho, atm_vol, bw_scale, l_min, l_max, q_lo, q_hi;
    const double* dt;
    const double* t0;
    const double* lv_lo;
    const double* lv_inv_dx;
    const double* lv_rows;
    const double* bw;          // n_steps: the kernel bandwidth of each step, computed on the host
    // the step's histogram and bins, added into by every binning block, cleared by the step phase after use
    unsigned* fine;            // nfp words, nfp / 2 of them when packed (bins from n_fine on stay zero)
    unsigned* cnt;             // nbq: bin counts
    unsigned long long* sv;    // nbq: v sums in fixed point, then (at n_bins) the sum of all v
    double* acc_ll;            // 3 n_bins: x, x^2, x v sums (local linear only)
    int n_step_blocks;         // blocks of lev_step, each with its min and max of the new x (three-kernel schedule)
    double* part_range;        // n_step_blocks x 2
    long long* rng;            // 2 x 2: min and max of the new x as order keys, by step parity (persistent kernel)
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

// A 64-bit integer added into a pair of 32-bit words of shared memory (low, high) with two native 32-bit atomics:
// the carry out of the low word goes into the high one, so the pair holds the exact sum modulo 2^64.
__device__ __forceinline__ void add_u64_pair(unsigned* lo, unsigned* hi, unsigned long long q) {
    const unsigned l = static_cast<unsigned>(q), h = static_cast<unsigned>(q >> 32);
    const unsigned old = atomicAdd(lo, l);
    const unsigned up = h + (old + l < old ? 1u : 0u);
    if (up) atomicAdd(hi, up);
}

// Bulk reductions of shared memory into global memory by the TMA unit (cp.reduce.async.bulk, each CTA its own): one
// thread hands over a whole array and the unit adds it element by element at L2. Both addresses must be 16-byte
// aligned and the size a multiple of 16 bytes (bulk_aligned); the writes of the shared source must be fenced for the
// async proxy before (fence_proxy_async_shared, by the threads that wrote it, then a barrier), and the issuing thread
// waits for completion (bulk_wait_all) before its release of the results.
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ bool bulk_aligned(const void* dst, const void* src, unsigned bytes) {
    return ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src) | bytes) & 15u) == 0;
}
__device__ __forceinline__ void bulk_add_u32(unsigned* dst, const unsigned* src, unsigned bytes) {
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.u32 [%0], [%1], %2;" ::"l"(dst),
                 "r"(static_cast<unsigned>(__cvta_generic_to_shared(src))), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_add_u64(unsigned long long* dst, const unsigned long long* src, unsigned bytes) {
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.u64 [%0], [%1], %2;" ::"l"(dst),
                 "r"(static_cast<unsigned>(__cvta_generic_to_shared(src))), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Doubles as signed 64-bit keys in the same order (negative values with their magnitude bits flipped), for
// atomicMin / atomicMax: the min and max of the particles are exact whatever the order of the blocks.
__device__ __forceinline__ long long order_key(double x) {
    const long long b = __double_as_longlong(x);
    return b >= 0 ? b : b ^ 0x7fffffffffffffffLL;
}

__device__ __forceinline__ double from_order_key(long long k) {
    return __longlong_as_double(k >= 0 ? k : k ^ 0x7fffffffffffffffLL);
}

// Min and max of x over the last step's blocks (three-kernel schedule), in every thread of the calling block.
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
// The binning block's shared memory, every array at a multiple of 16 bytes: the fine histogram (nfp), the bin counts
// (nbq), the v sums as 64-bit words for the bulk reduction (nbq), the v sums while binning (nbq low and nbq high
// 32-bit words, fixed point; at n_bins the sum of all v) and the local-linear moments (3 nb).
struct BinShared {
    unsigned* fine;
    unsigned* cnt;
    unsigned long long* sv;
    unsigned* sv_lo;
    unsigned* sv_hi;
    double* ll;
};

__host__ __device__ __forceinline__ size_t bin_smem_bytes(int nfp, int nbq, int nb, int ll) {
    return static_cast<size_t>(nfp) * sizeof(unsigned) + static_cast<size_t>(nbq) * (3 * sizeof(unsigned) + 8) +
           (ll ? 3 * static_cast<size_t>(nb) * sizeof(double) : 0);
}

__device__ __forceinline__ BinShared bin_shared(const LevDev& d, unsigned char* sm) {
    BinShared b;
    b.fine = reinterpret_cast<unsigned*>(sm);
    b.cnt = b.fine + d.nfp;
    b.sv = reinterpret_cast<unsigned long long*>(b.cnt + d.nbq);
    b.sv_lo = reinterpret_cast<unsigned*>(b.sv + d.nbq);
    b.sv_hi = b.sv_lo + d.nbq;
    b.ll = reinterpret_cast<double*>(b.sv_hi + d.nbq);
    return b;
}

__device__ __forceinline__ void bin_clear_shared(const LevDev& d, const BinShared& b) {
    uint4* f4 = reinterpret_cast<uint4*>(b.fine);
    const int n4 = (d.nfp + 5 * d.nbq) / 4;  // fine, cnt, sv (two words each), sv_lo, sv_hi: contiguous
    for (int k = threadIdx.x; k < n4; k += blockDim.x) f4[k] = make_uint4(0u, 0u, 0u, 0u);
    if (d.local_linear)
        for (int k = threadIdx.x; k < 3 * d.n_bins; k += blockDim.x) b.ll[k] = 0.0;
}

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

// One block's share of a step's binning on the range [lo, hi] of the particles (the block's shared memory cleared by
// bin_clear_shared before, and a barrier since): its particles into the shared histogram and bins, then these added
// into the step's global histogram and bins.
template <typename R, bool SH = false>
__device__ void bin_phase(const LevDev& d, const Particles<R>& pt, const BinShared& b, double lo_d, double hi_d) {
    const R* __restrict__ x = pt.x;
    const R* __restrict__ v = pt.v;
    const int nb = d.n_bins, nf = d.n_fine, ll = d.local_linear;
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
            const int f = min(max(wf > R(0) ? static_cast<int>((xj - lo) / wf) : 0, 0), nf - 1);
            if (d.packed) atomicAdd(&b.fine[f >> 1], (f & 1) ? 0x10000u : 1u);
            else atomicAdd(&b.fine[f], 1u);
            const int k = min(max(static_cast<int>((xj - lo) / we), 0), nb - 1);
            const double xd = static_cast<double>(xj), vd = static_cast<double>(vj);
            const long long q = __double2ll_rn(vd * kFix);
            atomicAdd(&b.cnt[k], 1u);
            add_u64_pair(&b.sv_lo[k], &b.sv_hi[k], static_cast<unsigned long long>(q));
            if (ll) {
                atomicAdd(&b.ll[k], xd);
                atomicAdd(&b.ll[nb + k], xd * xd);
                atomicAdd(&b.ll[2 * nb + k], xd * vd);
            }
            tot += q;
        }
    }
    tot = warp_sum_i64(tot);
    if ((threadIdx.x & 31) == 0) add_u64_pair(&b.sv_lo[nb], &b.sv_hi[nb], static_cast<unsigned long long>(tot));
    __syncthreads();
    // the block's histogram and bins into the step's: bulk reductions by the TMA unit (issued by thread 0, waited for
    // at the next grid_arrive or at the end of the kernel), lane atomics for any array the unit cannot take
    const int nq = d.nbq;
    for (int k = threadIdx.x; k < nq; k += blockDim.x) b.sv[k] = (static_cast<unsigned long long>(b.sv_hi[k]) << 32) | b.sv_lo[k];
    fence_proxy_async_shared();
    __syncthreads();
    unsigned* gc = d.cnt;
    unsigned long long* gs = d.sv;
    const int fine_words = d.packed ? d.nfp / 2 : d.nfp;
    const unsigned fine_bytes = static_cast<unsigned>(fine_words) * 4u, cnt_bytes = static_cast<unsigned>(nq) * 4u;
    const bool bulk = bulk_aligned(d.fine, b.fine, fine_bytes) && bulk_aligned(gc, b.cnt, cnt_bytes) &&
                      bulk_aligned(gs, b.sv, 2u * cnt_bytes);
    if (bulk) {
        if (threadIdx.x == 0) {
            fence_proxy_async_global();  // (the clearing of the step's arrays, before the last barrier)
            bulk_add_u32(d.fine, b.fine, fine_bytes);
            bulk_add_u32(gc, b.cnt, cnt_bytes);
            bulk_add_u64(gs, b.sv, 2u * cnt_bytes);
            bulk_commit();
        }
    } else {
        for (int k = threadIdx.x; k < fine_words; k += blockDim.x)
            if (b.fine[k]) atomicAdd(&d.fine[k], b.fine[k]);
        for (int k = threadIdx.x; k <= nb; k += blockDim.x) {
            if (k == nb) atomicAdd(&gs[nb], b.sv[k]);
            else if (b.cnt[k]) atomicAdd(&gc[k], b.cnt[k]), atomicAdd(&gs[k], b.sv[k]);
        }
    }
    if (ll)
        for (int k = threadIdx.x; k < 3 * nb; k += blockDim.x)
            if (b.ll[k] != 0.0) atomicAdd(&d.acc_ll[k], b.ll[k]);
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
    double lo, hi;
    range_of(d, lo, hi, s_mn, s_mx);  // (its barrier also orders the clearing before)
    bin_phase<R>(d, pt, b, lo, hi);
    if (threadIdx.x == 0) bulk_wait_all();
}

// Exclusive prefix of x over the block and the block's total (any block size that is a multiple of 32, up to 1024).
// Without `reuse` the caller guarantees a barrier before s_warp is written again, and the last one is left out.
__device__ unsigned long long block_scan(unsigned long long x, unsigned long long* s_warp, unsigned long long& total,
                                         bool reuse = true) {
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
    if (reuse) __syncthreads();
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
// fine bin k with a count and (counts before k) + count >= q total, at lo + (k + (q total - before) / count) width).
// The step's row and scalars are staged before (regress_stage); the particles' histogram and bins are loaded in one
// wave: each thread a run of the fine histogram's words (into s_fine) and its bins' counts and v sums. A block scan of
// the runs' totals finds, for each quantile, the first run that reaches it, and that run's thread finds its bin.
struct RegressShared {
    unsigned long long warp[32];
    int best[2];
    double q[2];
    double red[5][32];
    double bw, lv_lo, lv_hi;  // the step's kernel bandwidth and local-variance row bounds (regress_stage)
};

// The step's inputs that do not depend on the particles, staged ahead of the regression (while the block waits at a
// barrier, or after the three-kernel schedule's wait for the previous kernel): the local-variance row into s_row
// (when it is given) and the step's scalars into sh, by threads 1 on (thread 0 is then releasing the block's arrival
// at the barrier) when the block has more than one warp. A barrier separates this from regress_phase.
__device__ void regress_stage(const LevDev& d, int i, RegressShared& sh, double* s_row) {
    const double* row = d.lv_rows + static_cast<long long>(i) * d.n_lv;
    const int skip = blockDim.x > 32 ? 1 : 0, t = static_cast<int>(threadIdx.x) - skip, nt = blockDim.x - skip;
    if (s_row && t >= 0)
        for (int k0 = t; k0 < d.n_lv; k0 += 4 * nt) {
            double r[4];  // the loads issued together, then the stores
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u * nt;
                r[u] = k < d.n_lv ? __ldg(row + k) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u * nt;
                if (k < d.n_lv) s_row[k] = r[u];
            }
        }
    if (static_cast<int>(threadIdx.x) == (blockDim.x > 32 ? 32 : 0)) {
        const double lv_lo = __ldg(d.lv_lo + i), inv = __ldg(d.lv_inv_dx + i);
        sh.bw = __ldg(d.bw + i), sh.lv_lo = lv_lo, sh.lv_hi = lv_lo + (d.n_lv - 1) / inv;
    }
}

// `more`: the block regresses another grid point after this one (its shared memory must be free again).
__device__ void regress_phase(const LevDev& d, double n_particles, int g, int i, double lo, double hi,
                              RegressShared& sh, unsigned* s_fine, double* s_row, bool more) {
    const int nx = d.n_x, nb = d.n_bins, nf = d.n_fine, t = threadIdx.x, nt = blockDim.x;
    const int lane = t & 31, warp = t >> 5, nw = nt >> 5;
    const double* row = d.lv_rows + static_cast<long long>(i) * d.n_lv;
    double x0, cond = d.v0;
    unsigned long long all_v = 0;
    if (i == 0) {
        const double h = d.dt[i];
        x0 = (-6.0 + 12.0 * g / (nx - 1)) * d.atm_vol * sqrt(h > 1e-4 ? h : 1e-4);
    } else {
        // this thread's bins (n_bins <= 512, blocks of 256 or 512 threads: at most two)
        unsigned cn[2] = {0u, 0u};
        unsigned long long sq[2] = {0ull, 0ull};
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int k = t + u * nt;
            if (k < nb) cn[u] = __ldcg(d.cnt + k), sq[u] = __ldcg(d.sv + k);
        }
        if (t == 0) all_v = __ldcg(d.sv + nb);
        // this thread's run of the fine histogram: seg words (a multiple of 4) from word t seg, holding bins from
        // t seg_b on (two to a word when packed)
        const bool pk = d.packed;
        const int seg = (pk ? d.nfp / 2 : d.nfp) / nt, n4 = seg / 4, seg_b = pk ? 2 * seg : seg;
        const uint4* __restrict__ src = reinterpret_cast<const uint4*>(d.fine + static_cast<long long>(t) * seg);
        uint4* dst = reinterpret_cast<uint4*>(s_fine + t * seg);
        unsigned long long mine = 0;
        for (int m0 = 0; m0 < n4; m0 += 4) {
            uint4 f[4];  // the loads issued together, then the stores
#pragma unroll
            for (int u = 0; u < 4; ++u) f[u] = m0 + u < n4 ? __ldcg(src + m0 + u) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (m0 + u < n4) dst[m0 + u] = f[u];
                const unsigned w4[4] = {f[u].x, f[u].y, f[u].z, f[u].w};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    mine += pk ? (w4[j] & 0xffffu) + (w4[j] >> 16) : static_cast<unsigned long long>(w4[j]);
            }
        }
        if (t < 2) sh.best[t] = nt;
        unsigned long long total_u;
        // (its barrier publishes sh.best; the next write of sh.warp is in the next regression, barriers later)
        const unsigned long long before = block_scan(mine, sh.warp, total_u, false);
        // every particle is in one fine bin: a packed count that passed 2^16 - 1 shows here
        if (pk && t == 0 && total_u != static_cast<unsigned long long>(n_particles)) atomicCAS(d.status, 0, kPackOverflow);
        const double total = static_cast<double>(total_u);
        const double q2[2] = {d.q_lo, d.q_hi};
        // counts are integers: (count) >= q total exactly when (count) >= ceil(q total)
        const unsigned long long need[2] = {static_cast<unsigned long long>(ceil(q2[0] * total)),
                                            static_cast<unsigned long long>(ceil(q2[1] * total))};
        // the first run with a count whose end reaches the target holds the quantile's bin
#pragma unroll
        for (int qi = 0; qi < 2; ++qi)
            if (mine > 0 && before + mine >= need[qi]) atomicMin(&sh.best[qi], t);
        __syncthreads();
        const double width = (hi - lo) / static_cast<double>(nf);
#pragma unroll
        for (int qi = 0; qi < 2; ++qi) {
            const int w = sh.best[qi];
            if (t == w) {
                const uint4* run = reinterpret_cast<const uint4*>(s_fine + t * seg);
                unsigned long long cum = before, before_kb = 0;
                int kb = -1;
                unsigned c_kb = 0u;
                for (int m = 0; m < n4 && kb < 0; ++m) {
                    const uint4 f = run[m];
                    const unsigned w4[4] = {f.x, f.y, f.z, f.w};
                    // the run's bins in order: one a word, or (packed) a word's low half before its high half
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        if (!pk && (u & 1)) continue;
                        const unsigned c = pk ? ((u & 1) ? w4[u >> 1] >> 16 : w4[u >> 1] & 0xffffu) : w4[u >> 1];
                        const int bin = t * seg_b + (pk ? 8 * m + u : 4 * m + (u >> 1));
                        if (kb < 0 && c > 0 && cum + c >= need[qi]) kb = bin, c_kb = c, before_kb = cum;
                        cum += c;
                    }
                }
                const double target = q2[qi] * total;
                sh.q[qi] = kb < 0 ? hi
                                  : lo + (static_cast<double>(kb) +
                                          (target - static_cast<double>(before_kb)) / static_cast<double>(c_kb)) *
                                             width;
            } else if (w >= nt && t == 0) {
                sh.q[qi] = hi;
            }
        }
        __syncthreads();
        const double qv[2] = {sh.q[0], sh.q[1]};
        x0 = qv[0] + (qv[1] - qv[0]) * g / (nx - 1);
        const double bw = sh.bw;
        const double wc = (hi + 1e-12 - lo) / nb;
        const double *sx = d.acc_ll, *sxx = sx + nb, *sxv = sxx + nb;
        double r[5] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int k = t + u * nt;
            if (k >= nb) break;
            const double c = lo + (k + 0.5) * wc;
            const double dd = (x0 - c) / bw, w = exp(-0.5 * dd * dd);
            const double sv = static_cast<double>(static_cast<long long>(sq[u])) / kFix;
            r[0] += w * static_cast<double>(cn[u]), r[1] += w * sv;
            if (d.local_linear) r[2] += w * __ldcg(sx + k), r[3] += w * __ldcg(sxx + k), r[4] += w * __ldcg(sxv + k);
        }
        const int nq = d.local_linear ? 5 : 2;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            if (q >= nq) break;
            r[q] = warp_sum(r[q]);
            if (lane == 0) sh.red[q][warp] = r[q];
        }
        __syncthreads();
        // the warps' sums added by warp 0 (thread 0 uses them)
        if (warp == 0)
#pragma unroll
            for (int q = 0; q < 5; ++q) r[q] = q < nq ? warp_sum(lane < nw ? sh.red[q][lane] : 0.0) : 0.0;
        const double S0 = r[0], T0 = r[1], Ax = r[2], Axx = r[3], Axv = r[4];
        const double nw_e = S0 > 1e-8 ? T0 / (S0 > 1e-300 ? S0 : 1e-300)
                                      : static_cast<double>(static_cast<long long>(all_v)) / kFix / n_particles;
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
        const double loc = interp_uniform(x0, sh.lv_lo, sh.lv_hi, s_row ? s_row : row, d.n_lv);
        double L = sqrt(loc / (cond > 1e-8 ? cond : 1e-8));
        L = L > d.l_min ? L : d.l_min;
        L = L < d.l_max ? L : d.l_max;
        d.x_eval[g] = x0, d.lev[g] = L;
        d.x_grids[static_cast<long long>(i) * nx + g] = x0;
        d.values[static_cast<long long>(i) * nx + g] = L;
    }
    if (more) __syncthreads();  // the block's shared memory is free for its next grid point
}

// Dynamic shared memory of lev_regress: the fine histogram, then the local-variance row when it is staged.
__host__ __device__ __forceinline__ bool row_staged(int n_lv) { return n_lv <= kMaxRowSmem; }

__global__ void __launch_bounds__(256) lev_regress(LevDev d, double n_particles) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ RegressShared sh;
    __shared__ double s_mn[32], s_mx[32];
    unsigned* s_fine = reinterpret_cast<unsigned*>(sm);
    double* s_row = row_staged(d.n_lv) ? reinterpret_cast<double*>(s_fine + d.nfp) : nullptr;
    wait_previous();
    const int i = current_step(d);
    regress_stage(d, i, sh, s_row);
    double lo = 0.0, hi = 0.0;
    if (i > 0) range_of(d, lo, hi, s_mn, s_mx);  // (its barriers also order the staging)
    else __syncthreads();
    regress_phase(d, n_particles, blockIdx.x, i, lo, hi, sh, s_fine, s_row, false);
}

// The normals of this thread's pairs at step i (Philox counter (pair, i + 1, 0, 0)): z0 at p, z1 at n + p.
template <typename R>
__device__ void step_normals(const LevDev& d, const Particles<R>& pt, int i, R* s_z) {
    for (long long p = pt.start; p < pt.n; p += pt.stride) {
        R z0, z1, z2, z3;
        normals4<R>(static_cast<uint64_t>(pt.first + p), static_cast<uint64_t>(i + 1), 0u, d.k0, d.k1, z0, z1, z2, z3);
        s_z[p] = z0, s_z[pt.n + p] = z1;
    }
}

// The SLV Euler step of every pair, and the block's min and max of the new x: into part_range (SH false) or into the
// step parity's order keys (SH true; block 0 also resets the other parity's keys for the next step). The step's
// histogram and bins are read (the regression is done): the blocks clear them for the next step's binning. The
// normals come from s_z when the caller computed them ahead, else from Philox here.
template <typename R, bool SH = false>
__device__ void step_phase(const LevDev& d, const Particles<R>& pt, int i, R* s_lev, R* s_min, R* s_max,
                           const R* s_z) {
    R* __restrict__ x = pt.x;
    R* __restrict__ v = pt.v;
    {
        const int nb = d.n_bins, nf = d.n_fine, n_ll = d.local_linear ? 3 * nb : 0, n_c = d.nbq;
        const int stride = gridDim.x * blockDim.x;
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nf + 2 * n_c + n_ll; k += stride) {
            if (k < nf) d.fine[k] = 0u;
            else if (k < nf + n_c) d.cnt[k - nf] = 0u;
            else if (k < nf + 2 * n_c) d.sv[k - nf - n_c] = 0ull;
            else d.acc_ll[k - nf - 2 * n_c] = 0.0;
        }
    }
    if constexpr (SH) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            long long* r = d.rng + 2 * ((i + 1) & 1);
            r[0] = 0x7fffffffffffffffLL, r[1] = -0x7fffffffffffffffLL - 1;
        }
    }
    const int nx = d.n_x;
    // the grid's ends and the step's length, loaded with the leverage row
    const double xa = __ldcg(d.x_eval), xb = __ldcg(d.x_eval + nx - 1), hd = __ldg(d.dt + i);
    for (int g = threadIdx.x; g < nx; g += blockDim.x) s_lev[g] = static_cast<R>(__ldcg(d.lev + g));
    __syncthreads();
    const R h = static_cast<R>(hd);
    const R a = static_cast<R>(xa), b = static_cast<R>(xb);
    const R rho = static_cast<R>(d.rho), kappa = static_cast<R>(d.kappa), theta = static_cast<R>(d.theta);
    const R xi = static_cast<R>(d.xi);
    const R rc = m_sqrt(R(1) - rho * rho);
    R mn = sizeof(R) == 4 ? R(3.0e38f) : R(1.0e300), mx = -mn;
    for (long long p = pt.start; p < pt.n; p += pt.stride) {
        R z0, z1;
        if (s_z) {
            z0 = s_z[p], z1 = s_z[pt.n + p];
        } else {
            R z2, z3;
            normals4<R>(static_cast<uint64_t>(pt.first + p), static_cast<uint64_t>(i + 1), 0u, d.k0, d.k1, z0, z1, z2,
                        z3);
        }
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
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) s_min[warp] = mn, s_max[warp] = mx;
    __syncthreads();
    if (warp == 0) {
        // the warps' extremes, by warp 0
        mn = lane < nw ? s_min[lane] : s_min[0], mx = lane < nw ? s_max[lane] : s_max[0];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            mn = m_min(mn, __shfl_down_sync(0xffffffffu, mn, off));
            mx = m_max(mx, __shfl_down_sync(0xffffffffu, mx, off));
        }
    }
    if (threadIdx.x == 0) {
        if constexpr (SH) {
            long long* r = d.rng + 2 * (i & 1);
            atomicMin(r, order_key(static_cast<double>(mn)));
            atomicMax(r + 1, order_key(static_cast<double>(mx)));
        } else {
            d.part_range[2 * blockIdx.x] = static_cast<double>(mn);
            d.part_range[2 * blockIdx.x + 1] = static_cast<double>(mx);
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(256) lev_step(LevDev d, R* __restrict__ x, R* __restrict__ v) {
    __shared__ R s_lev[kMaxX];
    __shared__ R s_min[32], s_max[32];
    wait_previous();
    const Particles<R> pt{x, v, d.n_pairs, 0, blockIdx.x * (long long)blockDim.x + threadIdx.x,
                          static_cast<long long>(gridDim.x) * blockDim.x};
    step_phase<R>(d, pt, current_step(d), s_lev, s_min, s_max, nullptr);
}

// ------------------------------------------------------------------------------------------------ persistent
//
// The whole calibration as one cooperative launch (every block resident at once): per step the three phases above,
// separated by grid barriers, with the step index a loop variable. One block of 512 threads per SM. The barrier is an
// arrival counter in global memory, split in two: grid_arrive after the block's writes, then work that needs nothing
// from the other blocks (clearing the block's bins, the next step's normals), then grid_wait. A block that waits polls
// the counter at most d.wait_limit times, then records OB_ETIMEOUT in d.status and returns, and every other block
// leaves at its next barrier on seeing the status, so a calibration whose barrier cannot complete ends with an error
// instead of holding the GPU.

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int status_of(const LevDev& d) { return *reinterpret_cast<volatile int*>(d.status); }

__device__ __forceinline__ void red_release_gpu(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The counter only grows: a block adds one (a release) once all its threads' writes are done, and its next wait lasts
// until the count reaches every block's arrivals so far (`arrived`, advanced by gridDim.x at each arrival, the same in
// every thread).
__device__ __forceinline__ void grid_arrive(const LevDev& d, unsigned& arrived) {
    arrived += gridDim.x;
    __syncthreads();
    if (threadIdx.x == 0) {
        bulk_wait_all();             // this block's bulk reductions are done
        fence_proxy_async_global();  // and ordered before the release below
        __threadfence();
        red_release_gpu(d.bar_count, 1u);
    }
}

// Every block's writes before its grid_arrive are visible to every thread after this (the acquiring load, then the
// block's barrier). A block polls at most d.wait_limit times (with a limit of zero it gives up at once), then records
// OB_ETIMEOUT; a block that sees the status (read every 32 polls) leaves. Once the count is reached every block has
// arrived, so none has given up at this barrier. False: the calibration has failed and the caller returns.
__device__ bool grid_wait(const LevDev& d, unsigned arrived) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        for (long long polls = 0;; ++polls) {
            if (polls >= d.wait_limit) {
                atomicCAS(d.status, 0, OB_ETIMEOUT);
                ok = 0;
                break;
            }
            if (ld_acquire_gpu(d.bar_count) >= arrived) break;
            if ((polls & 31) == 31 && status_of(d) != 0) {
                ok = 0;
                break;
            }
            if (polls > 256) __nanosleep(32);
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

constexpr int kPersistentThreads = 512;

// Block b owns pairs [b chunk, (b + 1) chunk) and keeps their particles in its shared memory (after the binning
// arrays, at part_off) for the whole calibration: the binning and the step read them there, not through L2. With
// z_off, the block computes each step's normals ahead (while the range of the particles arrives) into shared memory
// at z_off; with row_off, a regression block stages the step's local-variance row there while it waits at the barrier
// before the regression.
template <typename R>
__global__ void __launch_bounds__(kPersistentThreads, 1)
    lev_persistent(LevDev d, long long chunk, int part_off, int z_off, int row_off, double n_particles) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ RegressShared rs;
    __shared__ R s_lev[kMaxX];
    __shared__ R s_min[32], s_max[32];
    const BinShared b = bin_shared(d, sm);
    const long long first = static_cast<long long>(blockIdx.x) * chunk;
    const long long count = first < d.n_pairs ? (d.n_pairs - first < chunk ? d.n_pairs - first : chunk) : 0;
    R* sx = reinterpret_cast<R*>(sm + part_off);
    R* sv = sx + 2 * chunk;
    R* s_z = z_off ? reinterpret_cast<R*>(sm + z_off) : nullptr;
    double* s_row = row_off ? reinterpret_cast<double*>(sm + row_off) : nullptr;
    const Particles<R> pt{sx, sv, count, first, threadIdx.x, blockDim.x};
    for (long long j = threadIdx.x; j < 2 * count; j += blockDim.x) sx[j] = R(0), sv[j] = static_cast<R>(d.v0);
    if (blockIdx.x == 0 && threadIdx.x == 0) d.rng[0] = 0x7fffffffffffffffLL, d.rng[1] = -0x7fffffffffffffffLL - 1;
    bin_clear_shared(d, b);
    unsigned arrived = 0;
    // (step 0's regression reads no particle; the barrier after it orders these stores before the first step)
    const bool regresses = static_cast<int>(blockIdx.x) < d.n_x;
    if (regresses) regress_stage(d, 0, rs, s_row);  // (ordered before step 0's regression by the barrier below)
    __syncthreads();
    for (int i = 0; i < d.n_steps; ++i) {
        double lo = 0.0, hi = 0.0;
        if (i > 0) {
            // the range's keys are loaded first; the step's normals are computed while they arrive
            const long long* r = d.rng + 2 * ((i - 1) & 1);
            const long long k_lo = __ldcg(r), k_hi = __ldcg(r + 1);
            if (s_z) step_normals(d, pt, i, s_z);
            lo = from_order_key(k_lo), hi = from_order_key(k_hi);
            bin_phase<R, true>(d, pt, b, lo, hi);
            grid_arrive(d, arrived);
            if (regresses) regress_stage(d, i, rs, s_row);  // (while thread 0 waits for the bulk reductions)
            if (!grid_wait(d, arrived)) return;
        }
        for (int g = blockIdx.x; g < d.n_x; g += gridDim.x)
            regress_phase(d, n_particles, g, i, lo, hi, rs, b.fine, s_row, g + static_cast<int>(gridDim.x) < d.n_x);
        grid_arrive(d, arrived);
        bin_clear_shared(d, b);
        if (i == 0 && s_z) step_normals(d, pt, 0, s_z);
        if (!grid_wait(d, arrived)) return;
        step_phase<R, true>(d, pt, i, s_lev, s_min, s_max, s_z);
        if (i + 1 < d.n_steps) {
            grid_arrive(d, arrived);
            if (!grid_wait(d, arrived)) return;
        }
    }
}

// Polls of a grid barrier before it gives up (ob_set_wait_limit): a barrier completes within one phase, microseconds;
// the default, 2^22 polls with a short sleep between them, is about a second.
constexpr long long kDefaultWaitLimit = 1LL << 22;
long long g_wait_limit = kDefaultWaitLimit;

// Dynamic shared memory of a persistent block at most: the binning arrays and the block's particles, then (when they
// fit) the step's normals and the local-variance row.
constexpr size_t kPersistentSmemMax = size_t(200) << 10;

__host__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~static_cast<size_t>(15); }

// The persistent calibration on stream st; false (nothing launched) when a block's particles do not fit its shared
// memory or the device cannot hold every block at once.
template <typename R>
bool run_persistent(LevDev& d, double n_particles, size_t bin_smem, int sms, cudaStream_t st) {
    const long long chunk = (d.n_pairs + sms - 1) / sms;
    const size_t part_off = align16(bin_smem);
    size_t smem = part_off + 4 * static_cast<size_t>(chunk) * sizeof(R);
    if (smem > kPersistentSmemMax) return false;
    size_t z_off = 0, row_off = 0;
    if (align16(smem) + 2 * static_cast<size_t>(chunk) * sizeof(R) <= kPersistentSmemMax)
        z_off = align16(smem), smem = z_off + 2 * static_cast<size_t>(chunk) * sizeof(R);
    if (row_staged(d.n_lv) && align16(smem) + static_cast<size_t>(d.n_lv) * sizeof(double) <= kPersistentSmemMax)
        row_off = align16(smem), smem = row_off + static_cast<size_t>(d.n_lv) * sizeof(double);
    allow_smem(reinterpret_cast<const void*>(lev_persistent<R>), smem);
    const int occ = occupancy(reinterpret_cast<const void*>(lev_persistent<R>), kPersistentThreads, smem);
    int coop = 0, dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "cudaDeviceGetAttribute");
    if (occ < 1 || !coop) return false;
    int p_off = static_cast<int>(part_off), zo = static_cast<int>(z_off), ro = static_cast<int>(row_off);
    long long ch = chunk;
    void* args[] = {&d, &ch, &p_off, &zo, &ro, &n_particles};
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
    d.nfp = (nf + kFinePad - 1) / kFinePad * kFinePad;
    d.nbq = (nb + 1 + 3) / 4 * 4;
    const size_t n_c = static_cast<size_t>(d.nbq);
    d.fine = arena.alloc<unsigned>(d.nfp);
    d.cnt = arena.alloc<unsigned>(n_c);
    d.sv = arena.alloc<unsigned long long>(n_c);
    d.acc_ll = arena.alloc<double>(3 * static_cast<size_t>(nb));
    d.rng = arena.alloc<long long>(4);
    check_cuda(cudaMemset(d.fine, 0, d.nfp * sizeof(unsigned)), "cudaMemset");
    check_cuda(cudaMemset(d.cnt, 0, n_c * sizeof(unsigned)), "cudaMemset");
    check_cuda(cudaMemset(d.sv, 0, n_c * sizeof(unsigned long long)), "cudaMemset");
    check_cuda(cudaMemset(d.acc_ll, 0, 3 * nb * sizeof(double)), "cudaMemset");
    d.x_eval = arena.alloc<double>(rq.n_x);
    d.lev = arena.alloc<double>(rq.n_x);
    d.x_grids = arena.alloc<double>(static_cast<size_t>(S) * rq.n_x);
    d.values = arena.alloc<double>(static_cast<size_t>(S) * rq.n_x);
    R* x = arena.alloc<R>(n);
    R* v = arena.alloc<R>(n);
    d.step = arena.alloc<int>(1);
    const size_t bin_smem = bin_smem_bytes(d.nfp, d.nbq, nb, ll);
    check_cuda(cudaFuncSetAttribute(lev_bin<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(bin_smem)),
               "cudaFuncSetAttribute");
    // one binning block an SM (fewer for small particle counts): each block bins many particles before it adds
    const int n_bin_blocks = static_cast<int>(std::max<long long>(1, std::min<long long>(sms, (n + 511) / 512)));
    // the three-kernel schedule's lev_step blocks (up to 4 an SM) each write their range
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
    // OPTLAB_B200_LEVERAGE=graphs runs the three-kernel schedule below instead, =unpacked the persistent kernel with a
    // 32-bit fine histogram (to compare them; same results)
    const char* mode = std::getenv("OPTLAB_B200_LEVERAGE");
    const bool graphs_only = mode && std::strcmp(mode, "graphs") == 0;
    const bool unpacked = mode && std::strcmp(mode, "unpacked") == 0;
    // a persistent block bins 2 chunk particles: packed 16-bit counts hold them
    d.packed = !unpacked && 2 * ((rq.n_pairs + sms - 1) / sms) < 65536;
    for (int attempt = 0; !graphs_only && attempt < 2; ++attempt) {
        if (!run_persistent<R>(d, n_particles, bin_smem, sms, st)) break;
        int status = 0;
        check_cuda(cudaMemcpyAsync(&status, d.status, sizeof status, cudaMemcpyDeviceToHost, st), "copy status");
        check_cuda(cudaStreamSynchronize(st), "leverage");
        if (status == kPackOverflow && d.packed) {
            // a fine bin held 2^16 particles or more: the same calibration again, unpacked, from clean buffers
            d.packed = 0;
            check_cuda(cudaMemset(d.fine, 0, d.nfp * sizeof(unsigned)), "cudaMemset");
            check_cuda(cudaMemset(d.cnt, 0, n_c * sizeof(unsigned)), "cudaMemset");
            check_cuda(cudaMemset(d.sv, 0, n_c * sizeof(unsigned long long)), "cudaMemset");
            check_cuda(cudaMemset(d.acc_ll, 0, 3 * nb * sizeof(double)), "cudaMemset");
            check_cuda(cudaMemset(d.bar_count, 0, 4 * sizeof(unsigned)), "cudaMemset");
            continue;
        }
        if (status == OB_ETIMEOUT)
            throw Error(OB_ETIMEOUT, "leverage: a grid barrier of the calibration gave up waiting for the other blocks");
        if (status != 0) throw Error(OB_ECUDA, "leverage: the calibration kernel reported a failure");
        check_cuda(cudaMemcpyAsync(rq.x_grids, d.x_grids, static_cast<size_t>(S) * rq.n_x * sizeof(double),
                                   cudaMemcpyDeviceToHost, st),
                   "copy x_grids");
        check_cuda(cudaMemcpyAsync(rq.values, d.values, static_cast<size_t>(S) * rq.n_x * sizeof(double),
                                   cudaMemcpyDeviceToHost, st),
                   "copy values");
        check_cuda(cudaStreamSynchronize(st), "leverage");
        rq.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        return;
    }
    // the device cannot hold the persistent kernel: three kernels a step, replayed as graphs
    d.packed = 0;
    d.n_step_blocks = static_cast<int>(std::max<long long>(1, std::min<long long>(4LL * sms, (rq.n_pairs + 255) / 256)));
    lev_init<R><<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(x, v, n, static_cast<R>(rq.v0), d.step);
    check_cuda(cudaGetLastError(), "lev_init launch");
    const R* cx = x;
    const R* cv = v;
    // step 0 (no binning: the particles all start at x = 0), launched directly
    const size_t reg_smem = static_cast<size_t>(d.nfp) * sizeof(unsigned) +
                            (row_staged(rq.n_lv) ? static_cast<size_t>(rq.n_lv) * sizeof(double) : 0);
    check_cuda(cudaFuncSetAttribute(lev_regress, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(reg_smem)),
               "cudaFuncSetAttribute");
    const cudaLaunchConfig_t c_reg0 = config(rq.n_x, 256, reg_smem), c_step0 = config(d.n_step_blocks, 256, 0);
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
    const cudaLaunchConfig_t c_reg = on(config(rq.n_x, 256, reg_smem));
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
