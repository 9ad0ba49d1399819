// The issuer's Longstaff-Schwartz policy fitted on the device (see exercise.cuh). The method is the reference's
// (packages/structured/src/optlab/structured/exercise.py:212-252): backward over the events from the last, a
// non-call event adds its flows to the note's future value; at a call the continuation per unit reached, in money of
// the call date, is regressed on polynomials and hinges of the normalised state (basis :125-140) over the paths the
// call reaches, and the issuer calls where the fitted continuation is above the amount.
//
// Every pass over the paths runs on the device, with the pilot's record where the pilot left it: the preparation of a
// call (the flows of the events since the last call, the regressand, the reached paths' state as dense columns,
// their count and sums), the state's variance and extremes, the order statistics of the deciles (one block per order
// statistic, a radix select on the doubles' sort keys), the normal equations of the regression (the Gram matrix of
// the features and their product with the regressand, per-block sums added in block order), the residual's products
// for the refinement, and the decisions with the new future value. Between the passes the host does what needs a few
// numbers only: numpy's quantile arithmetic on the selected order statistics (numpy.quantile, 'linear': the virtual
// index (n - 1) q, its floor and the next, and numpy's two-sided interpolation), the choice of the basis, and the
// Cholesky solve of the (at most 25 x 25) normal equations followed by two steps of iterative refinement, which
// brings the solution to the least-squares solution the reference's SVD solve (numpy.linalg.lstsq) finds, to the
// conditioning of the features times the double precision. A basis whose normal equations have a pivot below 1e-13
// of its diagonal (features nearly collinear) is refused: the caller fits on the host instead.
#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

#include "exercise.cuh"

namespace ob {

namespace {

constexpr int kMaxTerms = 25;         // regression terms, the constant included (exercise.py MAX_TERMS)
constexpr int kMaxKnots = 9;          // hinges per state variable, at its deciles (MAX_KNOTS)
constexpr int kMinPathsPerTerm = 20;  // paths a term needs (MIN_PATHS_PER_TERM)
constexpr int kFitThreads = 256;
constexpr int kSelThreads = 512;
constexpr int kMaxAcc = kMaxTerms * kMaxTerms + kMaxTerms;  // the Gram matrix, then its product with the regressand
constexpr int kMaxTargets = 4 * 2 * kMaxKnots;              // order statistics: two a decile, four state variables

struct FitDev {
    const double* rec;     // the pilot's record, n_paths x stride
    long long P;           // paths
    int stride, n_events, n_state;
    double* future;        // P: the note's value from the current event on, not called
    double* after;         // P: the call's flows after its call statement, plus the future
    double* y;             // P: the regressand (0 where the call does not reach the path)
    double* xcol;          // n_state x P: the call's state
    unsigned char* on;     // P: the call reaches the path
    int k, c;              // the current call's event and index
    double d;              // its payment's discount factor (1 where it pays nothing counted)
    int T, n_poly, n_knots;
    double mean[4], scale[4];
    signed char pw[kMaxTerms][4];
    signed char kvar[kMaxTerms];
    double knot[kMaxTerms];
    double coef[kMaxTerms];
};

__device__ __forceinline__ const double* row_of(const FitDev& f, long long j) { return f.rec + j * f.stride; }
__host__ __device__ __forceinline__ int call_base(int n_events, int n_state, int c) {
    return 2 * n_events + c * (3 + n_state);
}

// The sum of v over the block, in thread 0 (warp butterflies, then the warps in order).
__device__ double block_sum(double v, double* s_red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < nw; ++w) s += s_red[w];
    __syncthreads();
    return s;
}

__device__ double block_min(double v, double* s_red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    double s = v;
    if (threadIdx.x == 0)
        for (int w = 0; w < nw; ++w) s = fmin(s, s_red[w]);
    __syncthreads();
    return s;
}

__device__ double block_max(double v, double* s_red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    double s = v;
    if (threadIdx.x == 0)
        for (int w = 0; w < nw; ++w) s = fmax(s, s_red[w]);
    __syncthreads();
    return s;
}

// The events since the last call (pend, from the latest) add their flows to the future, (pre + post) + future as the
// reference adds them; with a call, its preparation: after = post + future, the reached mass mask x alive, the
// regressand after / (d reached) where it is positive, the state as dense columns; the block's count of reached paths
// and sums of their state into part (1 + n_state a block).
__global__ void __launch_bounds__(kFitThreads) ex_prep(FitDev f, const int* pend, int n_pend, int with_call,
                                                       double* part) {
    __shared__ double s_red[kFitThreads / 32];
    const int ns = f.n_state;
    const int base = call_base(f.n_events, ns, f.c);
    double cnt = 0.0, sx[4] = {0.0, 0.0, 0.0, 0.0};
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; j < f.P; j += stride) {
        const double* r = row_of(f, j);
        double fu = f.future[j];
        for (int q = 0; q < n_pend; ++q) {
            const int kk = pend[q];
            fu = (r[2 * kk] + r[2 * kk + 1]) + fu;
        }
        f.future[j] = fu;
        if (with_call) {
            const double af = r[2 * f.k + 1] + fu;
            const double reach = __dmul_rn(r[base], r[base + 1]);
            const bool o = reach > 0.0;
            f.after[j] = af;
            f.y[j] = o ? af / __dmul_rn(f.d, reach) : 0.0;
            f.on[j] = o ? 1 : 0;
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (i < ns) {
                    const double x = r[base + 3 + i];
                    f.xcol[i * f.P + j] = x;
                    sx[i] += o ? x : 0.0;
                }
            cnt += o ? 1.0 : 0.0;
        }
    }
    if (!with_call) return;
    const double c = block_sum(cnt, s_red);
    if (threadIdx.x == 0) part[blockIdx.x * 5] = c;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i >= ns) break;
        const double s = block_sum(sx[i], s_red);
        if (threadIdx.x == 0) part[blockIdx.x * 5 + 1 + i] = s;
    }
}

// The reached paths' squared deviations from the means, and their state's extremes: part (3 n_state a block: sums,
// then minima, then maxima).
__global__ void __launch_bounds__(kFitThreads) ex_moments(FitDev f, double* part) {
    __shared__ double s_red[kFitThreads / 32];
    const int ns = f.n_state;
    double ss[4] = {0.0, 0.0, 0.0, 0.0}, mn[4], mx[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) mn[i] = INFINITY, mx[i] = -INFINITY;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; j < f.P; j += stride) {
        if (!f.on[j]) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i < ns) {
                const double x = f.xcol[i * f.P + j], dx = x - f.mean[i];
                ss[i] += __dmul_rn(dx, dx);
                mn[i] = fmin(mn[i], x), mx[i] = fmax(mx[i], x);
            }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i >= ns) break;
        const double s = block_sum(ss[i], s_red), lo = block_min(mn[i], s_red), hi = block_max(mx[i], s_red);
        if (threadIdx.x == 0) {
            part[blockIdx.x * 12 + i] = s;
            part[blockIdx.x * 12 + 4 + i] = lo;
            part[blockIdx.x * 12 + 8 + i] = hi;
        }
    }
}

// Doubles as unsigned keys in the same order (negatives with every bit flipped, the others with the sign bit set).
__device__ __forceinline__ unsigned long long sort_key(double x) {
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double from_sort_key(unsigned long long k) {
    return __longlong_as_double(static_cast<long long>((k >> 63) ? (k & 0x7fffffffffffffffull) : ~k));
}

// Exclusive prefix of x over the block and the block's total (blocks of up to 1024 threads, a multiple of 32).
__device__ unsigned long long scan_block(unsigned long long x, unsigned long long* s_warp, unsigned long long& total) {
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

// Block b: the order statistic of rank t_rank[b] (0: the least) of state variable t_var[b] over the reached paths, by
// a most-significant-digit-first radix select on the sort keys (digits of 11, 11, 11, 11, 10, 10 bits).
__global__ void __launch_bounds__(kSelThreads) ex_select(FitDev f, const int* t_var, const long long* t_rank,
                                                         double* out) {
    __shared__ unsigned hist[2048];
    __shared__ unsigned long long s_warp[32];
    __shared__ int s_bin;
    __shared__ unsigned long long s_before;
    const double* x = f.xcol + static_cast<long long>(t_var[blockIdx.x]) * f.P;
    unsigned long long rank = static_cast<unsigned long long>(t_rank[blockIdx.x]);
    unsigned long long prefix = 0, known = 0;
    int shift = 64;
    for (int pass = 0; pass < 6; ++pass) {
        const int bits = pass < 4 ? 11 : 10;
        shift -= bits;
        const unsigned nbin = 1u << bits;
        for (int b = threadIdx.x; b < 2048; b += blockDim.x) hist[b] = 0u;
        if (threadIdx.x == 0) s_bin = 0, s_before = 0;
        __syncthreads();
        for (long long j = threadIdx.x; j < f.P; j += blockDim.x) {
            if (!f.on[j]) continue;
            const unsigned long long key = sort_key(x[j]);
            if ((key & known) != prefix) continue;
            atomicAdd(&hist[(key >> shift) & (nbin - 1)], 1u);
        }
        __syncthreads();
        // each thread a run of bins; the run holding the rank finds its bin
        const int per = static_cast<int>((nbin + blockDim.x - 1) / blockDim.x);
        const int b0 = static_cast<int>(threadIdx.x) * per;
        unsigned long long mine = 0;
        for (int b = b0; b < b0 + per && b < static_cast<int>(nbin); ++b) mine += hist[b];
        unsigned long long total;
        const unsigned long long before = scan_block(mine, s_warp, total);
        if (mine > 0 && rank >= before && rank < before + mine) {
            unsigned long long cum = before;
            for (int b = b0; b < b0 + per && b < static_cast<int>(nbin); ++b) {
                if (rank < cum + hist[b]) {
                    s_bin = b, s_before = cum;
                    break;
                }
                cum += hist[b];
            }
        }
        __syncthreads();
        prefix |= static_cast<unsigned long long>(s_bin) << shift;
        known |= static_cast<unsigned long long>(nbin - 1) << shift;
        rank -= s_before;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = from_sort_key(prefix);
}

__device__ __forceinline__ double ipow(double z, int p) {
    return p == 0 ? 1.0 : p == 1 ? z : p == 2 ? __dmul_rn(z, z) : __dmul_rn(__dmul_rn(z, z), z);
}

// The regression's terms of one path's state: the monomials of the normalised state z (the product of the variables'
// powers, in order), then the hinges max(z_i - k, 0).
__device__ __forceinline__ void features(const FitDev& f, const double* xs, double* F) {
    double z[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) z[i] = i < f.n_state ? (xs[i] - f.mean[i]) / f.scale[i] : 0.0;
#pragma unroll
    for (int a = 0; a < kMaxTerms; ++a) {
        if (a >= f.n_poly) break;
        double v = ipow(z[0], f.pw[a][0]);
#pragma unroll
        for (int i = 1; i < 4; ++i)
            if (i < f.n_state) v = __dmul_rn(v, ipow(z[i], f.pw[a][i]));
        F[a] = v;
    }
#pragma unroll
    for (int q = 0; q < kMaxTerms; ++q) {
        if (q >= f.n_knots) break;
        const int v = f.kvar[q];
        double zv = z[0];
#pragma unroll
        for (int i = 1; i < 4; ++i) zv = v == i ? z[i] : zv;
        F[f.n_poly + q] = fmax(zv - f.knot[q], 0.0);
    }
}

// The normal equations over the reached paths, a tile of blockDim paths at a time staged in shared memory (the terms
// of the tile's paths by term, then the weight): mode 0 the Gram matrix F'F (T x T) and F'y; mode 1 F'r, r = y - F
// coef, the refinement's right-hand side. Per-block sums into part (n_acc a block).
__global__ void __launch_bounds__(kFitThreads) ex_gram(FitDev f, int mode, double* part) {
    extern __shared__ double s_F[];  // (T + 1) rows of kFitThreads + 1
    const int T = f.T, ld = kFitThreads + 1, nt = blockDim.x, t = threadIdx.x;
    const int n_acc = mode == 0 ? T * T + T : T;
    double acc[3] = {0.0, 0.0, 0.0};
    for (long long tile = static_cast<long long>(blockIdx.x) * nt; tile < f.P; tile += static_cast<long long>(gridDim.x) * nt) {
        const long long j = tile + t;
        double F[kMaxTerms];
        double w = 0.0;
        const bool o = j < f.P && f.on[j];
        if (o) {
            double xs[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) xs[i] = i < f.n_state ? f.xcol[i * f.P + j] : 0.0;
            features(f, xs, F);
            if (mode == 0) {
                w = f.y[j];
            } else {
                double cont = 0.0;
#pragma unroll
                for (int a = 0; a < kMaxTerms; ++a)
                    if (a < T) cont += F[a] * f.coef[a];
                w = f.y[j] - cont;
            }
        }
#pragma unroll
        for (int a = 0; a < kMaxTerms; ++a)
            if (a < T) s_F[a * ld + t] = o ? F[a] : 0.0;
        s_F[T * ld + t] = w;
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const int e = t + u * nt;
            if (e >= n_acc) break;
            const int a = mode == 0 ? (e < T * T ? e / T : e - T * T) : e;
            const int b = mode == 0 && e < T * T ? e % T : T;
            double s = 0.0;
            for (int p = 0; p < nt; ++p) s += s_F[a * ld + p] * s_F[b * ld + p];
            acc[u] += s;
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 3; ++u) {
        const int e = t + u * nt;
        if (e < n_acc) part[static_cast<long long>(blockIdx.x) * n_acc + e] = acc[u];
    }
}

// Per-block sums added in block order: out[e] = sum over b of part[b n_acc + e].
__global__ void ex_finalize(const double* part, int n_blocks, int n_acc, double* out) {
    for (int e = threadIdx.x; e < n_acc; e += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < n_blocks; ++b) s += part[static_cast<long long>(b) * n_acc + e];
        out[e] = s;
    }
}

// The issuer's decisions at the current call and the future value from it on: called = mask x (continuation above
// the amount), paid = d called alive amount, future = pre + (1 - called) after + paid (every rounding as the
// reference's array operations make it).
__global__ void __launch_bounds__(kFitThreads) ex_decide(FitDev f, int has_rule) {
    const int base = call_base(f.n_events, f.n_state, f.c);
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; j < f.P; j += stride) {
        const double* r = row_of(f, j);
        double decide = 0.0;
        if (has_rule) {
            double xs[4], F[kMaxTerms];
#pragma unroll
            for (int i = 0; i < 4; ++i) xs[i] = i < f.n_state ? r[base + 3 + i] : 0.0;
            features(f, xs, F);
            double cont = 0.0;
#pragma unroll
            for (int a = 0; a < kMaxTerms; ++a)
                if (a < f.T) cont += F[a] * f.coef[a];
            decide = cont > r[base + 2] ? 1.0 : 0.0;
        }
        const double called = __dmul_rn(r[base], decide);
        const double paid = __dmul_rn(__dmul_rn(__dmul_rn(f.d, called), r[base + 1]), r[base + 2]);
        f.future[j] = __dadd_rn(__dadd_rn(r[2 * f.k], __dmul_rn(1.0 - called, f.after[j])), paid);
    }
}

// The future's sum, per block into part.
__global__ void __launch_bounds__(kFitThreads) ex_total(FitDev f, double* part) {
    __shared__ double s_red[kFitThreads / 32];
    double s = 0.0;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; j < f.P; j += stride)
        s += f.future[j];
    s = block_sum(s, s_red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Exponents of the monomials of total degree <= degree in d variables: the constant first, then by degree, each
// degree in the order of itertools.combinations_with_replacement(range(d), degree) (exercise.py:112-122).
std::vector<std::array<int, 4>> powers(int d, int degree) {
    std::vector<std::array<int, 4>> out;
    if (d <= 0) return {{0, 0, 0, 0}};  // no variable: the constant only
    for (int total = 0; total <= degree; ++total) {
        std::vector<int> combo(static_cast<size_t>(total), 0);
        while (true) {
            std::array<int, 4> p{0, 0, 0, 0};
            for (int v : combo) ++p[v];
            out.push_back(p);
            int pos = total - 1;
            while (pos >= 0 && combo[pos] == d - 1) --pos;
            if (pos < 0) break;
            ++combo[pos];
            for (int q = pos + 1; q < total; ++q) combo[q] = combo[pos];
        }
    }
    return out;
}

// numpy.quantile's linear interpolation between two order statistics a <= b at weight t (numpy's _lerp: from a below
// one half, from b above).
double np_lerp(double a, double b, double t) {
    const double diff = b - a;
    return t >= 0.5 ? b - diff * (1.0 - t) : a + diff * t;
}

// Cholesky solve of the normal equations G c = rhs over the terms `use` (the others' coefficients 0). False when a
// pivot falls below 1e-13 of its diagonal.
bool solve_normal(const std::vector<double>& G, int T, const std::vector<int>& use, const std::vector<double>& rhs,
                  std::vector<double>& c) {
    const int m = static_cast<int>(use.size());
    std::vector<double> L(static_cast<size_t>(m) * m, 0.0);
    for (int j = 0; j < m; ++j) {
        const double gjj = G[static_cast<size_t>(use[j]) * T + use[j]];
        double s = gjj;
        for (int k = 0; k < j; ++k) s -= L[j * m + k] * L[j * m + k];
        if (!(s > 1e-13 * gjj)) return false;
        const double l = std::sqrt(s);
        L[j * m + j] = l;
        for (int i = j + 1; i < m; ++i) {
            double v = G[static_cast<size_t>(use[i]) * T + use[j]];
            for (int k = 0; k < j; ++k) v -= L[i * m + k] * L[j * m + k];
            L[i * m + j] = v / l;
        }
    }
    std::vector<double> u(m);
    for (int i = 0; i < m; ++i) {
        double v = rhs[use[i]];
        for (int k = 0; k < i; ++k) v -= L[i * m + k] * u[k];
        u[i] = v / L[i * m + i];
    }
    c.assign(T, 0.0);
    for (int i = m - 1; i >= 0; --i) {
        double v = u[i];
        for (int k = i + 1; k < m; ++k) v -= L[k * m + i] * c[use[k]];
        c[use[i]] = v / L[i * m + i];
    }
    return true;
}

}  // namespace

bool fit_policy_on_device(const double* record, long long P, int stride, int n_events, int n_calls, int n_state,
                          const int* call_event, const double* pay_discount, double* rules, double* in_sample,
                          DeviceArena& arena) {
    const int sms = require_device();
    const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>(4LL * sms, (P + kFitThreads - 1) / kFitThreads)));
    const int ns = n_state;
    FitDev f{};
    f.rec = record, f.P = P, f.stride = stride, f.n_events = n_events, f.n_state = ns;
    f.future = arena.alloc<double>(P);
    f.after = arena.alloc<double>(P);
    f.y = arena.alloc<double>(P);
    f.xcol = arena.alloc<double>(static_cast<size_t>(std::max(1, ns)) * P);
    f.on = arena.alloc<unsigned char>(P);
    check_cuda(cudaMemset(f.future, 0, P * sizeof(double)), "cudaMemset");
    double* part = arena.alloc<double>(static_cast<size_t>(grid) * kMaxAcc);
    double* fin = arena.alloc<double>(kMaxAcc);
    int* d_pend = arena.alloc<int>(std::max(1, n_events));
    int* d_tvar = arena.alloc<int>(kMaxTargets);
    long long* d_trank = arena.alloc<long long>(kMaxTargets);
    double* d_tval = arena.alloc<double>(kMaxTargets);
    const size_t gram_smem = static_cast<size_t>(kMaxTerms + 1) * (kFitThreads + 1) * sizeof(double);
    check_cuda(cudaFuncSetAttribute(ex_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(gram_smem)),
               "cudaFuncSetAttribute");
    std::vector<int> call_of(n_events, -1);
    for (int c = 0; c < n_calls; ++c) call_of[call_event[c]] = c;
    std::fill(rules, rules + static_cast<size_t>(n_calls) * OB_RULE_STRIDE, 0.0);
    std::vector<double> host_part(static_cast<size_t>(grid) * kMaxAcc);
    // the per-block sums of a pass, added in block order on the host
    auto block_sums = [&](int width, std::vector<double>& out) {
        check_cuda(cudaMemcpy(host_part.data(), part, static_cast<size_t>(grid) * width * sizeof(double),
                              cudaMemcpyDeviceToHost),
                   "copy sums");
        out.assign(width, 0.0);
        for (int b = 0; b < grid; ++b)
            for (int e = 0; e < width; ++e) out[e] += host_part[static_cast<size_t>(b) * width + e];
    };
    auto normal_pass = [&](int mode, int n_acc, std::vector<double>& out) {
        ex_gram<<<grid, kFitThreads, gram_smem>>>(f, mode, part);
        check_cuda(cudaGetLastError(), "ex_gram launch");
        ex_finalize<<<1, 256>>>(part, grid, n_acc, fin);
        check_cuda(cudaGetLastError(), "ex_finalize launch");
        out.resize(n_acc);
        check_cuda(cudaMemcpy(out.data(), fin, n_acc * sizeof(double), cudaMemcpyDeviceToHost), "copy normal equations");
    };
    std::vector<int> pend;
    auto run_pending = [&](int with_call) {
        if (!pend.empty())
            check_cuda(cudaMemcpy(d_pend, pend.data(), pend.size() * sizeof(int), cudaMemcpyHostToDevice), "copy events");
        ex_prep<<<grid, kFitThreads>>>(f, d_pend, static_cast<int>(pend.size()), with_call, part);
        check_cuda(cudaGetLastError(), "ex_prep launch");
        pend.clear();
    };
    for (int k = n_events - 1; k >= 0; --k) {
        const int c = call_of[k];
        if (c < 0) {
            pend.push_back(k);
            continue;
        }
        f.k = k, f.c = c, f.d = pay_discount[k] > 0 ? pay_discount[k] : 1.0;
        run_pending(1);
        std::vector<double> s;
        block_sums(5, s);
        const long long n_on = static_cast<long long>(s[0]);
        int has_rule = 0;
        if (n_on > 0) {
            for (int i = 0; i < ns; ++i) f.mean[i] = s[1 + i] / static_cast<double>(n_on);
            ex_moments<<<grid, kFitThreads>>>(f, part);
            check_cuda(cudaGetLastError(), "ex_moments launch");
            std::vector<double> mom(12, 0.0);
            check_cuda(cudaMemcpy(host_part.data(), part, static_cast<size_t>(grid) * 12 * sizeof(double),
                                  cudaMemcpyDeviceToHost),
                       "copy moments");
            double mn[4], mx[4];
            for (int i = 0; i < ns; ++i) {
                double ss = 0.0;
                mn[i] = INFINITY, mx[i] = -INFINITY;
                for (int b = 0; b < grid; ++b) {
                    ss += host_part[static_cast<size_t>(b) * 12 + i];
                    mn[i] = std::fmin(mn[i], host_part[static_cast<size_t>(b) * 12 + 4 + i]);
                    mx[i] = std::fmax(mx[i], host_part[static_cast<size_t>(b) * 12 + 8 + i]);
                }
                const double sc = std::sqrt(ss / static_cast<double>(n_on));
                f.scale[i] = sc > 0 ? sc : 1.0;
            }
            // the basis (exercise.py:125-140): the highest degree whose monomials fit the room, then hinges at deciles
            const int room = static_cast<int>(std::min<long long>(kMaxTerms, n_on / kMinPathsPerTerm));
            const int degrees[3] = {ns == 1 ? 3 : (ns <= 4 ? 2 : 1), 1, 0};
            std::vector<std::array<int, 4>> pw;
            for (int deg : degrees) {
                pw = powers(ns, deg);
                if (static_cast<int>(pw.size()) <= room) break;
            }
            const int per = std::max(0, std::min(kMaxKnots, (room - static_cast<int>(pw.size())) / std::max(1, ns)));
            // order statistics the deciles need: numpy.quantile, 'linear', at q = j / (per + 1)
            std::vector<int> tv;
            std::vector<long long> tr;
            std::vector<double> gam;
            std::vector<int> tq;  // per (variable, decile): the index of its lower order statistic in tv
            const double step = 1.0 / static_cast<double>(per + 1);
            for (int i = 0; i < ns && per > 0; ++i)
                for (int j = 1; j <= per; ++j) {
                    const double q = static_cast<double>(j) * step;
                    const double h = static_cast<double>(n_on - 1) * q;
                    long long lo_i, hi_i;
                    double g;
                    if (h >= static_cast<double>(n_on - 1)) lo_i = hi_i = n_on - 1, g = h + 1.0;
                    else if (h < 0) lo_i = hi_i = 0, g = h;
                    else lo_i = static_cast<long long>(std::floor(h)), hi_i = lo_i + 1, g = h - std::floor(h);
                    tq.push_back(static_cast<int>(tv.size()));
                    tv.push_back(i), tr.push_back(lo_i);
                    tv.push_back(i), tr.push_back(hi_i);
                    gam.push_back(g);
                }
            std::vector<double> tval(tv.size());
            if (!tv.empty()) {
                check_cuda(cudaMemcpy(d_tvar, tv.data(), tv.size() * sizeof(int), cudaMemcpyHostToDevice), "copy targets");
                check_cuda(cudaMemcpy(d_trank, tr.data(), tr.size() * sizeof(long long), cudaMemcpyHostToDevice),
                           "copy targets");
                ex_select<<<static_cast<unsigned>(tv.size()), kSelThreads>>>(f, d_tvar, d_trank, d_tval);
                check_cuda(cudaGetLastError(), "ex_select launch");
                check_cuda(cudaMemcpy(tval.data(), d_tval, tv.size() * sizeof(double), cudaMemcpyDeviceToHost),
                           "copy order statistics");
            }
            std::vector<std::pair<int, double>> knots;
            for (int i = 0; i < ns && per > 0; ++i) {
                std::vector<double> levels;
                for (int j = 0; j < per; ++j) {
                    const int at = tq[static_cast<size_t>(i) * per + j];
                    const double a = (tval[at] - f.mean[i]) / f.scale[i], b = (tval[at + 1] - f.mean[i]) / f.scale[i];
                    levels.push_back(np_lerp(a, b, gam[static_cast<size_t>(i) * per + j]));
                }
                std::sort(levels.begin(), levels.end());
                levels.erase(std::unique(levels.begin(), levels.end()), levels.end());
                const double zlo = (mn[i] - f.mean[i]) / f.scale[i], zhi = (mx[i] - f.mean[i]) / f.scale[i];
                for (double lv : levels)
                    if (zlo < lv && lv < zhi) knots.emplace_back(i, lv);
            }
            f.n_poly = static_cast<int>(pw.size()), f.n_knots = static_cast<int>(knots.size());
            f.T = f.n_poly + f.n_knots;
            if (f.T > kMaxTerms) throw Error(OB_EINVAL, "the pilot fit's basis has more than 25 terms");
            for (int a = 0; a < std::min(f.n_poly, kMaxTerms); ++a)
                for (int i = 0; i < 4; ++i) f.pw[a][i] = static_cast<signed char>(i < ns ? pw[a][i] : 0);
            for (int q = 0; q < std::min(f.n_knots, kMaxTerms); ++q)
                f.kvar[q] = static_cast<signed char>(knots[q].first), f.knot[q] = knots[q].second;
            // normal equations, solved and refined twice (the residual's products on the device)
            const int T = f.T;
            std::vector<double> ge;
            normal_pass(0, T * T + T, ge);
            std::vector<double> G(ge.begin(), ge.begin() + static_cast<long long>(T) * T), rhs(ge.begin() + static_cast<long long>(T) * T, ge.end());
            std::vector<int> use;
            for (int a = 0; a < T; ++a)
                if (G[static_cast<size_t>(a) * T + a] > 0.0) use.push_back(a);  // a term zero on every reached path: 0
            std::vector<double> coef, delta;
            if (use.empty() || !solve_normal(G, T, use, rhs, coef)) return false;
            double last = 0.0, size = 0.0;
            for (int it = 0; it < 2; ++it) {
                for (int a = 0; a < T; ++a) f.coef[a] = coef[a];
                std::vector<double> g;
                normal_pass(1, T, g);
                if (!solve_normal(G, T, use, g, delta)) return false;
                last = size = 0.0;
                for (int a = 0; a < T; ++a) {
                    coef[a] += delta[a];
                    last = std::fmax(last, std::fabs(delta[a])), size = std::fmax(size, std::fabs(coef[a]));
                }
            }
            if (!(last <= 1e-8 * size + 1e-300)) return false;
            for (int a = 0; a < T; ++a) f.coef[a] = coef[a];
            double* row = rules + static_cast<size_t>(c) * OB_RULE_STRIDE;
            row[0] = 1.0, row[1] = f.n_poly, row[2] = f.n_knots;
            for (int i = 0; i < ns; ++i) row[3 + i] = f.mean[i], row[7 + i] = f.scale[i];
            for (int a = 0; a < f.n_poly; ++a)
                for (int i = 0; i < ns; ++i) row[11 + 4 * a + i] = pw[a][i];
            for (int q = 0; q < f.n_knots; ++q) row[111 + q] = knots[q].first, row[136 + q] = knots[q].second;
            for (int a = 0; a < T; ++a) row[161 + a] = coef[a];
            has_rule = 1;
        }
        ex_decide<<<grid, kFitThreads>>>(f, has_rule);
        check_cuda(cudaGetLastError(), "ex_decide launch");
    }
    if (!pend.empty()) run_pending(0);
    ex_total<<<grid, kFitThreads>>>(f, part);
    check_cuda(cudaGetLastError(), "ex_total launch");
    std::vector<double> tot;
    block_sums(1, tot);
    *in_sample = tot[0] / static_cast<double>(P);
    return true;
}

}  // namespace ob
