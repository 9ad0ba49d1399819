// ob_leverage: the drop-in for optlab::api::leverage(rq, 1, 0) (RC/include/optlab_cuda/requests.hpp:107-108), the SLV
// leverage by the particle method of Guyon and Henry-Labordere, as RC/src/leverage.cpp:97-152 (host algorithm) with
// the particle device of RC/src/leverage.cpp:156-214 / RC/src/leverage_gpu.cu:40-106.
//
// Per step i, everything stays on the device (the reference crosses PCIe three times a step):
//   lev_bin        particles -> fine histogram (u32) and the regression's binned sums (count, v, x, x^2, x v) in FP64,
//                  accumulated per block in shared memory, then added to the step's totals
//   lev_regress    one block per grid point g: the quantiles of the fine histogram bound the grid (the reference's
//                  sequential search, restated as a parallel first-match), the Gaussian-kernel regression E[v | x_g]
//                  (Nadaraya-Watson or local linear) over the bins in FP64, and L_g = clip(sqrt(sigma_loc^2 / E), lmin,
//                  lmax) with the local variance interpolated on its uniform row; the row and the grid go straight
//                  into the output tables
//   lev_step       one thread per antithetic pair: the SLV Euler step with the leverage row staged in shared memory,
//                  normals from Philox counter (pair, step + 1, 0, 0), the new range of x by block then global min/max
// Particles are float (OB_FP32) or double (OB_FP64); bins, regression and the leverage ratio are FP64 in both.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace ob {

namespace {

constexpr int kMaxBins = 512;
constexpr int kMaxFine = 16384;
constexpr int kMaxX = 1024;

struct LevDev {
    long long n_pairs;
    int n_x, n_bins, n_fine, n_lv, local_linear, positive_part;
    uint32_t k0, k1;
    double v0, kappa, theta, xi, rho, atm_vol, bw_scale, l_min, l_max, q_lo, q_hi;
    const double* dt;
    const double* t0;
    const double* lv_lo;
    const double* lv_inv_dx;
    const double* lv_rows;
    unsigned* fine;            // n_fine
    double* acc;               // 5 n_bins + 1 (the last: sum of v)
    long long* range;          // ordered min and max of x (double keys)
    double* x_eval;            // n_x, the current grid
    double* lev;               // n_x, the current leverage row
    double* x_grids;           // n_steps x n_x
    double* values;            // n_steps x n_x
};

// Order-preserving map of doubles to signed 64-bit integers, for atomicMin / atomicMax.
__device__ __forceinline__ long long ordered(double d) {
    const long long i = __double_as_longlong(d);
    return i >= 0 ? i : i ^ 0x7FFFFFFFFFFFFFFFLL;
}
__device__ __forceinline__ double unordered(long long i) {
    return __longlong_as_double(i >= 0 ? i : i ^ 0x7FFFFFFFFFFFFFFFLL);
}

__global__ void lev_reset(LevDev d) {
    for (int k = threadIdx.x; k < d.n_fine; k += blockDim.x) d.fine[k] = 0u;
    for (int k = threadIdx.x; k < 5 * d.n_bins + 1; k += blockDim.x) d.acc[k] = 0.0;
}

template <typename R>
__global__ void lev_init(R* x, R* v, long long n, R v0, long long* range) {
    const long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j < n) x[j] = R(0), v[j] = v0;
    if (j == 0) range[0] = ordered(0.0), range[1] = ordered(0.0);
}

// Bin edges and indices as the reference computes them: in double on the CPU, in float on its GPU.
template <typename R>
__global__ void __launch_bounds__(512) lev_bin(LevDev d, const R* __restrict__ x, const R* __restrict__ v) {
    extern __shared__ __align__(16) unsigned char sm[];
    double* sacc = reinterpret_cast<double*>(sm);                     // 5 nb + 1
    unsigned* sfine = reinterpret_cast<unsigned*>(sacc + 5 * d.n_bins + 1);  // n_fine
    const int nb = d.n_bins, nf = d.n_fine;
    for (int k = threadIdx.x; k < 5 * nb + 1; k += blockDim.x) sacc[k] = 0.0;
    for (int k = threadIdx.x; k < nf; k += blockDim.x) sfine[k] = 0u;
    __syncthreads();
    const R lo = static_cast<R>(unordered(d.range[0])), hi = static_cast<R>(unordered(d.range[1]));
    const R wf = (hi - lo) / static_cast<R>(nf), we = (hi + static_cast<R>(1e-12) - lo) / static_cast<R>(nb);
    const long long n = 2 * d.n_pairs;
    for (long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
         j += static_cast<long long>(gridDim.x) * blockDim.x) {
        const R xj = x[j], vj = d.positive_part ? m_max(v[j], R(0)) : v[j];
        const int f = wf > R(0) ? static_cast<int>((xj - lo) / wf) : 0;
        atomicAdd(&sfine[min(max(f, 0), nf - 1)], 1u);
        const int k = min(max(static_cast<int>((xj - lo) / we), 0), nb - 1);
        const double xd = static_cast<double>(xj), vd = static_cast<double>(vj);
        atomicAdd(&sacc[k], 1.0);
        atomicAdd(&sacc[nb + k], vd);
        atomicAdd(&sacc[2 * nb + k], xd);
        atomicAdd(&sacc[3 * nb + k], xd * xd);
        atomicAdd(&sacc[4 * nb + k], xd * vd);
        atomicAdd(&sacc[5 * nb], vd);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 5 * nb + 1; k += blockDim.x)
        if (sacc[k] != 0.0) atomicAdd(&d.acc[k], sacc[k]);
    for (int k = threadIdx.x; k < nf; k += blockDim.x)
        if (sfine[k]) atomicAdd(&d.fine[k], sfine[k]);
}

// First fine bin k with count > 0 and (counts before k) + count >= target (RC/src/leverage.cpp:26-38), found by a
// block of 256 threads over contiguous chunks; returns lo + (k + (target - before) / count) width, or hi.
__device__ double block_quantile(const unsigned* fine, int nf, double lo, double hi, double q, double total,
                                 double* s_chunk, double* s_cum, int* s_best) {
    const int t = threadIdx.x, nt = blockDim.x, per = (nf + nt - 1) / nt;
    const int a = min(t * per, nf), b = min(a + per, nf);
    double mine = 0.0;
    for (int k = a; k < b; ++k) mine += static_cast<double>(fine[k]);
    s_chunk[t] = mine;
    if (t == 0) *s_best = nf;
    __syncthreads();
    double before = 0.0;
    for (int u = 0; u < t; ++u) before += s_chunk[u];  // exact: integer counts below 2^53
    const double target = q * total;
    double cum = before;
    int found = nf;
    for (int k = a; k < b; ++k) {
        const double c = static_cast<double>(fine[k]), next = cum + c;
        if (next >= target && fine[k] > 0) {
            found = k;
            break;
        }
        cum = next;
    }
    if (found < nf) atomicMin(s_best, found), s_cum[t] = cum;
    __syncthreads();
    const int kb = *s_best;
    const double cb = kb < nf ? s_cum[kb / per] : 0.0;  // counts before kb, from the thread that owns kb's chunk
    __syncthreads();
    if (kb >= nf) return hi;
    const double width = (hi - lo) / static_cast<double>(nf);
    return lo + (static_cast<double>(kb) + (target - cb) / static_cast<double>(fine[kb])) * width;
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
// and E[v | x] = v0.
__global__ void __launch_bounds__(256) lev_regress(LevDev d, int i, double n_particles) {
    __shared__ double s_chunk[256];
    __shared__ double s_cum[256];
    __shared__ double s_red[5][256];
    __shared__ int s_best;
    __shared__ double s_q[2];
    const int g = blockIdx.x, nx = d.n_x, nb = d.n_bins, t = threadIdx.x;
    const double t0 = d.t0[i], h = d.dt[i];
    double x0, cond;
    if (i == 0) {
        x0 = (-6.0 + 12.0 * g / (nx - 1)) * d.atm_vol * sqrt(h > 1e-4 ? h : 1e-4);
        cond = d.v0;
    } else {
        const double lo = unordered(d.range[0]), hi = unordered(d.range[1]);
        double total = 0.0;
        {
            // total count, the same in every thread (sum over chunks in order)
            const int per = (d.n_fine + blockDim.x - 1) / blockDim.x;
            const int a = min(t * per, d.n_fine), b = min(a + per, d.n_fine);
            double mine = 0.0;
            for (int k = a; k < b; ++k) mine += static_cast<double>(d.fine[k]);
            s_chunk[t] = mine;
            __syncthreads();
            for (int u = 0; u < static_cast<int>(blockDim.x); ++u) total += s_chunk[u];
            __syncthreads();
        }
        const double qa = block_quantile(d.fine, d.n_fine, lo, hi, d.q_lo, total, s_chunk, s_cum, &s_best);
        const double qb = block_quantile(d.fine, d.n_fine, lo, hi, d.q_hi, total, s_chunk, s_cum, &s_best);
        if (t == 0) s_q[0] = qa, s_q[1] = qb;
        __syncthreads();
        const double a = s_q[0], b = s_q[1];
        x0 = a + (b - a) * g / (nx - 1);
        const double bw = d.bw_scale * d.atm_vol * sqrt(t0 > 0.15 ? t0 : 0.15) * pow(n_particles, -0.2);
        const double wc = (hi + 1e-12 - lo) / nb;
        const double *cnt = d.acc, *sv = cnt + nb, *sx = sv + nb, *sxx = sx + nb, *sxv = sxx + nb;
        double S0 = 0, T0 = 0, Ax = 0, Axx = 0, Axv = 0;
        for (int k = t; k < nb; k += blockDim.x) {
            const double c = lo + (k + 0.5) * wc;
            const double dd = (x0 - c) / bw, w = exp(-0.5 * dd * dd);
            S0 += w * cnt[k], T0 += w * sv[k];
            if (d.local_linear) Ax += w * sx[k], Axx += w * sxx[k], Axv += w * sxv[k];
        }
        s_red[0][t] = S0, s_red[1][t] = T0, s_red[2][t] = Ax, s_red[3][t] = Axx, s_red[4][t] = Axv;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (t < s)
                for (int r = 0; r < 5; ++r) s_red[r][t] += s_red[r][t + s];
            __syncthreads();
        }
        S0 = s_red[0][0], T0 = s_red[1][0], Ax = s_red[2][0], Axx = s_red[3][0], Axv = s_red[4][0];
        const double fallback = d.acc[5 * nb] / n_particles;
        const double nw = S0 > 1e-8 ? T0 / (S0 > 1e-300 ? S0 : 1e-300) : fallback;
        cond = nw;
        if (d.local_linear) {
            const double S1 = Ax - x0 * S0, S2 = Axx - 2 * x0 * Ax + x0 * x0 * S0, T1 = Axv - x0 * T0;
            const double det = S0 * S2 - S1 * S1;
            const bool ok = S0 >= 50 && det > 1e-12 * S0 * fabs(S2);
            const double ll = ok ? (S2 * T0 - S1 * T1) / det : nw;
            cond = ll > 1e-8 ? ll : 1e-8;
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
}

template <typename R>
__global__ void __launch_bounds__(256) lev_step(LevDev d, R* __restrict__ x, R* __restrict__ v, int i) {
    __shared__ R s_lev[kMaxX];
    __shared__ R s_min[8], s_max[8];
    for (int g = threadIdx.x; g < d.n_x; g += blockDim.x) s_lev[g] = static_cast<R>(d.lev[g]);
    __syncthreads();
    const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int nx = d.n_x;
    const R h = static_cast<R>(d.dt[i]);
    const R a = static_cast<R>(d.x_eval[0]), b = static_cast<R>(d.x_eval[nx - 1]);
    const R rho = static_cast<R>(d.rho), kappa = static_cast<R>(d.kappa), theta = static_cast<R>(d.theta);
    const R xi = static_cast<R>(d.xi);
    R mn = sizeof(R) == 4 ? R(3.0e38f) : R(1.0e300), mx = -mn;
    if (p < d.n_pairs) {
        R z0, z1, z2, z3;
        normals4<R>(static_cast<uint64_t>(p), static_cast<uint64_t>(i + 1), 0u, d.k0, d.k1, z0, z1, z2, z3);
        const R rc = m_sqrt(R(1) - rho * rho);
#pragma unroll
        for (int leg = 0; leg < 2; ++leg) {
            const long long j = leg ? d.n_pairs + p : p;
            const R sg = leg ? R(-1) : R(1), zz1 = sg * z0, zz2 = sg * z1;
            const R xj = x[j];
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
            const R vp = m_max(v[j], R(0)), var = L * L * vp;
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
        atomicMin(reinterpret_cast<long long*>(&d.range[0]), ordered(static_cast<double>(mn)));
        atomicMax(reinterpret_cast<long long*>(&d.range[1]), ordered(static_cast<double>(mx)));
    }
}

__global__ void lev_range_reset(long long* range) {
    range[0] = 0x7FFFFFFFFFFFFFFFLL;
    range[1] = static_cast<long long>(0x8000000000000000ULL);
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
    d.fine = arena.alloc<unsigned>(rq.n_fine);
    d.acc = arena.alloc<double>(5 * static_cast<size_t>(rq.n_bins) + 1);
    d.range = arena.alloc<long long>(2);
    d.x_eval = arena.alloc<double>(rq.n_x);
    d.lev = arena.alloc<double>(rq.n_x);
    d.x_grids = arena.alloc<double>(static_cast<size_t>(S) * rq.n_x);
    d.values = arena.alloc<double>(static_cast<size_t>(S) * rq.n_x);
    R* x = arena.alloc<R>(n);
    R* v = arena.alloc<R>(n);
    const size_t bin_smem = (5 * static_cast<size_t>(rq.n_bins) + 1) * sizeof(double) + rq.n_fine * sizeof(unsigned);
    check_cuda(cudaFuncSetAttribute(lev_bin<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(bin_smem)),
               "cudaFuncSetAttribute");
    int per_sm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lev_bin<R>, 512, bin_smem), "occupancy");
    const int bin_grid = static_cast<int>(std::max<long long>(
        1, std::min<long long>(static_cast<long long>(sms) * std::max(1, per_sm), (n + 511) / 512)));
    const unsigned step_grid = static_cast<unsigned>((rq.n_pairs + 255) / 256);
    const double n_particles = 2.0 * static_cast<double>(rq.n_pairs);
    lev_init<R><<<static_cast<unsigned>((n + 255) / 256), 256>>>(x, v, n, static_cast<R>(rq.v0), d.range);
    check_cuda(cudaGetLastError(), "lev_init launch");
    for (int i = 0; i < S; ++i) {
        if (i > 0) {
            lev_reset<<<1, 1024>>>(d);
            lev_bin<R><<<bin_grid, 512, bin_smem>>>(d, x, v);
        }
        lev_regress<<<rq.n_x, 256>>>(d, i, n_particles);
        lev_range_reset<<<1, 1>>>(d.range);
        lev_step<R><<<step_grid, 256>>>(d, x, v, i);
    }
    check_cuda(cudaGetLastError(), "leverage launches");
    check_cuda(cudaMemcpy(rq.x_grids, d.x_grids, static_cast<size_t>(S) * rq.n_x * sizeof(double),
                          cudaMemcpyDeviceToHost),
               "copy x_grids");
    check_cuda(cudaMemcpy(rq.values, d.values, static_cast<size_t>(S) * rq.n_x * sizeof(double),
                          cudaMemcpyDeviceToHost),
               "copy values");
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
