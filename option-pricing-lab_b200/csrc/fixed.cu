// ob_price: the drop-in for optlab::api::price(rq, 1, 0) (RC/include/optlab_cuda/requests.hpp:103-104), the fixed
// products of the reference's study: Black-Scholes or Heston (Andersen QE-M) on a flat market; European (three legs),
// Asian (arithmetic and geometric on leg 0) or down-and-out barrier (leg 0, knocked out when S <= H at a step end);
// output 3 = E[S_T]. Semantics of RC/include/optlab_cuda/schemes.hpp:188-245 (bs_european_unit, path_unit), with the
// engine's Philox normals in place of cuRAND: unit (antithetic pair) p reads stream 0 of pair p, one normal per step
// under Black-Scholes, (zv, zx) per step under Heston. Sums of the pair averages in FP64, per warp then per block.
#include <chrono>
#include <cmath>

#include "model.cuh"

namespace ob {

namespace {

struct FixedDev {
    int model, product, n_steps;
    int leg[3];
    double K[3];
    double S0, D, bs_drift, bs_vol, ln_h, inv_n;
};

template <typename R>
__device__ __forceinline__ R leg_payoff(int leg, R S, R K) {
    return leg == 1 ? m_max(S - K, R(0)) : leg == 2 ? m_max(K - S, R(0)) : leg == 3 ? S - K : R(0);
}

template <typename R>
__global__ void __launch_bounds__(256) fixed_kernel(FixedDev f, QeConsts<R> qe, long long n_units, uint32_t k0,
                                                    uint32_t k1, double* __restrict__ partial) {
    __shared__ double wacc[8][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < 64) wacc[threadIdx.x >> 3][threadIdx.x & 7] = 0.0;
    __syncthreads();
    const R S0 = static_cast<R>(f.S0), bs_drift = static_cast<R>(f.bs_drift), bs_vol = static_cast<R>(f.bs_vol);
    const R ln_h = static_cast<R>(f.ln_h), inv_n = static_cast<R>(f.inv_n), D = static_cast<R>(f.D);
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < n_units;
         base += stride) {
        const bool active = base + lane < n_units;
        const long long p = active ? base + lane : n_units - 1;
        NormalStream<R> rng;
        rng.init(static_cast<uint64_t>(p), k0, k1, 0u);
        R y[2] = {R(0), R(0)}, v[2] = {qe.v0, qe.v0}, ss[2] = {R(0), R(0)}, sy[2] = {R(0), R(0)};
        bool alive[2] = {true, true};
        const int steps = (f.product == 0 && f.model == 0) ? 1 : f.n_steps;
        for (int i = 0; i < steps; ++i) {
            R zv = R(0);
            if (f.model == 1) zv = rng.next();
            const R zx = rng.next();
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const R sg = a ? R(-1) : R(1);
                if (f.model == 1) qe_step(qe, y[a], v[a], sg * zv, sg * zx);
                else if (f.product == 0) y[a] = bs_drift + bs_vol * sg * zx;
                else y[a] += bs_drift + bs_vol * sg * zx;
                if (f.product == 1) ss[a] += m_exp(y[a]), sy[a] += y[a];
                if (f.product == 2) alive[a] = alive[a] && !(y[a] <= ln_h);
            }
        }
        R o[4] = {R(0), R(0), R(0), R(0)};
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const R S = S0 * m_exp(y[a]);
            if (f.product == 0) {
#pragma unroll
                for (int k = 0; k < 3; ++k) o[k] += D * leg_payoff(f.leg[k], S, static_cast<R>(f.K[k]));
            } else if (f.product == 1) {
                o[0] += D * leg_payoff(f.leg[0], S0 * ss[a] * inv_n, static_cast<R>(f.K[0]));
                o[1] += D * leg_payoff(f.leg[0], S0 * m_exp(sy[a] * inv_n), static_cast<R>(f.K[0]));
            } else {
                const R pay = D * leg_payoff(f.leg[0], S, static_cast<R>(f.K[0]));
                o[0] += alive[a] ? pay : R(0);
                o[1] += pay;
            }
            o[3] += S;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double yk = active ? 0.5 * static_cast<double>(o[k]) : 0.0;
            const double s1 = warp_sum(yk), s2 = warp_sum(yk * yk);
            if (lane == 0) wacc[warp][k] += s1, wacc[warp][4 + k] += s2;
        }
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += wacc[w][threadIdx.x];
        partial[static_cast<long long>(blockIdx.x) * 8 + threadIdx.x] = s;
    }
}

__global__ void fixed_finalize(const double* __restrict__ partial, int n_blocks, double* sums) {
    const int t = threadIdx.x;
    if (t >= 8) return;
    double s = 0.0;
    for (int b = 0; b < n_blocks; ++b) s += partial[static_cast<long long>(b) * 8 + t];
    sums[t] = s;
}

// Blocks of one launch over n_units pairs: enough for every pair, at most the resident blocks of the device.
template <typename R>
long long fixed_grid(long long n_units, int sms) {
    const int per_sm = occupancy(reinterpret_cast<const void*>(fixed_kernel<R>), 256, 0);
    return std::max<long long>(1, std::min<long long>((n_units + 255) / 256,
                                                      static_cast<long long>(sms) * std::max(1, per_sm)));
}

// RC/src/requests.cpp:140-165 (convert): the same checks and messages.
void check_request(const ob_request& c) {
    if (c.model < 0 || c.model > 1) invalid("model must be 0 (Black-Scholes) or 1 (Heston)");
    if (c.product < 0 || c.product > 2) invalid("product must be 0, 1 or 2");
    if (c.n_steps < 1) invalid("n_steps must be >= 1");
    if (c.n_paths < 4 || c.n_paths % 2) invalid("n_paths must be even and >= 4");
    if (!(c.S0 > 0 && c.T > 0)) invalid("S0 and T must be positive");
    if (c.model == 0 && !(c.sigma > 0)) invalid("sigma must be positive");
    if (c.model == 1 && !(c.v0 >= 0 && c.kappa > 0 && c.theta > 0 && c.xi > 0 && std::fabs(c.rho) <= 1))
        invalid("Heston parameters out of range");
    if (c.product == 2 && !(c.H > 0 && c.H < c.S0)) invalid("barrier: need 0 < H < S0");
    for (int k = 0; k < 3; ++k)
        if (c.legs[k] < 0 || c.legs[k] > 3) invalid("legs must be 0 to 3");
}

// One priced request on the current device: the kernel over the pairs, its block partial sums in `partial` (room for
// `max_blocks` blocks), the totals in `sums`; kernel_ms from events around the two launches, total_ms from the host
// clock since t_start. Both entry points below call it: ob_price with buffers from the call's arena, ob_price_noalloc
// with the library's fixed array.
template <typename R>
void price_fixed(const ob_request& rq, ob_result& res, std::chrono::steady_clock::time_point t_start, int sms,
                 double* partial, long long max_blocks, double* sums) {
    FixedDev f{};
    f.model = rq.model, f.product = rq.product, f.n_steps = rq.n_steps;
    for (int k = 0; k < 3; ++k) f.leg[k] = rq.legs[k], f.K[k] = rq.strikes[k];
    const double dt = rq.T / rq.n_steps;
    f.S0 = rq.S0, f.D = std::exp(-rq.r * rq.T);
    f.bs_drift = (rq.r - rq.q - 0.5 * rq.sigma * rq.sigma) * dt;
    f.bs_vol = rq.sigma * std::sqrt(dt);
    f.ln_h = rq.product == 2 ? std::log(rq.H / rq.S0) : 0.0;
    f.inv_n = 1.0 / rq.n_steps;
    const double h[5] = {rq.v0, rq.kappa, rq.theta, rq.xi, rq.rho};
    QeConsts<R> qe{};
    if (rq.model == 1) qe = make_qe_consts<R>(h, rq.r, rq.q, dt);
    const long long n_units = rq.n_paths / 2;
    const long long grid = fixed_grid<R>(n_units, sms);
    if (grid > max_blocks) invalid("the launch needs more blocks than the no-allocation scratch holds (4096)");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    const cudaError_t ee = cudaEventCreate(&e1);
    if (ee != cudaSuccess) cudaEventDestroy(e0);
    check_cuda(ee, "cudaEventCreate");
    cudaEventRecord(e0);
    fixed_kernel<R><<<static_cast<unsigned>(grid), 256>>>(f, qe, n_units, static_cast<uint32_t>(rq.seed),
                                                          static_cast<uint32_t>(rq.seed >> 32), partial);
    const cudaError_t le = cudaGetLastError();
    if (le == cudaSuccess) fixed_finalize<<<1, 32>>>(partial, static_cast<int>(grid), sums);
    const cudaError_t le2 = cudaGetLastError();
    cudaEventRecord(e1);
    double hs[8];
    const cudaError_t ce = cudaMemcpy(hs, sums, sizeof hs, cudaMemcpyDeviceToHost);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0), cudaEventDestroy(e1);
    check_cuda(le, "fixed_kernel launch");
    check_cuda(le2, "fixed_finalize launch");
    check_cuda(ce, "fixed_kernel");
    std::memset(&res, 0, sizeof res);
    const double n = static_cast<double>(n_units);
    for (int k = 0; k < 4; ++k) {
        const double mean = hs[k] / n, var = hs[4 + k] / n - mean * mean;  // RC/src/cpu_mc.cpp:8-12
        res.price[k] = mean, res.se[k] = n_units > 1 ? std::sqrt(std::fmax(var, 0.0) / (n - 1.0)) : 0.0;
    }
    res.n_paths = rq.n_paths;
    res.kernel_ms = ms;
    res.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
}

template <typename R>
void run_fixed(const ob_request& rq, ob_result& res) {
    const auto t_start = std::chrono::steady_clock::now();
    const int sms = require_device();
    const long long grid = fixed_grid<R>(rq.n_paths / 2, sms);
    DeviceArena arena;
    arena.recycle = true;  // the blocking copy of the sums ends the call's device work
    double* partial = arena.alloc<double>(static_cast<size_t>(grid) * 8);
    double* sums = arena.alloc<double>(8);
    price_fixed<R>(rq, res, t_start, sms, partial, grid, sums);
}

}  // namespace
}  // namespace ob

extern "C" int ob_price(const ob_request* rq, ob_result* res, int precision) {
    return ob::guarded([&] {
        if (!rq || !res) ob::invalid("null argument");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        ob::check_request(*rq);
        if (precision == OB_FP32) ob::run_fixed<float>(*rq, *res);
        else ob::run_fixed<double>(*rq, *res);
    });
}

// ------------------------------------------------------------------------------------------------ no allocation
//
// ob_price_noalloc: ob_price for callers that must not allocate device memory while they price. Some risk services
// hand all device memory to one allocator at start-up (a framework's caching pool, a fixed budget per desk) and
// cannot have a library take more behind its back; others run quote loops where cudaMalloc and cudaFree are not
// allowed, because they take the driver's allocation lock and cudaFree waits for the whole device. This entry point
// runs the same kernel as ob_price, with its per-block partial sums and final sums in a fixed array that is part of
// the library image: g_noalloc_scratch, 4096 blocks x 8 sums + 8 totals (about 256 KiB), held on every device that
// loads the library until the process exits. A launch needing more blocks than that is refused.
//
// Set-up: every call, with the caller's device current, asks the driver for the array's device address in that
// device's context (cudaGetSymbolAddress; it allocates nothing). On a device's first call this also loads the
// library's device code into the context, so make the first call on each device before any stream capture. Every
// call uses the same array, and each call overwrites in full the slots it reads (every block writes its partial sums,
// the last kernel writes the totals), so nothing carries over from one call to the next. Calls that overlap on the
// GPU would race for the array: within one process the library's lock and the call's blocking read-back keep calls
// apart; two processes share no array (each has its own context), but work that the caller queues on other streams
// must not touch it. The timing events are driver objects, not device memory.
namespace ob {
namespace {

constexpr int kNoAllocMaxBlocks = 4096;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxBlocks * 8 + 8];

// The array's device address in the current device's context, asked of the driver on every call: the lookup is
// cheap and allocates nothing, and a context created again (after cudaDeviceReset, say) may hold the array at
// another address, so an address kept from an earlier call could point at memory that is no longer the array.
double* noalloc_scratch() {
    void* p = nullptr;
    check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    return static_cast<double*>(p);
}

template <typename R>
void run_fixed_noalloc(const ob_request& rq, ob_result& res) {
    const auto t_start = std::chrono::steady_clock::now();
    const int sms = require_device();
    double* partial = noalloc_scratch();
    double* sums = partial + static_cast<size_t>(kNoAllocMaxBlocks) * 8;
    price_fixed<R>(rq, res, t_start, sms, partial, kNoAllocMaxBlocks, sums);
}

}  // namespace
}  // namespace ob

extern "C" int ob_price_noalloc(const ob_request* rq, ob_result* res, int precision) {
    return ob::guarded([&] {
        if (!rq || !res) ob::invalid("null argument");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        ob::check_request(*rq);
        if (precision == OB_FP32) ob::run_fixed_noalloc<float>(*rq, *res);
        else ob::run_fixed_noalloc<double>(*rq, *res);
    });
}
