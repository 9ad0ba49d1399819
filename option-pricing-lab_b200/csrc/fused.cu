// The specialised fused kernel (fused.cuh): path, payoff and FP64 sums for baskets whose names share one kind.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <type_traits>
#include <vector>

#include "mc.cuh"

namespace ob {

namespace {

constexpr int gcd4(int c) { return c % 4 == 0 ? 4 : c % 2 == 0 ? 2 : 1; }

// Product bookkeeping of one leg, kept small: the ladder's extremes or the autocall's state.
template <typename R>
struct Leg {
    R hi, lo;       // ladder: extremes of ln perf; autocall: lo is the lowest ln perf
    double pv;      // autocall: discounted cash flows
    float coupons;  // autocall: coupons paid
    int flags;      // autocall: missed coupons (bits 0-15), alive (16), called (17), knocked (18)
};

constexpr int kAlive = 1 << 16, kCalled = 1 << 17, kKnocked = 1 << 18;

template <typename R, int PRODUCT>
__device__ __forceinline__ void leg_init(Leg<R>& l) {
    l.hi = R(-1e30), l.lo = PRODUCT == OB_PRODUCT_LADDER ? R(1e30) : R(0);
    l.pv = 0.0, l.coupons = 0.0f, l.flags = kAlive;
}

// Observation j of one leg (autocall): coupon with memory, then the call, or the redemption on the last date
// (packages/structured/src/optlab/structured/compiler.py:114-127,141-161,271-280).
template <typename R>
__device__ __forceinline__ void leg_observe(const FusedArgs<R>& a, const R* ln_trig, const double* disc, Leg<R>& l,
                                            R lp, int j) {
    if (!(l.flags & kAlive)) return;
    const double D = disc[j];
    if (a.has_coupon) {
        if (lp >= a.ln_cb) {
            const int k = a.memory ? 1 + (l.flags & 0xFFFF) : 1;
            l.pv += D * a.coupon * k, l.coupons += static_cast<float>(k), l.flags &= ~0xFFFF;
        } else {
            l.flags += 1;
        }
    }
    if (j < a.n_obs - 1) {
        if (lp >= ln_trig[j]) l.pv += D, l.flags = (l.flags & ~kAlive) | kCalled;
    } else {
        const bool ki = a.ki_daily ? l.lo < a.ln_ki : lp < a.ln_ki;
        const double perf = static_cast<double>(m_exp(lp));
        const double put = a.put_strike - perf > 0.0 ? a.put_strike - perf : 0.0;
        l.pv += D * (ki ? 1.0 - put : 1.0);
        l.flags = (l.flags & ~kAlive) | (ki ? kKnocked : 0);
    }
}

template <typename R, int PRODUCT>
__device__ __forceinline__ double leg_output(const FusedArgs<R>& a, const int* leg_type, const R* leg_strike,
                                             const int* leg_barrier, const R* ln_level, const Leg<R>& l, R lp_T,
                                             int k) {
    if (PRODUCT == OB_PRODUCT_AUTOCALL) {
        return k == 0 ? l.pv : k == 1 ? ((l.flags & kCalled) ? 1.0 : 0.0)
                                      : k == 2 ? ((l.flags & kKnocked) ? 1.0 : 0.0) : static_cast<double>(l.coupons);
    }
    const R U = a.spot0 * m_exp(lp_T);
    if (k == a.n_legs) return static_cast<double>(U);
    const int type = leg_type[k];
    const R K = leg_strike[k];
    R pay = type == 1 ? m_max(U - K, R(0)) : type == 2 ? m_max(K - U, R(0)) : type == 3 ? U - K : R(0);
    const int bt = leg_barrier[k];
    const R H = ln_level[k];
    const bool up = l.hi >= H, down = l.lo <= H;
    if ((bt == OB_BARRIER_UP_OUT && up) || (bt == OB_BARRIER_DOWN_OUT && down) || (bt == OB_BARRIER_UP_IN && !up) ||
        (bt == OB_BARRIER_DOWN_IN && !down))
        pay = R(0);
    return a.discount * static_cast<double>(pay);
}

template <typename R>
constexpr int min_blocks() {
    return sizeof(R) == 4 ? 2 : 1;
}

// KIND: 1 local vol (table), 2 Heston (Euler), 3 SLV (table x Heston, residuals on the aux stream), 4 Heston QE-M.
// GT: the table is read from global memory (a.tab) instead of the stage.
// Blocks of 512 an SM the register budget allows: two in float (64 registers), one in double; one for the mixer's
// 4- and 5-name baskets in float too, whose two legs' normals would spill at 64.
template <typename R, int N, bool MIX>
constexpr int fused_min_blocks() {
    return MIX && N >= 4 ? 1 : min_blocks<R>();
}

// MIX (local vol, 2 to 5 names): the local-correlation mixer, one more normal a step after the names'.
template <typename R, int N, int KIND, int PRODUCT, bool GT = false, bool MIX = false>
__global__ void __launch_bounds__(512, (fused_min_blocks<R, N, MIX>()))
    fused_kernel(FusedArgs<R> a, long long n_pairs, long long first_pair, uint32_t k0, uint32_t k1,
                 double* __restrict__ partial) {
    constexpr bool QE = KIND == 4;
    constexpr bool VAR = KIND == 2 || KIND == 3;
    constexpr bool TABLE = KIND == 1 || KIND == 3;
    static_assert(!MIX || (KIND == 1 && N >= 2), "the mixer runs local-vol baskets");
    constexpr int C = QE ? 2 : (KIND == 2 ? 2 * N : N + (MIX ? 1 : 0));  // normals per step, stream 0
    constexpr int CA = KIND == 3 ? N : 0;                // normals per step, aux stream
    // steps per batch of whole Philox blocks; one local-vol name draws two blocks a batch (8 steps), whose two
    // independent multiply chains interleave (1.317 -> 1.300 ms for the 2^20-path Phoenix; one SLV name would draw four
    // and spill in FP64)
    constexpr int G = C == 1 && KIND == 1 ? 8 : 4 / gcd4(C);
    constexpr int NB = C * G / 4, NBA = CA * G / 4;

    extern __shared__ __align__(16) unsigned char sm[];
    {
        const int4* src = reinterpret_cast<const int4*>(a.blob);
        int4* dst = reinterpret_cast<int4*>(sm);
        for (int t = threadIdx.x; t < a.smem_blob / 16; t += blockDim.x) dst[t] = src[t];
    }
    const int n_warps = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n_acc = 2 * a.n_out;
    double* wacc = reinterpret_cast<double*>(sm + a.smem_blob);
    for (int t = threadIdx.x; t < n_warps * n_acc; t += blockDim.x) wacc[t] = 0.0;
    __syncthreads();
    const StepRec<R>* s_step = reinterpret_cast<const StepRec<R>*>(sm + a.off.step);
    const NameStep<R>* s_ns = reinterpret_cast<const NameStep<R>*>(sm + a.off.name_step);
    const R* s_root = reinterpret_cast<const R*>(sm + a.off.root);
    const R* s_hes = reinterpret_cast<const R*>(sm + a.off.hes);
    const Pair2<R>* s_tab = GT ? a.tab : reinterpret_cast<const Pair2<R>*>(sm + a.off.table2);
    const R* s_trig = reinterpret_cast<const R*>(sm + a.off.ln_trig);
    const double* s_disc = reinterpret_cast<const double*>(sm + a.off.obs_disc);
    const int S = a.n_steps;
    // the correlation root: in registers for one or two names, read from shared memory for more (registers spill)
    constexpr bool kRootRegs = N <= 2;
    R rt[kRootRegs ? N * N : 1];
#pragma unroll
    for (int k = 0; k < (kRootRegs ? N * N : 0); ++k) rt[k] = s_root[k];

    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < n_pairs;
         base += stride) {
        const bool active = base + lane < n_pairs;
        const uint64_t pair = static_cast<uint64_t>(first_pair + (active ? base + lane : n_pairs - 1));
        R x0[N], x1[N], v0[N], v1[N];
#pragma unroll
        for (int n = 0; n < N; ++n) {
            x0[n] = x1[n] = R(0);
            v0[n] = v1[n] = QE ? a.qe.v0 : (VAR ? s_hes[8 * n] : R(0));
        }
        Leg<R> l0, l1;
        leg_init<R, PRODUCT>(l0), leg_init<R, PRODUCT>(l1);
        R lp0 = R(0), lp1 = R(0);
        // One batch of G steps from step i0, its normals drawn first. For one local-vol name the full batches run
        // without testing for the last step and only the tail batch (CHECK) may stop inside, and an autocall's batches
        // without an observation run without testing each step for one (OBS false).
        auto run_batch = [&](int i0, int batch, auto check, auto observe) {
            constexpr bool CHECK = decltype(check)::value, OBS = decltype(observe)::value;
            R z[C * G];
            R za[CA > 0 ? CA * G : 1];
#pragma unroll
            for (int k = 0; k < NB; ++k)
                normals4<R>(pair, static_cast<uint64_t>(batch) * NB + k, 0u, k0, k1, z[4 * k], z[4 * k + 1],
                            z[4 * k + 2], z[4 * k + 3]);
#pragma unroll
            for (int k = 0; k < NBA; ++k)
                normals4<R>(pair, static_cast<uint64_t>(batch) * NBA + k, kAuxStream, k0, k1, za[4 * k],
                            za[4 * k + 1], za[4 * k + 2], za[4 * k + 3]);
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int i = i0 + g;
                if constexpr (CHECK && G > 1) {
                    if (i > S) break;
                }
                if (QE) {
                    const R zv = z[2 * g], zx = z[2 * g + 1];
                    qe_step(a.qe, x0[0], v0[0], zv, zx);
                    qe_step(a.qe, x1[0], v1[0], -zv, -zx);
                    lp0 = x0[0], lp1 = x1[0];
                } else {
                    const StepRec<R> st = s_step[i - 1];
                    const R* zs = &z[g * C];
                    R zc[N], wc[N];
                    R zm0[MIX ? N : 1], zm1[MIX ? N : 1];  // with the mixer each leg's own normals (signs in)
                    if (MIX) {
                        // paths.hpp:219-237: a common factor whose weight moves with the level of the basket (the
                        // log of the mean of S / F at the step's start), per leg
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
#pragma unroll
                    for (int n = 0; n < N; ++n) {
                        R acc = R(0);
                        if (!MIX) {
#pragma unroll
                            for (int b = 0; b < N; ++b)
                                acc += (kRootRegs ? rt[n * N + b] : s_root[n * N + b]) * zs[b];
                        }
                        zc[n] = acc;
                    }
                    if (VAR) {
                        const R* zr = KIND == 3 ? &za[g * CA] : &z[g * C + N];
#pragma unroll
                        for (int n = 0; n < N; ++n) {
                            if (a.same) {
                                R acc = R(0);
#pragma unroll
                                for (int b = 0; b < N; ++b) acc += (kRootRegs ? rt[n * N + b] : s_root[n * N + b]) * zr[b];
                                wc[n] = acc;
                            } else {
                                wc[n] = zr[n];
                            }
                        }
                    }
                    R w0 = R(0), w1 = R(0);  // the worst log performance: the first name's, then the minimum
#pragma unroll
                    for (int n = 0; n < N; ++n) {
                        const NameStep<R> ns = s_ns[(i - 1) * N + n];
                        R var0, var1, vp0 = R(0), vp1 = R(0);
                        if (VAR) vp0 = m_max(v0[n], R(0)), vp1 = m_max(v1[n], R(0));
                        if (TABLE) {
                            int j0, j1;
                            R f0, f1;
                            table_cell(ns, a.top, x0[n], j0, f0), table_cell(ns, a.top, x1[n], j1, f1);
                            const Pair2<R> y0 = GT ? ldg_pair(s_tab + ns.row + j0) : s_tab[ns.row + j0];
                            const Pair2<R> y1 = GT ? ldg_pair(s_tab + ns.row + j1) : s_tab[ns.row + j1];
                            const R t0 = y0.a + f0 * y0.b, t1 = y1.a + f1 * y1.b;
                            var0 = KIND == 1 ? t0 : t0 * vp0, var1 = KIND == 1 ? t1 : t1 * vp1;
                        } else if (VAR) {
                            var0 = vp0, var1 = vp1;
                        } else {
                            var0 = var1 = s_hes[8 * n + 6];  // Black-Scholes: the name's constant variance
                        }
                        if (VAR) {
                            const R* h = s_hes + 8 * n;  // v0, kappa, theta, xi, rho, sqrt(1 - rho^2)
                            const R zv = h[4] * zc[n] + h[5] * wc[n];
                            v0[n] += h[1] * (h[2] - vp0) * st.dt + h[3] * (m_sqrt(vp0) * st.sdt) * zv;
                            v1[n] += h[1] * (h[2] - vp1) * st.dt + h[3] * (m_sqrt(vp1) * st.sdt) * (-zv);
                        }
                        if (MIX) {
                            x0[n] = lv_advance(x0[n], var0, st.hdt, st.sdt * zm0[n]);
                            x1[n] = lv_advance(x1[n], var1, st.hdt, st.sdt * zm1[n]);
                        } else {
                            const R zd = st.sdt * zc[n];  // sqrt(dt) z, the legs' +-
                            x0[n] = lv_advance(x0[n], var0, st.hdt, zd);
                            x1[n] = lv_advance(x1[n], var1, st.hdt, -zd);
                        }
                        if (n == 0) w0 = x0[n] + ns.lf, w1 = x1[n] + ns.lf;
                        else w0 = m_min(w0, x0[n] + ns.lf), w1 = m_min(w1, x1[n] + ns.lf);
                    }
                    lp0 = w0, lp1 = w1;
                }
                if (PRODUCT == OB_PRODUCT_LADDER) {
                    l0.hi = m_max(l0.hi, lp0), l0.lo = m_min(l0.lo, lp0);
                    l1.hi = m_max(l1.hi, lp1), l1.lo = m_min(l1.lo, lp1);
                } else {
                    l0.lo = m_min(l0.lo, lp0), l1.lo = m_min(l1.lo, lp1);
                    const int j = OBS ? s_step[i - 1].obs : -1;
                    if (j >= 0) {
                        leg_observe(a, s_trig, s_disc, l0, lp0, j);
                        leg_observe(a, s_trig, s_disc, l1, lp1, j);
                    }
                }
            }
        };
        if constexpr (N == 1 && KIND == 1) {  // (a second copy of the loop costs the wider kernels registers)
            // a step without an observation holds minus the steps to the next one: none in steps i0 .. i0 + G - 1
            // when step i0's entry is at most -G
            constexpr bool kSplitObs = PRODUCT == OB_PRODUCT_AUTOCALL;
            const int n_full = S / G;
            int i0 = 1, batch = 0;
            for (; batch < n_full; i0 += G, ++batch) {
                if (!kSplitObs || s_step[i0 - 1].obs <= -G)
                    run_batch(i0, batch, std::false_type{}, std::false_type{});
                else
                    run_batch(i0, batch, std::false_type{}, std::true_type{});
            }
            if (i0 <= S) run_batch(i0, batch, std::true_type{}, std::true_type{});
        } else {
            for (int i0 = 1, batch = 0; i0 <= S; i0 += G, ++batch)
                run_batch(i0, batch, std::true_type{}, std::true_type{});
        }
        const int* leg_type = reinterpret_cast<const int*>(sm + a.off.leg_type);
        const R* leg_strike = reinterpret_cast<const R*>(sm + a.off.leg_strike);
        const int* leg_barrier = reinterpret_cast<const int*>(sm + a.off.leg_barrier);
        const R* ln_level = reinterpret_cast<const R*>(sm + a.off.ln_level);
        for (int k = 0; k < a.n_out; ++k) {
            const double y =
                active ? 0.5 * (leg_output<R, PRODUCT>(a, leg_type, leg_strike, leg_barrier, ln_level, l0, lp0, k) +
                                leg_output<R, PRODUCT>(a, leg_type, leg_strike, leg_barrier, ln_level, l1, lp1, k))
                       : 0.0;
            const double s1 = warp_sum(y), s2 = warp_sum(y * y);
            if (lane == 0) wacc[warp * n_acc + k] += s1, wacc[warp * n_acc + a.n_out + k] += s2;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n_acc; t += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < n_warps; ++w) s += wacc[w * n_acc + t];
        partial[static_cast<long long>(blockIdx.x) * n_acc + t] = s;
    }
}

// Heston QE-M with the two legs of an antithetic pair on neighbouring lanes (lane 2k: +z, lane 2k+1: -z): twice the
// threads of fused_kernel for the same pairs, for the small path counts of QE books (2^15 pairs are 7 warps an SM at
// one pair a thread; the FP64 step is a long dependent chain and needs the warps to hide its latency). Philox block b
// of a pair holds (zv, zx) of steps 2b + 1 and 2b + 2; the two lanes draw alternate blocks (lane 2k block 2m, lane
// 2k + 1 block 2m + 1) and swap them, so each lane draws half the normals and steps one leg. The pair's value is
// the average of the lanes' payoffs, added once (by the even lane).
template <typename R, int PRODUCT>
__global__ void __launch_bounds__(512, min_blocks<R>())
    qe_pair_kernel(FusedArgs<R> a, long long n_pairs, long long first_pair, uint32_t k0, uint32_t k1,
                   double* __restrict__ partial) {
    extern __shared__ __align__(16) unsigned char sm[];
    {
        const int4* src = reinterpret_cast<const int4*>(a.blob);
        int4* dst = reinterpret_cast<int4*>(sm);
        for (int t = threadIdx.x; t < a.smem_blob / 16; t += blockDim.x) dst[t] = src[t];
    }
    const int n_warps = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n_acc = 2 * a.n_out;
    double* wacc = reinterpret_cast<double*>(sm + a.smem_blob);
    for (int t = threadIdx.x; t < n_warps * n_acc; t += blockDim.x) wacc[t] = 0.0;
    __syncthreads();
    const StepRec<R>* s_step = reinterpret_cast<const StepRec<R>*>(sm + a.off.step);
    const R* s_trig = reinterpret_cast<const R*>(sm + a.off.ln_trig);
    const double* s_disc = reinterpret_cast<const double*>(sm + a.off.obs_disc);
    const int* leg_type = reinterpret_cast<const int*>(sm + a.off.leg_type);
    const R* leg_strike = reinterpret_cast<const R*>(sm + a.off.leg_strike);
    const int* leg_barrier = reinterpret_cast<const int*>(sm + a.off.leg_barrier);
    const R* ln_level = reinterpret_cast<const R*>(sm + a.off.ln_level);
    const int S = a.n_steps;
    const int odd = lane & 1;
    const R sgn = odd ? R(-1) : R(1);
    constexpr unsigned kFull = 0xffffffffu;

    const long long stride = (static_cast<long long>(gridDim.x) * blockDim.x) >> 1;
    for (long long base = (static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31)) >> 1;
         base < n_pairs; base += stride) {
        const long long p = base + (lane >> 1);
        const bool active = p < n_pairs;
        const uint64_t pair = static_cast<uint64_t>(first_pair + (active ? p : n_pairs - 1));
        R x = R(0), v = a.qe.v0, lp = R(0);
        Leg<R> l;
        leg_init<R, PRODUCT>(l);
        for (int i0 = 1, m = 0; i0 <= S; i0 += 4, ++m) {
            R z[4], e[8];
            normals4<R>(pair, static_cast<uint64_t>(2 * m + odd), 0u, k0, k1, z[0], z[1], z[2], z[3]);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const R o = __shfl_xor_sync(kFull, z[k], 1);
                e[k] = odd ? o : z[k];      // block 2m: steps i0, i0 + 1
                e[4 + k] = odd ? z[k] : o;  // block 2m + 1: steps i0 + 2, i0 + 3
            }
            // one copy of the (long, FP64) step in the loop body: the four steps rotate the normals through e[0..1]
#pragma unroll 1
            for (int g = 0; g < 4; ++g) {
                const int i = i0 + g;
                if (i > S) break;
                qe_step_warp(a.qe, x, v, sgn * e[0], sgn * e[1]);  // (all 32 lanes step together)
                e[0] = e[2], e[1] = e[3], e[2] = e[4], e[3] = e[5], e[4] = e[6], e[5] = e[7];
                lp = x;
                if (PRODUCT == OB_PRODUCT_LADDER) {
                    l.hi = m_max(l.hi, lp), l.lo = m_min(l.lo, lp);
                } else {
                    l.lo = m_min(l.lo, lp);
                    const int j = s_step[i - 1].obs;
                    if (j >= 0) leg_observe(a, s_trig, s_disc, l, lp, j);
                }
            }
        }
        for (int k = 0; k < a.n_out; ++k) {
            const double mine = leg_output<R, PRODUCT>(a, leg_type, leg_strike, leg_barrier, ln_level, l, lp, k);
            const double other = __shfl_xor_sync(kFull, mine, 1);
            const double y = active && !odd ? 0.5 * (mine + other) : 0.0;
            const double s1 = warp_sum(y), s2 = warp_sum(y * y);
            if (lane == 0) wacc[warp * n_acc + k] += s1, wacc[warp * n_acc + a.n_out + k] += s2;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n_acc; t += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < n_warps; ++w) s += wacc[w * n_acc + t];
        partial[static_cast<long long>(blockIdx.x) * n_acc + t] = s;
    }
}

template <typename R>
using FusedFn = void (*)(FusedArgs<R>, long long, long long, uint32_t, uint32_t, double*);

template <typename R, int KIND, int PRODUCT, bool GT>
FusedFn<R> pick_n(int n) {
    if (n == 1) return fused_kernel<R, 1, KIND, PRODUCT, GT>;
    if (n == 2) return fused_kernel<R, 2, KIND, PRODUCT, GT>;
    if (n == 3) return fused_kernel<R, 3, KIND, PRODUCT, GT>;
    if constexpr (KIND == 1 || KIND == 0) {
        if (n == 4) return fused_kernel<R, 4, KIND, PRODUCT, GT>;
        if (n == 5) return fused_kernel<R, 5, KIND, PRODUCT, GT>;
    }
    return nullptr;
}

// Local-vol baskets of 2 to 5 names with the local-correlation mixer.
template <typename R, int PRODUCT, bool GT>
FusedFn<R> pick_mix(int n) {
    switch (n) {
        case 2: return fused_kernel<R, 2, 1, PRODUCT, GT, true>;
        case 3: return fused_kernel<R, 3, 1, PRODUCT, GT, true>;
        case 4: return fused_kernel<R, 4, 1, PRODUCT, GT, true>;
        case 5: return fused_kernel<R, 5, 1, PRODUCT, GT, true>;
        default: return nullptr;
    }
}

// table_global: the kinds with a table (local vol, SLV) read it from global memory.
template <typename R, int PRODUCT>
FusedFn<R> pick_fused(int kind, int n, bool table_global) {
    switch (kind) {
        case 0: return table_global ? nullptr : pick_n<R, 0, PRODUCT, false>(n);
        case 1: return table_global ? pick_n<R, 1, PRODUCT, true>(n) : pick_n<R, 1, PRODUCT, false>(n);
        case 2: return pick_n<R, 2, PRODUCT, false>(n);
        case 3: return table_global ? pick_n<R, 3, PRODUCT, true>(n) : pick_n<R, 3, PRODUCT, false>(n);
        case 4: return n == 1 ? qe_pair_kernel<R, PRODUCT> : nullptr;
        default: return nullptr;
    }
}

struct Blob {
    std::vector<unsigned char> bytes;
    template <typename T>
    int put(const T* src, size_t count) {
        const size_t at = (bytes.size() + 15) & ~static_cast<size_t>(15);
        const size_t n = count * sizeof(T);
        bytes.resize(at + ((n + 15) & ~static_cast<size_t>(15)), 0);
        if (src && n) std::memcpy(bytes.data() + at, src, n);
        return static_cast<int>(at);
    }
    template <typename T>
    int put(const std::vector<T>& v) {
        return put(v.data(), v.size());
    }
};

}  // namespace

// Packs the request for the specialised kernel; false when it does not apply (mixed kinds, a basket size without an
// instantiation, or inputs that would not fit the shared-memory budget), and the generic kernel then runs. The
// table goes into the stage when it fits beside the rest, else into global memory (the reference plan's rows: 801
// points for every step, megabytes), where it stays in L2 and is read through the read-only cache.
template <typename R>
bool fused_build(McPlan& plan, const ob_mc_request& rq) {
    const int n = rq.n_names, S = rq.n_steps;
    int kind = -1;
    if (rq.model == OB_MODEL_HESTON_QE) {
        kind = 4;
    } else {
        kind = rq.kind[0];
        for (int a = 1; a < n; ++a)
            if (rq.kind[a] != kind) return false;
    }
    if (rq.mixer && kind != 1) return false;  // the mixer beside other kinds: the generic kernel
    auto pick = [&](bool table_global) -> FusedFn<R> {
        const bool ladder = rq.product == OB_PRODUCT_LADDER;
        if (rq.mixer)
            return ladder ? (table_global ? pick_mix<R, OB_PRODUCT_LADDER, true>(n) : pick_mix<R, OB_PRODUCT_LADDER, false>(n))
                          : (table_global ? pick_mix<R, OB_PRODUCT_AUTOCALL, true>(n)
                                          : pick_mix<R, OB_PRODUCT_AUTOCALL, false>(n));
        return ladder ? pick_fused<R, OB_PRODUCT_LADDER>(kind, n, table_global)
                      : pick_fused<R, OB_PRODUCT_AUTOCALL>(kind, n, table_global);
    };
    if (!pick(false)) return false;
    FusedArgs<R> a{};
    a.n_steps = S, a.n_x = rq.n_x, a.same = rq.same;
    a.n_obs = rq.product == OB_PRODUCT_AUTOCALL ? rq.n_obs : 0;
    a.n_legs = rq.product == OB_PRODUCT_LADDER ? rq.n_legs : 0;
    a.n_out = rq.product == OB_PRODUCT_LADDER ? rq.n_legs + 1 : 4;
    a.top = static_cast<R>(rq.n_x - 1) - static_cast<R>(1e-4);
    a.spot0 = static_cast<R>(rq.spot[0]);
    Blob blob;
    std::vector<StepRec<R>> steps(S);
    for (int i = 0; i < S; ++i) {
        std::memset(&steps[i], 0, sizeof steps[i]);
        steps[i].dt = static_cast<R>(rq.dt[i]);
        steps[i].hdt = static_cast<R>(-0.5 * rq.dt[i]);
        steps[i].sdt = static_cast<R>(std::sqrt(rq.dt[i]));
        steps[i].obs = -1;
    }
    if (rq.product == OB_PRODUCT_AUTOCALL) {
        for (int j = 0; j < rq.n_obs; ++j) steps[rq.obs_step[j] - 1].obs = j;
        // steps without an observation: minus the number of steps to the next one (past the last, more than any
        // batch)
        int next = S + (1 << 20);
        for (int i = S; i >= 1; --i) {
            if (steps[i - 1].obs >= 0) next = i;
            else steps[i - 1].obs = i - next;
        }
    }
    a.off.step = blob.put(steps);
    const bool table = kind == 1 || kind == 3;
    if (kind == 4) {
        a.qe = make_qe_consts<R>(rq.heston, rq.r, rq.q, rq.dt[0]);
    } else {
        std::vector<NameStep<R>> ns(static_cast<size_t>(S) * n);
        for (int i = 1; i <= S; ++i)
            for (int k = 0; k < n; ++k) {
                NameStep<R>& r = ns[static_cast<size_t>(i - 1) * n + k];
                std::memset(&r, 0, sizeof r);
                r.lf = static_cast<R>(rq.log_fwd[static_cast<size_t>(k) * (S + 1) + i]);
                if (table) {
                    const int row = rq.step_row[static_cast<size_t>(k) * S + (i - 1)];
                    set_cell_row(r, rq.row_lo[row], rq.row_inv_dx[row], a.top);
                    r.row = row * (rq.n_x - 1);
                }
            }
        a.off.name_step = blob.put(ns);
        std::vector<R> root(static_cast<size_t>(n) * n);
        for (size_t k = 0; k < root.size(); ++k) root[k] = static_cast<R>(rq.root[k]);
        a.off.root = blob.put(root);
        std::vector<R> hes(8 * static_cast<size_t>(n), R(0));
        for (int k = 0; k < n; ++k) {
            for (int f = 0; f < 5; ++f) hes[8 * k + f] = static_cast<R>(rq.heston[5 * k + f]);
            const R rho = hes[8 * k + 4];
            hes[8 * k + 5] = static_cast<R>(std::sqrt(R(1) - rho * rho));
            hes[8 * k + 6] = static_cast<R>(rq.cvar[k]);  // Black-Scholes
        }
        a.off.hes = blob.put(hes);
        if (rq.mixer) {
            std::vector<R> den(S), low(static_cast<size_t>(n) * n);
            for (int i = 0; i < S; ++i)  // R arithmetic as the generic step: sigma sqrt(max(t0, 1/12))
                den[i] = static_cast<R>(rq.mix[4]) * std::sqrt(std::max(static_cast<R>(rq.t0[i]), R(1.0 / 12)));
            for (size_t k = 0; k < low.size(); ++k) low[k] = static_cast<R>(rq.low_root[k]);
            a.off.mix_den = blob.put(den), a.off.low_root = blob.put(low);
            a.mix_base = static_cast<R>(rq.mix[0]) + static_cast<R>(rq.mix[1]);
            a.mix_down = static_cast<R>(rq.mix[2]), a.mix_up = static_cast<R>(rq.mix[3]);
            a.mix_sign = static_cast<R>(rq.mix[5]), a.mix_cos = static_cast<R>(rq.mix[6]);
            a.mix_sin = static_cast<R>(rq.mix[7]);
        }
    }
    if (rq.product == OB_PRODUCT_LADDER) {
        std::vector<int> type(rq.n_legs), bar(rq.n_legs);
        std::vector<R> strike(rq.n_legs), lvl(rq.n_legs);
        for (int k = 0; k < rq.n_legs; ++k) {
            type[k] = rq.leg_type[k];
            strike[k] = static_cast<R>(rq.leg_strike[k]);
            bar[k] = rq.leg_barrier ? rq.leg_barrier[k] : 0;
            lvl[k] = bar[k] ? static_cast<R>(std::log(rq.leg_level[k] / rq.spot[0])) : R(0);
        }
        a.off.leg_type = blob.put(type), a.off.leg_strike = blob.put(strike);
        a.off.leg_barrier = blob.put(bar), a.off.ln_level = blob.put(lvl);
        a.discount = rq.discount;
    } else {
        std::vector<R> trig(rq.n_obs);
        for (int j = 0; j < rq.n_obs; ++j)
            trig[j] = rq.trigger[j] > 0 ? static_cast<R>(std::log(rq.trigger[j])) : R(1e30);
        a.off.ln_trig = blob.put(trig);
        a.off.obs_disc = blob.put(rq.obs_discount, rq.n_obs);
        a.has_coupon = rq.coupon > 0.0 || rq.coupon_barrier > 0.0;
        a.ln_cb = rq.coupon_barrier > 0 ? static_cast<R>(std::log(rq.coupon_barrier)) : R(-1e30);
        a.ln_ki = rq.ki_barrier > 0 ? static_cast<R>(std::log(rq.ki_barrier)) : R(-1e30);
        a.coupon = rq.coupon, a.put_strike = rq.put_strike, a.memory = rq.memory, a.ki_daily = rq.ki_daily;
    }
    const int block = 512;
    const size_t acc_bytes = static_cast<size_t>(block / 32) * 2 * a.n_out * sizeof(double);
    const size_t budget = sizeof(R) == 4 ? (110u << 10) : (220u << 10);  // two blocks a SM in float, one in double
    bool table_global = false;
    if (table) {
        std::vector<Pair2<R>> tab(static_cast<size_t>(rq.n_rows) * (rq.n_x - 1));
        for (int r = 0; r < rq.n_rows; ++r)
            for (int k = 0; k + 1 < rq.n_x; ++k) {
                const double* row = rq.table + static_cast<size_t>(r) * rq.n_x;
                tab[static_cast<size_t>(r) * (rq.n_x - 1) + k] = {static_cast<R>(row[k]),
                                                                   static_cast<R>(row[k + 1] - row[k])};
            }
        const size_t at = (blob.bytes.size() + 15) & ~static_cast<size_t>(15);
        table_global = at + tab.size() * sizeof(Pair2<R>) + acc_bytes > budget;
        if (table_global) a.tab = plan.arena.put_raw(tab.data(), tab.size());
        else a.off.table2 = blob.put(tab);
    }
    const FusedFn<R> fn = pick(table_global);
    a.smem_blob = static_cast<int>((blob.bytes.size() + 15) & ~static_cast<size_t>(15));
    const size_t smem = a.smem_blob + acc_bytes;
    if (smem > budget) return false;
    unsigned char* d = plan.arena.alloc<unsigned char>(std::max<size_t>(16, blob.bytes.size()));
    check_cuda(cudaMemcpy(d, blob.bytes.data(), blob.bytes.size(), cudaMemcpyHostToDevice), "copy blob");
    a.blob = d;
    const void* k = reinterpret_cast<const void*>(fn);
    allow_smem(k, smem);
    const int per_sm = occupancy(k, block, smem);
    if (per_sm < 1) return false;
    plan.fused = true;
    plan.threads_per_pair = kind == 4 ? 2 : 1;
    plan.kernel = k;
    plan.block = block;
    plan.smem_bytes = smem;
    plan.blocks_per_sm = per_sm;
    plan.n_out = a.n_out;
    plan.fused_args<R>() = a;
    return true;
}

template bool fused_build<float>(McPlan&, const ob_mc_request&);
template bool fused_build<double>(McPlan&, const ob_mc_request&);

}  // namespace ob
