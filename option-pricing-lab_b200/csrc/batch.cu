// Batched risk revaluation: a book of trades of uneven sizes, each revalued under spot, carry, volatility and
// correlation scenarios, in one replay of a CUDA graph of persistent kernels.
//
// What the reference does one simulation at a time (packages/risk/src/optlab/risk/engine.py:382-425,563-644: spot
// shocks share the base simulation as path factors, every vol or skew shock re-simulates on the group's seed) runs
// here as work items (trade, simulation, tile of pairs) pulled from device queues: one queue and one persistent
// kernel per trade class (local vol with N = 1..5 names or Heston QE, ladder or autocall), the kernels on their own
// streams inside one graph, so that large and small trades fill the GPU together. A base simulation evaluates the base
// and every spot scenario at once: the path keeps its observation log-performances and extremes, and a spot move is
// a shift of them (the local vol is in log-moneyness). A vol scenario reads its own copy of the tables, made once on
// the host with every node moved to (sigma + shift + tilt k)^2, floored at 1 % vol (1 + n_vol copies of the pool,
// 42 MB in float for the benchmark's book: L2-sized), on the same random numbers; the step is then the fused
// kernel's (one table read, one multiply-add). A carry scenario (a move of the rate, discounting included, or of
// the dividend yield) also rides on the base simulation, as the reference's forward ratio F'(t) / F(t) (:8-11): the
// path keeps its extremes and daily low again under each carry's drift (Delta t per step), and the payments take
// the moved discount. A correlation scenario re-simulates the multi-name local-vol trades on a moved root, on the
// same random numbers. Each tile writes its own partial sums, and a last kernel adds the
// tiles of each (trade, scenario) in order, so the results do not depend on the schedule. Tiles and block sizes
// are chosen per class by ob_batch_tune, which times candidates on the class's own work.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <numeric>
#include <vector>

#include "mc.cuh"

namespace ob {

namespace {

constexpr int kBatchMaxObs = 64;
constexpr int kBatchMaxOut = 32;  // 1 + spot + carry scenarios per base simulation
constexpr int kBatchMaxCarry = OB_BATCH_MAX_CARRY;

template <typename R>
struct BTrade {
    int kind, product, n, n_steps;
    long long n_pairs;
    uint32_t k0, k1;
    int row0, root0, n_legs, leg0, n_obs, obs0;
    R lf_rate;  // (r - q): the log-forward at grid point i is lf_rate i dt
    QeConsts<R> qe;
    int has_coupon, memory, ki_daily;
    R ln_cb, ln_ki;
    double coupon, put_strike, discount;
    int slot0;       // first partial slot of its base simulation
    int corr_root0;  // its moved roots, one per correlation scenario
    double carry_df[kBatchMaxCarry];  // the ladder's payment under each carry: exp(-rate move T)
};

template <typename R>
struct BDev {
    const BTrade<R>* trades;
    const Pair2<R>* tab;  // (1 + n_vol) x pool rows x (n_x - 1): (var_i, var_i+1 - var_i), base then each vol move
    long long tab_stride; // pool rows x (n_x - 1)
    const R* row_org;     // the row's origin and 1 / dx in the cell form (cell_row)
    const R* row_inv_dx;
    const int* row_of;    // step -> expiry row
    const R* root;
    const int* leg_type;
    const R* leg_strike;
    const int* leg_barrier;
    const R* ln_level;
    const int* obs_step;
    const R* ln_trig;
    const double* obs_disc;
    const R* ln_spot;     // n_spot: ln(1 + spot move)
    const double* obs_carry_df;  // n_carry x observation pool: exp(-rate move t_obs)
    R carry_dt[kBatchMaxCarry];  // per carry: the drift move (rate - dividend) times dt
    int n_spot, n_carry, n_vol, n_obs_pool, n_exp, n_x;
    R hdt, sdt, dt, top;
    double* slots;        // partial sums: per tile, 2 x outputs
    const int* sim_slot;  // per (trade, simulation): first slot
    int tile;
};

// What a leg keeps of its path for the payoffs: the ladder's terminal and extreme log performances, or the
// autocall's observations and its lowest daily log performance.
template <typename R, int PRODUCT>
struct Rec;
template <typename R>
struct Rec<R, OB_PRODUCT_LADDER> {
    R last, hi, lo;
    R hc[kBatchMaxCarry], lc[kBatchMaxCarry];  // extremes under each carry's drift
};
template <typename R>
struct Rec<R, OB_PRODUCT_AUTOCALL> {
    R low;
    R lowc[kBatchMaxCarry];  // daily low under each carry's drift
    R obs[kBatchMaxObs];
};

// The legs' undiscounted sum at a terminal log performance and extremes.
template <typename R>
__device__ __forceinline__ double ladder_legs(const BDev<R>& d, const BTrade<R>& t, R lpT, R hi, R lo) {
    const R U = m_exp(lpT);
    double v = 0.0;
    for (int k = 0; k < t.n_legs; ++k) {
        const int type = d.leg_type[t.leg0 + k];
        const R K = d.leg_strike[t.leg0 + k];
        R pay = type == 1 ? m_max(U - K, R(0)) : type == 2 ? m_max(K - U, R(0)) : type == 3 ? U - K : R(0);
        const int bt = d.leg_barrier[t.leg0 + k];
        const R H = d.ln_level[t.leg0 + k];
        const bool up = hi >= H, down = lo <= H;
        if ((bt == OB_BARRIER_UP_OUT && up) || (bt == OB_BARRIER_DOWN_OUT && down) || (bt == OB_BARRIER_UP_IN && !up) ||
            (bt == OB_BARRIER_DOWN_IN && !down))
            pay = R(0);
        v += static_cast<double>(pay);
    }
    return v;
}

// c < 0: the recorded path shifted by a spot move; c >= 0: under carry c (no spot move).
template <typename R>
__device__ __forceinline__ double ladder_value(const BDev<R>& d, const BTrade<R>& t, const Rec<R, OB_PRODUCT_LADDER>& r,
                                               R shift, int c) {
    if (c < 0) return t.discount * ladder_legs(d, t, r.last + shift, r.hi + shift, r.lo + shift);
    const R lpT = r.last + d.carry_dt[c] * static_cast<R>(t.n_steps);
    return t.discount * t.carry_df[c] * ladder_legs(d, t, lpT, r.hc[c], r.lc[c]);
}

// The Phoenix of the fused kernel (coupon with memory, call before the last date, knock-in put at the last), on the
// recorded observations shifted by a spot move (c < 0) or moved by carry c.
template <typename R>
__device__ __forceinline__ double autocall_value(const BDev<R>& d, const BTrade<R>& t,
                                                 const Rec<R, OB_PRODUCT_AUTOCALL>& r, R shift, int c) {
    double pv = 0.0;
    int missed = 0;
    for (int j = 0; j < t.n_obs; ++j) {
        R lp = r.obs[j] + shift;
        double D = d.obs_disc[t.obs0 + j];
        if (c >= 0) {
            lp += d.carry_dt[c] * static_cast<R>(d.obs_step[t.obs0 + j]);
            D *= d.obs_carry_df[c * d.n_obs_pool + t.obs0 + j];
        }
        if (t.has_coupon) {
            if (lp >= t.ln_cb) {
                pv += D * t.coupon * (t.memory ? 1 + missed : 1);
                missed = 0;
            } else {
                ++missed;
            }
        }
        if (j < t.n_obs - 1) {
            if (lp >= d.ln_trig[t.obs0 + j]) return pv + D;
        } else {
            const R low = m_min((c < 0 ? r.low : r.lowc[c]) + shift, shift);  // the start is part of the window
            const bool ki = t.ki_daily ? low < t.ln_ki : lp < t.ln_ki;
            const double perf = static_cast<double>(m_exp(lp));
            const double put = t.put_strike - perf > 0.0 ? t.put_strike - perf : 0.0;
            pv += D * (ki ? 1.0 - put : 1.0);
        }
    }
    return pv;
}

template <typename R>
__device__ __forceinline__ double value(const BDev<R>& d, const BTrade<R>& t, const Rec<R, OB_PRODUCT_LADDER>& r, R s,
                                        int c) {
    return ladder_value(d, t, r, s, c);
}
template <typename R>
__device__ __forceinline__ double value(const BDev<R>& d, const BTrade<R>& t, const Rec<R, OB_PRODUCT_AUTOCALL>& r,
                                        R s, int c) {
    return autocall_value(d, t, r, s, c);
}

template <typename R>
__device__ __forceinline__ void rec_init(Rec<R, OB_PRODUCT_LADDER>& r) {
    const R big = static_cast<R>(sizeof(R) == 4 ? 1e30 : 1e300);
    r.last = R(0), r.hi = -big, r.lo = big;
#pragma unroll
    for (int c = 0; c < kBatchMaxCarry; ++c) r.hc[c] = -big, r.lc[c] = big;
}
template <typename R>
__device__ __forceinline__ void rec_init(Rec<R, OB_PRODUCT_AUTOCALL>& r) {
    r.low = R(0);
#pragma unroll
    for (int c = 0; c < kBatchMaxCarry; ++c) r.lowc[c] = R(0);
}

// Step end i of one leg, with lp the worst log performance and j the observation ending there (-1: none).
template <typename R>
__device__ __forceinline__ void rec_step(Rec<R, OB_PRODUCT_LADDER>& r, R lp, int j) {
    r.last = lp, r.hi = m_max(r.hi, lp), r.lo = m_min(r.lo, lp);
}
template <typename R>
__device__ __forceinline__ void rec_step(Rec<R, OB_PRODUCT_AUTOCALL>& r, R lp, int j) {
    r.low = m_min(r.low, lp);
    if (j >= 0) r.obs[j] = lp;
}

// The first nc carry moves at step end i: the log performance lp + Delta_c i dt.
template <typename R>
__device__ __forceinline__ void rec_carry(Rec<R, OB_PRODUCT_LADDER>& r, R lp, R fi, const BDev<R>& d, int nc) {
#pragma unroll
    for (int c = 0; c < kBatchMaxCarry; ++c)
        if (c < nc) {
            const R l = lp + d.carry_dt[c] * fi;
            r.hc[c] = m_max(r.hc[c], l), r.lc[c] = m_min(r.lc[c], l);
        }
}
template <typename R>
__device__ __forceinline__ void rec_carry(Rec<R, OB_PRODUCT_AUTOCALL>& r, R lp, R fi, const BDev<R>& d, int nc) {
#pragma unroll
    for (int c = 0; c < kBatchMaxCarry; ++c)
        if (c < nc) r.lowc[c] = m_min(r.lowc[c], lp + d.carry_dt[c] * fi);
}

template <typename R, int N, bool QE, int PRODUCT>
__global__ void __launch_bounds__(256) batch_kernel(BDev<R> d, const int4* __restrict__ items, int n_items,
                                                    int* counter) {
    constexpr int C = QE ? 2 : N;
    constexpr int G = C % 4 == 0 ? 1 : (C % 2 == 0 ? 2 : 4);
    constexpr int NB = C * G / 4;
    __shared__ int s_item;
    __shared__ double wacc[8][2 * kBatchMaxOut];
    __shared__ R s_root[25];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const int4 item = items[it];
        const BTrade<R>& t = d.trades[item.x];
        // sim 0: the base (with spot and carry moves); 1..n_vol: vol moves; after those: correlation moves
        const int sim = item.y, tile = item.z;
        const int nc = sim == 0 ? d.n_carry : 0;
        const int n_out = sim == 0 ? 1 + d.n_spot + nc : 1;
        const bool shocked = sim > 0 && sim <= d.n_vol;
        for (int k = threadIdx.x; k < 8 * 2 * kBatchMaxOut; k += blockDim.x) (&wacc[0][0])[k] = 0.0;
        if (!QE) {
            const int root = sim > d.n_vol ? t.corr_root0 + (sim - 1 - d.n_vol) * N * N : t.root0;
            for (int k = threadIdx.x; k < N * N; k += blockDim.x) s_root[k] = d.root[root + k];
        }
        __syncthreads();
        const Pair2<R>* tab = d.tab + (shocked ? sim : 0) * d.tab_stride;
        const long long p0 = static_cast<long long>(tile) * d.tile;
        const long long p1 = min(p0 + d.tile, t.n_pairs);
        const int S = t.n_steps;
        for (long long base = p0 + warp * 32; base < p1; base += blockDim.x) {
            const bool active = base + lane < p1;
            const uint64_t pair = static_cast<uint64_t>(active ? base + lane : p1 - 1);
            R x0[N], x1[N], v0 = t.qe.v0, v1 = t.qe.v0;
#pragma unroll
            for (int n = 0; n < N; ++n) x0[n] = x1[n] = R(0);
            Rec<R, PRODUCT> r0, r1;
            rec_init(r0), rec_init(r1);
            // the next observation and its step, in registers (the schedule is read again only at an observation)
            int next_obs = 0;
            int obs_at = PRODUCT == OB_PRODUCT_AUTOCALL && t.n_obs > 0 ? d.obs_step[t.obs0] : -1;
            for (int i0 = 1, b = 0; i0 <= S; i0 += G, ++b) {
                R z[C * G];
#pragma unroll
                for (int k = 0; k < NB; ++k)
                    normals4<R>(pair, static_cast<uint64_t>(b) * NB + k, 0u, t.k0, t.k1, z[4 * k], z[4 * k + 1],
                                z[4 * k + 2], z[4 * k + 3]);
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    const int i = i0 + g;
                    if (G > 1 && i > S) break;
                    R lp0, lp1;
                    if (QE) {
                        qe_step(t.qe, x0[0], v0, z[2 * g], z[2 * g + 1]);
                        qe_step(t.qe, x1[0], v1, -z[2 * g], -z[2 * g + 1]);
                        lp0 = x0[0], lp1 = x1[0];
                    } else {
                        const int erow = d.row_of[i - 1];
                        const R lf = t.lf_rate * (static_cast<R>(i) * d.dt);
                        lp0 = R(1e30), lp1 = R(1e30);
#pragma unroll
                        for (int n = 0; n < N; ++n) {
                            R zc = R(0);
#pragma unroll
                            for (int m = 0; m < N; ++m) zc += s_root[n * N + m] * z[g * C + m];
                            const int row = t.row0 + n * d.n_exp + erow;
                            const R org = d.row_org[row], inv = d.row_inv_dx[row];
                            const Pair2<R>* trow = tab + static_cast<long long>(row) * (d.n_x - 1);
                            const R zd = d.sdt * zc;  // sqrt(dt) z, the legs' +-
#pragma unroll
                            for (int leg = 0; leg < 2; ++leg) {
                                R& x = leg ? x1[n] : x0[n];
                                int j;
                                R w;
                                table_cell(org, inv, d.top, x, j, w);
                                const Pair2<R> p = trow[j];
                                const R var = p.a + w * p.b;
                                x = lv_advance(x, var, d.hdt, leg ? -zd : zd);
                                if (leg) lp1 = m_min(lp1, x + lf);
                                else lp0 = m_min(lp0, x + lf);
                            }
                        }
                    }
                    int j = -1;
                    if (PRODUCT == OB_PRODUCT_AUTOCALL && obs_at == i) {
                        j = next_obs++;
                        obs_at = next_obs < t.n_obs ? d.obs_step[t.obs0 + next_obs] : -1;
                    }
                    rec_step(r0, lp0, j);
                    rec_step(r1, lp1, j);
                    if (nc) rec_carry(r0, lp0, static_cast<R>(i), d, nc), rec_carry(r1, lp1, static_cast<R>(i), d, nc);
                }
            }
            for (int o = 0; o < 1 + (sim == 0 ? d.n_spot : 0); ++o) {
                const R sh = o == 0 ? R(0) : d.ln_spot[o - 1];
                const double y = active ? 0.5 * (value(d, t, r0, sh, -1) + value(d, t, r1, sh, -1)) : 0.0;
                const double s1 = warp_sum(y), s2 = warp_sum(y * y);
                if (lane == 0) wacc[warp][o] += s1, wacc[warp][kBatchMaxOut + o] += s2;
            }
#pragma unroll
            for (int c = 0; c < kBatchMaxCarry; ++c)
                if (c < nc) {
                    const int o = 1 + d.n_spot + c;
                    const double y = active ? 0.5 * (value(d, t, r0, R(0), c) + value(d, t, r1, R(0), c)) : 0.0;
                    const double s1 = warp_sum(y), s2 = warp_sum(y * y);
                    if (lane == 0) wacc[warp][o] += s1, wacc[warp][kBatchMaxOut + o] += s2;
                }
        }
        __syncthreads();
        double* out = d.slots + (static_cast<long long>(d.sim_slot[item.w]) + tile) * 2 * kBatchMaxOut;
        for (int k = threadIdx.x; k < n_out; k += blockDim.x) {
            double s = 0.0, s2 = 0.0;
            for (int w = 0; w < n_warps; ++w) s += wacc[w][k], s2 += wacc[w][kBatchMaxOut + k];
            out[k] = s, out[kBatchMaxOut + k] = s2;
        }
        __syncthreads();
    }
}

// Per (trade, simulation): the sums of its tiles, in tile order. One warp per (simulation, output).
__global__ void batch_reduce(const double* __restrict__ slots, const int* __restrict__ sim_slot,
                             const int* __restrict__ sim_tiles, const int* __restrict__ sim_outs, int n_sims,
                             double* __restrict__ sums) {
    const int lane = threadIdx.x & 31;
    const long long w = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (w >= static_cast<long long>(n_sims) * kBatchMaxOut) return;
    const int sim = static_cast<int>(w / kBatchMaxOut), o = static_cast<int>(w % kBatchMaxOut);
    if (o >= sim_outs[sim]) return;
    double s = 0.0, s2 = 0.0;
    for (int k = lane; k < sim_tiles[sim]; k += 32) {
        const double* p = slots + (static_cast<long long>(sim_slot[sim]) + k) * 2 * kBatchMaxOut;
        s += p[o], s2 += p[kBatchMaxOut + o];
    }
    s = warp_sum(s), s2 = warp_sum(s2);
    if (lane == 0) sums[(static_cast<long long>(sim) * kBatchMaxOut + o) * 2] = s,
                   sums[(static_cast<long long>(sim) * kBatchMaxOut + o) * 2 + 1] = s2;
}

template <typename R>
using BatchFn = void (*)(BDev<R>, const int4*, int, int*);

template <typename R, int PRODUCT>
BatchFn<R> pick_batch(bool qe, int n) {
    if (qe) return batch_kernel<R, 1, true, PRODUCT>;
    switch (n) {
        case 1: return batch_kernel<R, 1, false, PRODUCT>;
        case 2: return batch_kernel<R, 2, false, PRODUCT>;
        case 3: return batch_kernel<R, 3, false, PRODUCT>;
        case 4: return batch_kernel<R, 4, false, PRODUCT>;
        default: return batch_kernel<R, 5, false, PRODUCT>;
    }
}

}  // namespace

// A trade class: the trades sharing one kernel (model, names, product), with its tuned shape.
struct BClass {
    bool qe = false;
    int n = 1, product = 0;
    int tile = 8192, block = 256;
    double untuned_ms = 0.0, tuned_ms = 0.0;  // the autotuner's sample at the shape before tuning and at the kept one
    std::vector<int> trades;
    const void* kernel = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
};

// Slots and work items for one choice of tiles: per (trade, simulation) its tiles and first slot, per class its
// items. A layout owns its device buffers; a captured graph reads the main layout's.
struct BLayout {
    DeviceArena arena;
    std::vector<int> tile_of_class;
    std::vector<int> sim_tiles, sim_slot;
    int n_slots = 0;
    int* d_sim_slot = nullptr;
    int* d_sim_tiles = nullptr;
    double* d_slots = nullptr;
    double* d_sums = nullptr;
    std::vector<int4*> d_items;   // per class
    std::vector<int> n_items;     // per class
    std::vector<int*> d_counter;  // per class
    // the per-trade comparison: every simulation's items contiguous, one counter each
    std::vector<int4> pt_items;
    std::vector<int> pt_first, pt_count, pt_class;
    int4* d_pt_items = nullptr;
    int* d_pt_counters = nullptr;
};

struct Batch {
    DeviceArena arena;
    int precision = OB_FP32, sms = 0;
    int n_trades = 0, n_spot = 0, n_vol = 0, n_carry = 0, n_corr = 0;
    std::vector<ob_batch_trade> trades;
    std::vector<BClass> classes;
    std::vector<int> class_of_trade;
    BDev<float> df{};
    BDev<double> dd{};
    std::vector<int> sim_of_trade, sim_outs;
    int n_sims = 0;
    int* d_sim_outs = nullptr;
    BLayout main, per_trade;
    BLayout* last_layout = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, fork = nullptr;
    cudaStream_t last = nullptr;

    template <typename R>
    BDev<R>& dev();
    template <typename R>
    void build(const ob_batch_request& rq);
    void simulations();
    // per trade: its base, then under local vol one per vol move, then (2 names or more) one per correlation move
    int sims_of(int i) const {
        const ob_batch_trade& t = trades[i];
        return t.model == OB_MODEL_PATHS ? 1 + n_vol + (t.n_names > 1 ? n_corr : 0) : 1;
    }
    void layout(BLayout& L, const std::vector<int>& tiles, int only_class = -1, int max_sims = 0);
    template <typename R>
    void launch_class(const BLayout& L, int ci, cudaStream_t st, const int4* items, int n_items, int* counter,
                      int grid, int block);
    void run_all(cudaStream_t st);
    void reduce(const BLayout& L, cudaStream_t st);
    double time_class(int ci, int tile, int block, int max_sims);
    std::vector<int> tiles() const {
        std::vector<int> t;
        for (const auto& c : classes) t.push_back(c.tile);
        return t;
    }
    ~Batch();
};

template <>
BDev<float>& Batch::dev<float>() {
    return df;
}
template <>
BDev<double>& Batch::dev<double>() {
    return dd;
}

Batch::~Batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto& c : classes) {
        if (c.stream) cudaStreamDestroy(c.stream);
        if (c.done) cudaEventDestroy(c.done);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (fork) cudaEventDestroy(fork);
}

namespace {

void check_batch(const ob_batch_request& rq) {
    if (rq.n_trades < 1 || !rq.trades) invalid("a batch needs trades");
    if (!(rq.dt > 0) || rq.n_exp < 1 || rq.n_x < 2 || !(rq.horizon > 0)) invalid("bad step or table grid");
    if (rq.n_spot < 0 || rq.n_spot + 1 > kBatchMaxOut || (rq.n_spot && !rq.spot_shift)) invalid("n_spot must be 0 to 31");
    if (rq.n_vol < 0 || (rq.n_vol && (!rq.vol_shift || !rq.vol_tilt || !rq.vol_table))) invalid("bad vol scenarios");
    if (rq.n_carry < 0 || rq.n_carry > kBatchMaxCarry || (rq.n_carry && (!rq.carry_rate || !rq.carry_div)))
        invalid("n_carry must be 0 to 4, with its moves");
    if (1 + rq.n_spot + rq.n_carry > kBatchMaxOut) invalid("1 + n_spot + n_carry must be at most 32");
    for (int k = 0; k < rq.n_carry; ++k)
        if (!std::isfinite(rq.carry_rate[k]) || !std::isfinite(rq.carry_div[k])) invalid("carry moves must be finite");
    if (rq.n_corr < 0) invalid("n_corr must be 0 or more");
    for (int k = 0; k < rq.n_spot; ++k)
        if (!(rq.spot_shift[k] > -1.0)) invalid("a spot move must be above -100 %");
    for (int i = 0; i < rq.n_trades; ++i) {
        const ob_batch_trade& t = rq.trades[i];
        if (t.model != OB_MODEL_PATHS && t.model != OB_MODEL_HESTON_QE) invalid("trade model must be 0 or 1");
        if (t.model == OB_MODEL_HESTON_QE && t.n_names != 1) invalid("a Heston trade has one name");
        if (t.n_names < 1 || t.n_names > 5) invalid("a trade has 1 to 5 names");
        if (t.n_steps < 1 || t.n_pairs < 1) invalid("a trade needs steps and pairs");
        if (t.model == OB_MODEL_PATHS) {
            if (!rq.table || !rq.row_lo || !rq.row_inv_dx || !rq.root) invalid("local-vol trades need the pools");
            if (t.table_row0 < 0 || t.root0 < 0) invalid("bad pool offsets");
            if (rq.n_corr && t.n_names > 1 && t.corr_root0 < 0) invalid("bad moved-root offset");
        } else {
            const double* h = t.heston;
            if (!(h[0] >= 0 && h[1] > 0 && h[2] > 0 && h[3] > 0 && std::fabs(h[4]) <= 1))
                invalid("Heston parameters out of range");
        }
        if (t.product == OB_PRODUCT_LADDER) {
            if (t.n_legs < 1 || t.leg0 < 0 || !rq.leg_type || !rq.leg_strike || !rq.leg_barrier || !rq.leg_level)
                invalid("a ladder trade needs legs");
        } else if (t.product == OB_PRODUCT_AUTOCALL) {
            if (t.n_obs < 1 || t.n_obs > kBatchMaxObs || t.obs0 < 0 || !rq.obs_step || !rq.obs_trigger ||
                !rq.obs_discount)
                invalid("an autocall trade needs 1 to 64 observations");
            for (int j = 0; j < t.n_obs; ++j) {
                const int s = rq.obs_step[t.obs0 + j];
                if (s < 1 || s > t.n_steps || (j && s <= rq.obs_step[t.obs0 + j - 1]))
                    invalid("observation steps must increase within the trade's steps");
            }
        } else {
            invalid("product must be 0 or 1");
        }
    }
}

}  // namespace

template <typename R>
void Batch::build(const ob_batch_request& rq) {
    n_trades = rq.n_trades, n_spot = rq.n_spot, n_vol = rq.n_vol, n_carry = rq.n_carry, n_corr = rq.n_corr;
    trades.assign(rq.trades, rq.trades + rq.n_trades);
    BDev<R>& d = dev<R>();
    d = BDev<R>{};
    d.n_spot = n_spot, d.n_carry = n_carry, d.n_vol = n_vol, d.n_exp = rq.n_exp, d.n_x = rq.n_x;
    for (int c = 0; c < n_carry; ++c) d.carry_dt[c] = static_cast<R>((rq.carry_rate[c] - rq.carry_div[c]) * rq.dt);
    d.hdt = static_cast<R>(-0.5 * rq.dt), d.sdt = static_cast<R>(std::sqrt(rq.dt)), d.dt = static_cast<R>(rq.dt);
    d.top = static_cast<R>(rq.n_x - 1) - static_cast<R>(1e-4);
    int max_steps = 1, max_row = 0, max_root = 0, max_leg = 0, max_obs = 0;
    for (const auto& t : trades) {
        max_steps = std::max(max_steps, t.n_steps);
        if (t.model == OB_MODEL_PATHS) {
            max_row = std::max(max_row, t.table_row0 + t.n_names * rq.n_exp);
            max_root = std::max(max_root, t.root0 + t.n_names * t.n_names);
            if (n_corr && t.n_names > 1)
                max_root = std::max(max_root, t.corr_root0 + n_corr * t.n_names * t.n_names);
        }
        if (t.product == OB_PRODUCT_LADDER) max_leg = std::max(max_leg, t.leg0 + t.n_legs);
        else max_obs = std::max(max_obs, t.obs0 + t.n_obs);
    }
    // step -> expiry row: the first expiry strictly after the step's start
    std::vector<int> row_of(max_steps);
    for (int i = 0; i < max_steps; ++i) {
        const double t0 = i * rq.dt;
        int j = 0;
        while (j < rq.n_exp - 1 && rq.horizon * (j + 1) / rq.n_exp <= t0 + 1e-12) ++j;
        row_of[i] = j;
    }
    d.row_of = arena.put<int>(row_of.data(), row_of.size());
    if (max_row > rq.n_rows) invalid("a trade reads table rows beyond the pool's n_rows");
    if (max_row > 0) {
        // the base tables, then each vol move's (the host re-tabulated the pool under each move of the implied vols),
        // as (var_i, var_i+1 - var_i) pairs
        const int nx = rq.n_x;
        d.tab_stride = static_cast<long long>(max_row) * (nx - 1);
        const double tab_bytes = static_cast<double>(1 + n_vol) * d.tab_stride * sizeof(Pair2<R>);
        size_t free_mem = 0, total_mem = 0;
        check_cuda(cudaMemGetInfo(&free_mem, &total_mem), "cudaMemGetInfo");
        if (tab_bytes > 0.5 * static_cast<double>(free_mem))
            invalid("the vol scenarios' tables (one copy of the table pool per scenario) need more than half the free "
                    "device memory: fewer vol scenarios or a smaller pool");
        std::vector<Pair2<R>> tab(static_cast<size_t>(1 + n_vol) * d.tab_stride);
        std::vector<double> v(nx);
        const long long pool = static_cast<long long>(rq.n_rows) * nx;
        for (int s = 0; s <= n_vol; ++s)
            for (int r = 0; r < max_row; ++r) {
                const double* src = s == 0 ? rq.table + static_cast<size_t>(r) * nx
                                           : rq.vol_table + (s - 1) * pool + static_cast<long long>(r) * nx;
                for (int k = 0; k < nx; ++k) v[k] = src[k];
                Pair2<R>* out = tab.data() + s * d.tab_stride + static_cast<long long>(r) * (nx - 1);
                for (int k = 0; k + 1 < nx; ++k) out[k] = {static_cast<R>(v[k]), static_cast<R>(v[k + 1] - v[k])};
            }
        d.tab = arena.put<Pair2<R>>(tab.data(), tab.size());
        std::vector<R> org(max_row), inv(max_row);
        for (int r = 0; r < max_row; ++r) cell_row(rq.row_lo[r], rq.row_inv_dx[r], d.top, org[r], inv[r]);
        d.row_org = arena.put<R>(org.data(), org.size());
        d.row_inv_dx = arena.put<R>(inv.data(), inv.size());
        d.root = arena.put<R>(rq.root, max_root);
    }
    if (max_leg > 0) {
        std::vector<R> lvl(max_leg);
        for (int k = 0; k < max_leg; ++k)
            lvl[k] = rq.leg_barrier[k] ? static_cast<R>(std::log(rq.leg_level[k])) : R(0);
        d.leg_type = arena.put<int>(rq.leg_type, max_leg);
        d.leg_strike = arena.put<R>(rq.leg_strike, max_leg);
        d.leg_barrier = arena.put<int>(rq.leg_barrier, max_leg);
        d.ln_level = arena.put<R>(lvl.data(), lvl.size());
    }
    if (max_obs > 0) {
        std::vector<R> trig(max_obs);
        for (int k = 0; k < max_obs; ++k)
            trig[k] = rq.obs_trigger[k] > 0 ? static_cast<R>(std::log(rq.obs_trigger[k])) : R(1e30);
        d.obs_step = arena.put<int>(rq.obs_step, max_obs);
        d.ln_trig = arena.put<R>(trig.data(), trig.size());
        d.obs_disc = arena.put<double>(rq.obs_discount, max_obs);
        d.n_obs_pool = max_obs;
        if (n_carry) {
            std::vector<double> df(static_cast<size_t>(n_carry) * max_obs);
            for (int c = 0; c < n_carry; ++c)
                for (int k = 0; k < max_obs; ++k)
                    df[static_cast<size_t>(c) * max_obs + k] = std::exp(-rq.carry_rate[c] * rq.obs_step[k] * rq.dt);
            d.obs_carry_df = arena.put<double>(df.data(), df.size());
        }
    }
    if (n_spot) {
        std::vector<R> ls(n_spot);
        for (int k = 0; k < n_spot; ++k) ls[k] = static_cast<R>(std::log1p(rq.spot_shift[k]));
        d.ln_spot = arena.put<R>(ls.data(), ls.size());
    }
    std::vector<BTrade<R>> bt(n_trades);
    std::map<std::tuple<bool, int, int>, int> cls;
    class_of_trade.assign(n_trades, 0);
    for (int i = 0; i < n_trades; ++i) {
        const ob_batch_trade& t = trades[i];
        BTrade<R>& b = bt[i];
        b = BTrade<R>{};
        b.kind = t.model, b.product = t.product, b.n = t.n_names, b.n_steps = t.n_steps, b.n_pairs = t.n_pairs;
        b.k0 = static_cast<uint32_t>(t.seed), b.k1 = static_cast<uint32_t>(t.seed >> 32);
        b.row0 = t.table_row0, b.root0 = t.root0, b.n_legs = t.n_legs, b.leg0 = t.leg0, b.n_obs = t.n_obs;
        b.obs0 = t.obs0, b.lf_rate = static_cast<R>(t.r - t.q);
        if (t.model == OB_MODEL_HESTON_QE) b.qe = make_qe_consts<R>(t.heston, t.r, t.q, rq.dt);
        b.has_coupon = t.coupon > 0.0 || t.coupon_barrier > 0.0;
        b.memory = t.memory, b.ki_daily = t.ki_daily;
        b.ln_cb = t.coupon_barrier > 0 ? static_cast<R>(std::log(t.coupon_barrier)) : R(-1e30);
        b.ln_ki = t.ki_barrier > 0 ? static_cast<R>(std::log(t.ki_barrier)) : R(-1e30);
        b.coupon = t.coupon, b.put_strike = t.put_strike, b.discount = t.discount;
        b.corr_root0 = t.corr_root0;
        for (int c = 0; c < n_carry; ++c) b.carry_df[c] = std::exp(-rq.carry_rate[c] * t.n_steps * rq.dt);
        const auto key = std::make_tuple(t.model == OB_MODEL_HESTON_QE, t.n_names, t.product);
        auto f = cls.find(key);
        if (f == cls.end()) {
            f = cls.emplace(key, static_cast<int>(classes.size())).first;
            BClass c;
            c.qe = std::get<0>(key), c.n = std::get<1>(key), c.product = std::get<2>(key);
            c.kernel = reinterpret_cast<const void*>(c.product == OB_PRODUCT_LADDER
                                                         ? pick_batch<R, OB_PRODUCT_LADDER>(c.qe, c.n)
                                                         : pick_batch<R, OB_PRODUCT_AUTOCALL>(c.qe, c.n));
            classes.push_back(c);
        }
        classes[f->second].trades.push_back(i);
        class_of_trade[i] = f->second;
    }
    d.trades = arena.put<BTrade<R>>(bt.data(), bt.size());
    for (auto& c : classes) {
        check_cuda(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        check_cuda(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming), "cudaEventCreate");
    }
    simulations();
}

template void Batch::build<float>(const ob_batch_request&);
template void Batch::build<double>(const ob_batch_request&);

// The simulations of each trade (sims_of) and their outputs: the base carries the base, spot and carry moves.
void Batch::simulations() {
    sim_of_trade.assign(n_trades, 0);
    sim_outs.clear();
    for (int i = 0; i < n_trades; ++i) {
        sim_of_trade[i] = static_cast<int>(sim_outs.size());
        for (int s = 0; s < sims_of(i); ++s) sim_outs.push_back(s == 0 ? 1 + n_spot + n_carry : 1);
    }
    n_sims = static_cast<int>(sim_outs.size());
    d_sim_outs = arena.put<int>(sim_outs.data(), sim_outs.size());
}

// Slots and items for per-class tiles. Items of a class go largest trade first, so that the persistent blocks end
// together. With only_class, the items of that class alone, and with max_sims > 0 of at most that many of its
// simulations, evenly spread over its largest-first order (the autotuner's sample).
void Batch::layout(BLayout& L, const std::vector<int>& tiles, int only_class, int max_sims) {
    L.arena.release();
    L.pt_items.clear(), L.pt_first.clear(), L.pt_count.clear(), L.pt_class.clear();
    L.tile_of_class = tiles;
    L.sim_tiles.assign(n_sims, 0), L.sim_slot.assign(n_sims, 0);
    L.n_slots = 0;
    std::vector<char> keep(n_sims, 1);
    if (only_class >= 0 && max_sims > 0) {
        std::vector<int> sims;
        std::vector<int> order = classes[only_class].trades;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return static_cast<double>(trades[a].n_steps) * trades[a].n_pairs >
                   static_cast<double>(trades[b].n_steps) * trades[b].n_pairs;
        });
        for (int t : order)
            for (int s = 0; s < sims_of(t); ++s) sims.push_back(sim_of_trade[t] + s);
        if (static_cast<int>(sims.size()) > max_sims) {
            std::fill(keep.begin(), keep.end(), 0);
            for (int k = 0; k < max_sims; ++k)
                keep[sims[static_cast<size_t>(static_cast<double>(k) * sims.size() / max_sims)]] = 1;
        }
    }
    for (int i = 0; i < n_trades; ++i) {
        const int tile = tiles[class_of_trade[i]];
        const int tl = static_cast<int>((trades[i].n_pairs + tile - 1) / tile);
        for (int s = 0; s < sims_of(i); ++s) {
            const int sim = sim_of_trade[i] + s;
            L.sim_slot[sim] = L.n_slots, L.sim_tiles[sim] = keep[sim] ? tl : 0;
            if (only_class < 0 || class_of_trade[i] == only_class) L.n_slots += L.sim_tiles[sim];
        }
    }
    L.d_sim_slot = L.arena.put<int>(L.sim_slot.data(), L.sim_slot.size());
    L.d_sim_tiles = L.arena.put<int>(L.sim_tiles.data(), L.sim_tiles.size());
    L.d_slots = L.arena.alloc<double>(static_cast<size_t>(std::max(1, L.n_slots)) * 2 * kBatchMaxOut);
    L.d_sums = L.arena.alloc<double>(static_cast<size_t>(n_sims) * kBatchMaxOut * 2);
    L.d_items.assign(classes.size(), nullptr), L.n_items.assign(classes.size(), 0), L.d_counter.assign(classes.size(), nullptr);
    int* counters = L.arena.alloc<int>(classes.size());
    for (size_t ci = 0; ci < classes.size(); ++ci) {
        L.d_counter[ci] = counters + ci;
        if (only_class >= 0 && static_cast<int>(ci) != only_class) continue;
        std::vector<int> order = classes[ci].trades;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return static_cast<double>(trades[a].n_steps) * trades[a].n_names * trades[a].n_pairs >
                   static_cast<double>(trades[b].n_steps) * trades[b].n_names * trades[b].n_pairs;
        });
        std::vector<int4> items;
        for (int t : order) {
            for (int s = 0; s < sims_of(t); ++s)
                for (int k = 0; k < L.sim_tiles[sim_of_trade[t] + s]; ++k)
                    items.push_back(make_int4(t, s, k, sim_of_trade[t] + s));
        }
        L.n_items[ci] = static_cast<int>(items.size());
        L.d_items[ci] = L.arena.put<int4>(items.data(), items.size());
    }
}

template <typename R>
void Batch::launch_class(const BLayout& L, int ci, cudaStream_t st, const int4* items, int n_items, int* counter,
                         int grid, int block) {
    BDev<R> d = dev<R>();
    d.tile = L.tile_of_class[ci];
    d.slots = L.d_slots;
    d.sim_slot = L.d_sim_slot;
    reinterpret_cast<BatchFn<R>>(const_cast<void*>(classes[ci].kernel))<<<grid, block, 0, st>>>(d, items, n_items,
                                                                                               counter);
}

void Batch::reduce(const BLayout& L, cudaStream_t st) {
    const long long warps = static_cast<long long>(n_sims) * kBatchMaxOut;
    batch_reduce<<<static_cast<unsigned>((warps * 32 + 255) / 256), 256, 0, st>>>(L.d_slots, L.d_sim_slot,
                                                                                 L.d_sim_tiles, d_sim_outs, n_sims,
                                                                                 L.d_sums);
}

// Every class's persistent kernel on its own stream, forked from and joined back to st, then the reduction: the
// body of the captured graph (or of a direct run).
void Batch::run_all(cudaStream_t st) {
    BLayout& L = main;
    check_cuda(cudaEventRecord(fork, st), "cudaEventRecord");
    for (size_t ci = 0; ci < classes.size(); ++ci) {
        BClass& c = classes[ci];
        check_cuda(cudaStreamWaitEvent(c.stream, fork, 0), "cudaStreamWaitEvent");
        check_cuda(cudaMemsetAsync(L.d_counter[ci], 0, sizeof(int), c.stream), "cudaMemsetAsync");
        const int per_sm = occupancy(c.kernel, c.block, 0);
        const int grid = std::max(1, std::min(L.n_items[ci], sms * std::max(1, per_sm)));
        if (precision == OB_FP32)
            launch_class<float>(L, static_cast<int>(ci), c.stream, L.d_items[ci], L.n_items[ci], L.d_counter[ci], grid,
                                c.block);
        else
            launch_class<double>(L, static_cast<int>(ci), c.stream, L.d_items[ci], L.n_items[ci], L.d_counter[ci], grid,
                                 c.block);
        check_cuda(cudaGetLastError(), "batch_kernel launch");
        check_cuda(cudaEventRecord(c.done, c.stream), "cudaEventRecord");
        check_cuda(cudaStreamWaitEvent(st, c.done, 0), "cudaStreamWaitEvent");
    }
    reduce(L, st);
    check_cuda(cudaGetLastError(), "batch_reduce launch");
    last_layout = &main;
}

// Time of a sample of one class's work (at most max_sims of its simulations) at a given tile and block, in ms: the
// autotuner's measure.
double Batch::time_class(int ci, int tile, int block, int max_sims) {
    BLayout L;
    std::vector<int> t = tiles();
    t[ci] = tile;
    layout(L, t, ci, max_sims);
    BClass& c = classes[ci];
    cudaEvent_t a, b;
    check_cuda(cudaEventCreate(&a), "cudaEventCreate");
    check_cuda(cudaEventCreate(&b), "cudaEventCreate");
    const int per_sm = occupancy(c.kernel, block, 0);
    const int grid = std::max(1, std::min(L.n_items[ci], sms * std::max(1, per_sm)));
    check_cuda(cudaMemsetAsync(L.d_counter[ci], 0, sizeof(int)), "cudaMemsetAsync");
    check_cuda(cudaEventRecord(a), "cudaEventRecord");
    if (precision == OB_FP32) launch_class<float>(L, ci, nullptr, L.d_items[ci], L.n_items[ci], L.d_counter[ci], grid, block);
    else launch_class<double>(L, ci, nullptr, L.d_items[ci], L.n_items[ci], L.d_counter[ci], grid, block);
    check_cuda(cudaGetLastError(), "batch_kernel launch");
    check_cuda(cudaEventRecord(b), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(b), "autotune");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a), cudaEventDestroy(b);
    return ms;
}

}  // namespace ob

struct ob_batch {
    ob::Batch impl;
};

extern "C" {

int ob_batch_create(const ob_batch_request* rq, int precision, ob_batch** batch) {
    return ob::guarded([&] {
        if (!rq || !batch) ob::invalid("null argument");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        *batch = nullptr;
        ob::check_batch(*rq);
        auto* b = new ob_batch();
        try {
            b->impl.sms = ob::require_device();
            b->impl.precision = precision;
            if (precision == OB_FP32) b->impl.build<float>(*rq);
            else b->impl.build<double>(*rq);
            ob::check_cuda(cudaEventCreate(&b->impl.e0), "cudaEventCreate");
            ob::check_cuda(cudaEventCreate(&b->impl.e1), "cudaEventCreate");
            ob::check_cuda(cudaEventCreateWithFlags(&b->impl.fork, cudaEventDisableTiming), "cudaEventCreate");
            b->impl.layout(b->impl.main, b->impl.tiles());
        } catch (...) {
            delete b;
            throw;
        }
        *batch = b;
    });
}

// The autotuner, by successive halving per class: every (tile, block) candidate is timed on a small sample of the
// class's work (kProbeSims simulations spread over its sizes), the kFinalists fastest again on a larger one
// (kTuneSims: enough pairs to fill the GPU several times over), each after one untimed launch, and the fastest kept;
// the shape the class had before is timed on the larger sample too, so that the class records what tuning gained.
// Past budget_ms the untried candidates are skipped.
int ob_batch_tune(ob_batch* batch, int budget_ms) {
    return ob::guarded([&] {
        if (!batch) ob::invalid("null batch");
        ob::Batch& b = batch->impl;
        if (b.exec) ob::invalid("tune before capture");
        constexpr int kProbeSims = 4, kTuneSims = 32, kFinalists = 3;
        const auto t0 = std::chrono::steady_clock::now();
        auto over = [&] {
            const double el = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return budget_ms > 0 && el > budget_ms;
        };
        const int tiles[] = {512, 1024, 2048, 4096, 8192, 16384};
        const int blocks[] = {128, 256};
        for (size_t ci = 0; ci < b.classes.size(); ++ci) {
            ob::BClass& c = b.classes[ci];
            const int k = static_cast<int>(ci);
            b.time_class(k, c.tile, c.block, kProbeSims);  // warm: module load, caches
            std::vector<std::pair<double, std::pair<int, int>>> probe;
            for (int tile : tiles)
                for (int block : blocks)
                    if (!over()) probe.push_back({b.time_class(k, tile, block, kProbeSims), {tile, block}});
            std::sort(probe.begin(), probe.end());
            const double before = b.time_class(k, c.tile, c.block, kTuneSims);
            double best = before;
            int bt = c.tile, bb = c.block;
            for (int f = 0; f < std::min<int>(kFinalists, static_cast<int>(probe.size())); ++f) {
                const auto [tile, block] = probe[f].second;
                const double ms = b.time_class(k, tile, block, kTuneSims);
                if (ms < best) best = ms, bt = tile, bb = block;
            }
            c.tile = bt, c.block = bb, c.untuned_ms = before, c.tuned_ms = best;
        }
        b.layout(b.main, b.tiles());
    });
}

int ob_batch_capture(ob_batch* batch, void* stream) {
    return ob::guarded([&] {
        if (!batch) ob::invalid("null batch");
        ob::Batch& b = batch->impl;
        cudaStream_t cap = static_cast<cudaStream_t>(stream);
        bool own = false;
        if (!cap) {
            ob::check_cuda(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "cudaStreamCreate");
            own = true;
        }
        if (b.exec) cudaGraphExecDestroy(b.exec), b.exec = nullptr;
        if (b.graph) cudaGraphDestroy(b.graph), b.graph = nullptr;
        ob::check_cuda(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        try {
            b.run_all(cap);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(cap, &g);
            if (g) cudaGraphDestroy(g);
            if (own) cudaStreamDestroy(cap);
            throw;
        }
        ob::check_cuda(cudaStreamEndCapture(cap, &b.graph), "cudaStreamEndCapture");
        ob::check_cuda(cudaGraphInstantiate(&b.exec, b.graph, 0), "cudaGraphInstantiate");
        if (own) cudaStreamDestroy(cap);
    });
}

int ob_batch_launch(ob_batch* batch, void* stream) {
    return ob::guarded([&] {
        if (!batch) ob::invalid("null batch");
        ob::Batch& b = batch->impl;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        ob::check_cuda(cudaEventRecord(b.e0, st), "cudaEventRecord");
        if (b.exec) ob::check_cuda(cudaGraphLaunch(b.exec, st), "cudaGraphLaunch");
        else b.run_all(st);
        ob::check_cuda(cudaEventRecord(b.e1, st), "cudaEventRecord");
        b.last = st, b.last_layout = &b.main;
    });
}

// The comparison: the same simulations as one launch each (one pair per thread, one-block tiles of 256 pairs, the
// grid the simulation's tiles), in trade order on one stream, as a per-trade loop issues them.
int ob_batch_run_per_trade(ob_batch* batch, void* stream) {
    return ob::guarded([&] {
        if (!batch) ob::invalid("null batch");
        ob::Batch& b = batch->impl;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        ob::BLayout& L = b.per_trade;
        if (L.tile_of_class.empty()) b.layout(L, std::vector<int>(b.classes.size(), 256));
        if (L.pt_items.empty()) {
            std::vector<int4> items;
            for (int t = 0; t < b.n_trades; ++t) {
                for (int s = 0; s < b.sims_of(t); ++s) {
                    const int sim = b.sim_of_trade[t] + s;
                    L.pt_first.push_back(static_cast<int>(items.size()));
                    L.pt_count.push_back(L.sim_tiles[sim]);
                    L.pt_class.push_back(b.class_of_trade[t]);
                    for (int k = 0; k < L.sim_tiles[sim]; ++k) items.push_back(make_int4(t, s, k, sim));
                }
            }
            L.pt_items = items;
            L.d_pt_items = L.arena.put<int4>(items.data(), items.size());
            L.d_pt_counters = L.arena.alloc<int>(L.pt_first.size());
        }
        ob::check_cuda(cudaMemsetAsync(L.d_pt_counters, 0, L.pt_first.size() * sizeof(int), st), "cudaMemsetAsync");
        ob::check_cuda(cudaEventRecord(b.e0, st), "cudaEventRecord");
        for (size_t k = 0; k < L.pt_first.size(); ++k) {
            if (b.precision == OB_FP32)
                b.launch_class<float>(L, L.pt_class[k], st, L.d_pt_items + L.pt_first[k], L.pt_count[k],
                                      L.d_pt_counters + k, L.pt_count[k], 256);
            else
                b.launch_class<double>(L, L.pt_class[k], st, L.d_pt_items + L.pt_first[k], L.pt_count[k],
                                       L.d_pt_counters + k, L.pt_count[k], 256);
        }
        ob::check_cuda(cudaGetLastError(), "batch_kernel launch");
        b.reduce(L, st);
        ob::check_cuda(cudaEventRecord(b.e1, st), "cudaEventRecord");
        b.last = st, b.last_layout = &L;
    });
}

int ob_batch_result(ob_batch* batch, double* price, double* se, double* device_ms) {
    return ob::guarded([&] {
        if (!batch || !price || !se) ob::invalid("null argument");
        ob::Batch& b = batch->impl;
        if (!b.last_layout) ob::invalid("the batch has not run");
        ob::check_cuda(cudaStreamSynchronize(b.last), "batch");
        std::vector<double> sums(static_cast<size_t>(b.n_sims) * ob::kBatchMaxOut * 2);
        ob::check_cuda(cudaMemcpy(sums.data(), b.last_layout->d_sums, sums.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost),
                       "copy");
        const int per = 1 + b.n_spot + b.n_carry + b.n_vol + b.n_corr;
        for (int t = 0; t < b.n_trades; ++t) {
            const double n = static_cast<double>(b.trades[t].n_pairs);
            auto est = [&](int sim, int o, double& m, double& s) {
                const double s1 = sums[(static_cast<size_t>(sim) * ob::kBatchMaxOut + o) * 2];
                const double s2 = sums[(static_cast<size_t>(sim) * ob::kBatchMaxOut + o) * 2 + 1];
                m = s1 / n;
                s = n > 1 ? std::sqrt(std::fmax(s2 / n - m * m, 0.0) / (n - 1.0)) : 0.0;
            };
            const int s0 = b.sim_of_trade[t], n_sim = b.sims_of(t);
            const int on_base = 1 + b.n_spot + b.n_carry;
            for (int o = 0; o < on_base; ++o) est(s0, o, price[t * per + o], se[t * per + o]);
            // vol then correlation moves: their own simulations, or the base where the trade does not move
            for (int v = 0; v < b.n_vol + b.n_corr; ++v) {
                double& p = price[t * per + on_base + v];
                double& e = se[t * per + on_base + v];
                if (1 + v < n_sim) est(s0 + 1 + v, 0, p, e);
                else p = price[t * per], e = se[t * per];
            }
        }
        if (device_ms) {
            float ms = 0.0f;
            ob::check_cuda(cudaEventElapsedTime(&ms, b.e0, b.e1), "cudaEventElapsedTime");
            *device_ms = ms;
        }
    });
}

int ob_batch_classes(const ob_batch* batch, int max_classes, int* n_classes, int* info) {
    return ob::guarded([&] {
        if (!batch || !n_classes) ob::invalid("null argument");
        const ob::Batch& b = batch->impl;
        *n_classes = static_cast<int>(b.classes.size());
        for (int k = 0; k < std::min(max_classes, *n_classes) && info; ++k) {
            const ob::BClass& c = b.classes[k];
            int* o = info + 8 * k;
            o[0] = c.qe ? OB_MODEL_HESTON_QE : OB_MODEL_PATHS, o[1] = c.n, o[2] = c.product;
            o[3] = static_cast<int>(c.trades.size()), o[4] = c.tile, o[5] = c.block;
            o[6] = static_cast<int>(c.untuned_ms * 1e3 + 0.5), o[7] = static_cast<int>(c.tuned_ms * 1e3 + 0.5);
        }
    });
}

int ob_batch_destroy(ob_batch* batch) {
    return ob::guarded([&] { delete batch; });
}

}  // extern "C"
