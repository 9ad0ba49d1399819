// Fused Monte Carlo pricing: path, payoff and the FP64 sums of the pair averages in one kernel.
//
// Replaces, for the products it covers, the reference's chain "paths to the host, then NumPy evaluation"
// (packages/structured/src/optlab/structured/engine.py:143-153,260-330) and its fixed-product kernel
// (RC/src/gpu_mc.cu:116-145). Models: the log-Euler path engine of paths.hpp (model.cuh) or Andersen's QE-M for one
// Heston name. Products: a ladder of payoffs at maturity with optional barriers monitored at every step end, or an
// autocall (Phoenix, single or worst-of) with coupon memory and a knock-in put; the product semantics are those of the
// term-sheet compiler (packages/structured/src/optlab/structured/compiler.py:37-59,114-161,271-280) and of
// packages/core/src/optlab/core/products.py:82-102 for barriers.
//
// Layout: everything a path reads per step (time steps, table rows of each step, log-forwards, observation index
// of each step, product constants) is packed on the host into one "blob", staged into shared memory once per block,
// and read there as warp-wide broadcasts; the local-variance table joins it when it fits (the 40 x 200 grid of the
// local-vol benchmark is 32 KB in float). One thread carries both legs of one pair in registers; pairs are handed out
// grid-stride to a grid sized to fill every SM once. Each warp reduces its pair averages by shuffles into per-warp
// FP64 accumulators in shared memory; each block writes its totals, and a one-block kernel adds the blocks in order,
// so a result is bit-reproducible for a given launch shape.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <vector>

#include "mc.cuh"

namespace ob {

namespace {

template <typename R>
struct McView {
    const R* dt;
    const R* root;
    const int* kind;
    const R* cvar;
    const R* hes;
    const int* step_row;
    const R* lo;
    const R* inv_dx;
    const R* lf;
    const int* obs_of_step;
    const R* ln_trig;
    const double* obs_disc;
    const int* leg_type;
    const R* leg_strike;
    const int* leg_barrier;
    const R* ln_level;
    const R* table;
};

template <typename R>
__device__ __forceinline__ McView<R> view_of(const McArgs<R>& a, const unsigned char* base, const R* table) {
    McView<R> v;
    v.dt = reinterpret_cast<const R*>(base + a.off.dt);
    v.root = reinterpret_cast<const R*>(base + a.off.root);
    v.kind = reinterpret_cast<const int*>(base + a.off.kind);
    v.cvar = reinterpret_cast<const R*>(base + a.off.cvar);
    v.hes = reinterpret_cast<const R*>(base + a.off.hes);
    v.step_row = reinterpret_cast<const int*>(base + a.off.step_row);
    v.lo = reinterpret_cast<const R*>(base + a.off.lo);
    v.inv_dx = reinterpret_cast<const R*>(base + a.off.inv_dx);
    v.lf = reinterpret_cast<const R*>(base + a.off.lf);
    v.obs_of_step = reinterpret_cast<const int*>(base + a.off.obs_of_step);
    v.ln_trig = reinterpret_cast<const R*>(base + a.off.ln_trig);
    v.obs_disc = reinterpret_cast<const double*>(base + a.off.obs_disc);
    v.leg_type = reinterpret_cast<const int*>(base + a.off.leg_type);
    v.leg_strike = reinterpret_cast<const R*>(base + a.off.leg_strike);
    v.leg_barrier = reinterpret_cast<const int*>(base + a.off.leg_barrier);
    v.ln_level = reinterpret_cast<const R*>(base + a.off.ln_level);
    v.table = table;
    return v;
}

// What one leg remembers of its path for the product.
template <typename R>
struct Book {
    R hi, lo;     // ladder: extremes of ln(U / spot0) over the step ends
    R low;        // autocall: lowest ln(worst perf) over the step ends
    double pv;    // autocall: discounted cash flows
    float called, knocked, coupons;
    int missed;
    bool alive;
};

template <typename R>
__device__ __forceinline__ void book_init(Book<R>& b) {
    b.hi = R(-1e30), b.lo = R(1e30), b.low = R(0), b.pv = 0.0;
    b.called = b.knocked = b.coupons = 0.0f, b.missed = 0, b.alive = true;
}

// One step end of one leg: lp = ln of the basket performance (worst of S_a / S0_a) at step i.
template <typename R, int PRODUCT>
__device__ __forceinline__ void book_step(const McArgs<R>& a, const McView<R>& v, Book<R>& b, R lp, int i) {
    if (PRODUCT == OB_PRODUCT_LADDER) {
        b.hi = m_max(b.hi, lp), b.lo = m_min(b.lo, lp);
        return;
    }
    b.low = m_min(b.low, lp);
    const int j = v.obs_of_step[i];
    if (j < 0 || !b.alive) return;
    const double D = v.obs_disc[j];
    const bool last = j == a.n_obs - 1;
    if (a.has_coupon) {
        if (lp >= a.ln_cb) {
            const int k = a.memory ? 1 + b.missed : 1;
            b.pv += D * a.coupon * k, b.coupons += static_cast<float>(k), b.missed = 0;
        } else {
            ++b.missed;
        }
    }
    if (!last) {
        if (lp >= v.ln_trig[j]) b.pv += D, b.called = 1.0f, b.alive = false;
    } else {
        const bool ki = a.ki_daily ? b.low < a.ln_ki : lp < a.ln_ki;
        const double perf = static_cast<double>(m_exp(lp));
        const double put = a.put_strike - perf > 0.0 ? a.put_strike - perf : 0.0;
        b.pv += D * (ki ? 1.0 - put : 1.0), b.knocked = ki ? 1.0f : 0.0f, b.alive = false;
    }
}

// Output k of one leg at maturity (lp_T: ln perf at the last step).
template <typename R, int PRODUCT>
__device__ __forceinline__ double book_output(const McArgs<R>& a, const McView<R>& v, const Book<R>& b, R lp_T,
                                              int k) {
    if (PRODUCT == OB_PRODUCT_AUTOCALL) {
        return k == 0 ? b.pv : k == 1 ? b.called : k == 2 ? b.knocked : b.coupons;
    }
    const R U = a.spot0 * m_exp(lp_T);
    if (k == a.n_legs) return static_cast<double>(U);
    const int type = v.leg_type[k];
    const R K = v.leg_strike[k];
    R pay = type == 1 ? m_max(U - K, R(0)) : type == 2 ? m_max(K - U, R(0)) : type == 3 ? U - K : R(0);
    const int bt = v.leg_barrier[k];
    const R H = v.ln_level[k];
    const bool up = b.hi >= H, down = b.lo <= H;
    if ((bt == OB_BARRIER_UP_OUT && up) || (bt == OB_BARRIER_DOWN_OUT && down) || (bt == OB_BARRIER_UP_IN && !up) ||
        (bt == OB_BARRIER_DOWN_IN && !down))
        pay = R(0);
    return a.discount * static_cast<double>(pay);
}

template <typename R, int N, int MODEL, int PRODUCT>
__global__ void __launch_bounds__(256) mc_kernel(McArgs<R> a, long long n_pairs, long long first_pair, uint32_t k0,
                                                 uint32_t k1, double* __restrict__ partial) {
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
    const R* table = a.table_in_smem ? reinterpret_cast<const R*>(sm + a.off.table) : a.table_global;
    const McView<R> v = view_of(a, sm, table);

    ModelDev<R> m;
    m.n_names = a.n_names, m.n_steps = a.n_steps, m.n_x = a.n_x, m.same = a.same, m.mixer = a.mixer;
    m.has_var = a.has_var, m.has_slv = a.has_slv, m.k0 = k0, m.k1 = k1;
    m.dt = v.dt, m.root = v.root, m.kind = v.kind, m.cvar = v.cvar, m.hes = v.hes;
    m.step_row = v.step_row, m.lo = v.lo, m.inv_dx = v.inv_dx, m.table = v.table;
    m.t0 = a.mixer ? reinterpret_cast<const R*>(sm + a.off.t0) : nullptr;
    m.low_root = a.mixer ? reinterpret_cast<const R*>(sm + a.off.low_root) : nullptr;
#pragma unroll
    for (int k = 0; k < 8; ++k) m.mix[k] = a.mix[k];

    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    const int S = a.n_steps;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < n_pairs;
         base += stride) {
        const bool active = base + lane < n_pairs;
        const long long p = active ? base + lane : n_pairs - 1;
        const uint64_t pair = static_cast<uint64_t>(first_pair + p);
        Book<R> b0, b1;
        book_init(b0), book_init(b1);
        R lp0 = R(0), lp1 = R(0);
        if (MODEL == OB_MODEL_HESTON_QE) {
            NormalStream<R> rng;
            rng.init(pair, k0, k1, 0u);
            R y0 = R(0), y1 = R(0), v0 = a.qe.v0, v1 = a.qe.v0;
            for (int i = 1; i <= S; ++i) {
                const R zv = rng.next(), zx = rng.next();
                qe_step(a.qe, y0, v0, zv, zx);
                qe_step(a.qe, y1, v1, -zv, -zx);
                book_step<R, PRODUCT>(a, v, b0, y0, i);
                book_step<R, PRODUCT>(a, v, b1, y1, i);
            }
            lp0 = y0, lp1 = y1;
        } else {
            PairDev<R, N> st;
            pair_init<R, N>(m, st, pair);
            for (int i = 1; i <= S; ++i) {
                pair_step<R, N>(m, st, i);
                R w0 = R(1e30), w1 = R(1e30);
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    if (n >= a.n_names) continue;
                    const R f = v.lf[n * (S + 1) + i];
                    w0 = m_min(w0, st.x[0][n] + f), w1 = m_min(w1, st.x[1][n] + f);
                }
                book_step<R, PRODUCT>(a, v, b0, w0, i);
                book_step<R, PRODUCT>(a, v, b1, w1, i);
                lp0 = w0, lp1 = w1;
            }
        }
        for (int k = 0; k < a.n_out; ++k) {
            const double y = active ? 0.5 * (book_output<R, PRODUCT>(a, v, b0, lp0, k) +
                                             book_output<R, PRODUCT>(a, v, b1, lp1, k))
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

// Adds the blocks' totals to the plan's running sums: one warp per sum, lane l adding blocks l, l + 32, ... and the
// lanes combined by a fixed shuffle tree, so the order (and the result) depends only on the grid.
// The blocks' partial sums of one run into the plan's sums: added to them (add), or replacing them on the first run
// after a result was read (so the sums need no clearing between calls).
__global__ void mc_finalize(const double* __restrict__ partial, int n_blocks, int n_acc, double* sums, int add) {
    const int lane = threadIdx.x & 31;
    for (int t = threadIdx.x >> 5; t < n_acc; t += blockDim.x >> 5) {
        double s = 0.0;
        for (int b = lane; b < n_blocks; b += 32) s += partial[static_cast<long long>(b) * n_acc + t];
        s = warp_sum(s);
        if (lane == 0) sums[t] = add ? sums[t] + s : s;
    }
}

template <typename R>
using KernelFn = void (*)(McArgs<R>, long long, long long, uint32_t, uint32_t, double*);

template <typename R, int PRODUCT>
KernelFn<R> pick_paths(int n) {
    if (n <= 1) return mc_kernel<R, 1, OB_MODEL_PATHS, PRODUCT>;
    if (n <= 2) return mc_kernel<R, 2, OB_MODEL_PATHS, PRODUCT>;
    if (n <= 4) return mc_kernel<R, 4, OB_MODEL_PATHS, PRODUCT>;
    return mc_kernel<R, 8, OB_MODEL_PATHS, PRODUCT>;
}

template <typename R>
KernelFn<R> pick(int model, int product, int n) {
    if (model == OB_MODEL_HESTON_QE)
        return product == OB_PRODUCT_LADDER ? mc_kernel<R, 1, OB_MODEL_HESTON_QE, OB_PRODUCT_LADDER>
                                            : mc_kernel<R, 1, OB_MODEL_HESTON_QE, OB_PRODUCT_AUTOCALL>;
    return product == OB_PRODUCT_LADDER ? pick_paths<R, OB_PRODUCT_LADDER>(n) : pick_paths<R, OB_PRODUCT_AUTOCALL>(n);
}

// Host-side packing of the blob, in R, 16-byte aligned segments.
struct Packer {
    std::vector<unsigned char> bytes;
    int put_raw(const void* p, size_t n) {
        const size_t at = (bytes.size() + 15) & ~static_cast<size_t>(15);
        bytes.resize(at + ((n + 15) & ~static_cast<size_t>(15)), 0);
        if (p && n) std::memcpy(bytes.data() + at, p, n);
        return static_cast<int>(at);
    }
    template <typename T, typename S>
    int put(const S* src, size_t count) {
        std::vector<T> tmp(count);
        for (size_t i = 0; i < count; ++i) tmp[i] = static_cast<T>(src ? src[i] : S(0));
        return put_raw(tmp.data(), count * sizeof(T));
    }
    template <typename T>
    int put_vec(const std::vector<T>& v) {
        return put_raw(v.data(), v.size() * sizeof(T));
    }
};

}  // namespace

void check_mc_model(const ob_mc_request& rq) {
    if (rq.model != OB_MODEL_PATHS && rq.model != OB_MODEL_HESTON_QE) invalid("model must be 0 or 1");
    if (rq.n_names < 1 || rq.n_names > OB_MAX_NAMES) invalid("n_names must be 1 to 8");
    if (rq.model == OB_MODEL_HESTON_QE && rq.n_names != 1) invalid("the QE model has one name");
    if (rq.n_pairs < 2 || rq.first_pair < 0) invalid("n_pairs must be >= 2 and first_pair >= 0");
    if (rq.n_steps < 1 || !rq.dt || !rq.t0 || !rq.spot) invalid("null time grid or spot");
    if (rq.model == OB_MODEL_PATHS) {
        if (!rq.root || !rq.kind || !rq.cvar || !rq.heston || !rq.log_fwd) invalid("null array");
        for (int a = 0; a < rq.n_names; ++a) {
            const int k = rq.kind[a];
            if (k < 0 || k > 3) invalid("kind must be 0 to 3");
            if ((k == 2 || k == 3) && !(rq.heston[a * 5 + 1] > 0 && rq.heston[a * 5 + 2] > 0 &&
                                        rq.heston[a * 5 + 3] >= 0 && std::fabs(rq.heston[a * 5 + 4]) <= 1))
                invalid("Heston parameters out of range");
            if (k == 1 || k == 3) {
                if (rq.n_x < 2 || rq.n_rows < 1 || !rq.step_row || !rq.table || !rq.row_lo || !rq.row_inv_dx)
                    invalid("a tabulated variance needs n_x >= 2, rows and step_row");
                for (int i = 0; i < rq.n_steps; ++i)
                    if (rq.step_row[a * rq.n_steps + i] < 0 || rq.step_row[a * rq.n_steps + i] >= rq.n_rows)
                        invalid("step_row out of range");
            }
        }
        // requests.cpp:89 (the paths request's check, the same message)
        if (rq.mixer && (rq.mixer != 1 || !rq.low_root || !(rq.mix[4] > 0))) invalid("bad local correlation");
    } else {
        if (rq.mixer) invalid("bad local correlation");
        if (!rq.heston) invalid("null heston");
        const double* h = rq.heston;
        if (!(h[0] >= 0 && h[1] > 0 && h[2] > 0 && h[3] > 0 && std::fabs(h[4]) <= 1))
            invalid("Heston parameters out of range");
        for (int i = 1; i < rq.n_steps; ++i)
            if (std::fabs(rq.dt[i] - rq.dt[0]) > 1e-9 * rq.dt[0]) invalid("the QE model needs uniform steps");
    }
}

void check_mc_request(const ob_mc_request& rq) {
    check_mc_model(rq);
    if (rq.product == OB_PRODUCT_LADDER) {
        if (rq.n_legs < 1 || rq.n_legs > OB_MAX_OUT - 1 || !rq.leg_type || !rq.leg_strike)
            invalid("ladder: n_legs must be 1 to 31 with leg_type and leg_strike");
        for (int k = 0; k < rq.n_legs; ++k) {
            if (rq.leg_type[k] < 0 || rq.leg_type[k] > 3) invalid("leg_type must be 0 to 3");
            const int bt = rq.leg_barrier ? rq.leg_barrier[k] : 0;
            if (bt < 0 || bt > 4) invalid("leg_barrier must be 0 to 4");
            if (bt && !(rq.leg_level && rq.leg_level[k] > 0)) invalid("a barrier leg needs a positive level");
        }
    } else if (rq.product == OB_PRODUCT_AUTOCALL) {
        if (rq.n_obs < 1 || !rq.obs_step || !rq.obs_discount || !rq.trigger) invalid("autocall: null schedule");
        for (int j = 0; j < rq.n_obs; ++j)
            if (rq.obs_step[j] < 1 || rq.obs_step[j] > rq.n_steps || (j && rq.obs_step[j] <= rq.obs_step[j - 1]))
                invalid("obs_step must be increasing in [1, n_steps]");
        if (!(rq.ki_barrier >= 0) || !(rq.coupon_barrier >= 0)) invalid("barriers must be >= 0");
    } else {
        invalid("product must be 0 or 1");
    }
}

template <typename R>
void McPlan::build(const ob_mc_request& rq) {
    if (!force_generic && fused_build<R>(*this, rq)) return;
    const int n = rq.n_names, S = rq.n_steps;
    McArgs<R>& a = args<R>();
    a = McArgs<R>{};
    a.n_names = n, a.n_steps = S, a.n_x = rq.n_x, a.same = rq.same;
    a.n_obs = rq.product == OB_PRODUCT_AUTOCALL ? rq.n_obs : 0;
    a.n_legs = rq.product == OB_PRODUCT_LADDER ? rq.n_legs : 0;
    a.n_out = rq.product == OB_PRODUCT_LADDER ? rq.n_legs + 1 : 4;
    n_out = a.n_out;
    bool table = false;
    for (int k = 0; rq.model == OB_MODEL_PATHS && k < n; ++k) {
        a.has_var |= rq.kind[k] == 2 || rq.kind[k] == 3;
        a.has_slv |= rq.kind[k] == 3;
        table |= rq.kind[k] == 1 || rq.kind[k] == 3;
    }
    Packer pk;
    a.off.dt = pk.put<R>(rq.dt, S);
    if (rq.model == OB_MODEL_PATHS) {
        a.off.root = pk.put<R>(rq.root, static_cast<size_t>(n) * n);
        a.off.kind = pk.put<int>(rq.kind, n);
        a.off.cvar = pk.put<R>(rq.cvar, n);
        a.off.hes = pk.put<R>(rq.heston, 5 * static_cast<size_t>(n));
        a.off.lf = pk.put<R>(rq.log_fwd, static_cast<size_t>(n) * (S + 1));
        if (table) {
            a.off.step_row = pk.put<int>(rq.step_row, static_cast<size_t>(n) * S);
            a.off.lo = pk.put<R>(rq.row_lo, rq.n_rows);
            a.off.inv_dx = pk.put<R>(rq.row_inv_dx, rq.n_rows);
        }
        if (rq.mixer) {
            a.mixer = 1;
            a.off.t0 = pk.put<R>(rq.t0, S);
            a.off.low_root = pk.put<R>(rq.low_root, static_cast<size_t>(n) * n);
            for (int k = 0; k < 8; ++k) a.mix[k] = static_cast<R>(rq.mix[k]);
        }
    } else {
        a.qe = make_qe_consts<R>(rq.heston, rq.r, rq.q, rq.dt[0]);
    }
    a.spot0 = static_cast<R>(rq.spot[0]);
    if (rq.product == OB_PRODUCT_LADDER) {
        std::vector<R> lvl(rq.n_legs, R(0));
        std::vector<int> bar(rq.n_legs, 0);
        for (int k = 0; k < rq.n_legs; ++k) {
            bar[k] = rq.leg_barrier ? rq.leg_barrier[k] : 0;
            lvl[k] = bar[k] ? static_cast<R>(std::log(rq.leg_level[k] / rq.spot[0])) : R(0);
        }
        a.off.leg_type = pk.put<int>(rq.leg_type, rq.n_legs);
        a.off.leg_strike = pk.put<R>(rq.leg_strike, rq.n_legs);
        a.off.leg_barrier = pk.put_vec(bar);
        a.off.ln_level = pk.put_vec(lvl);
        a.discount = rq.discount;
    } else {
        std::vector<int> obs_of(S + 1, -1);
        std::vector<R> trig(rq.n_obs);
        for (int j = 0; j < rq.n_obs; ++j) {
            obs_of[rq.obs_step[j]] = j;
            trig[j] = rq.trigger[j] > 0 ? static_cast<R>(std::log(rq.trigger[j])) : R(1e30);
        }
        a.off.obs_of_step = pk.put_vec(obs_of);
        a.off.ln_trig = pk.put_vec(trig);
        a.off.obs_disc = pk.put<double>(rq.obs_discount, rq.n_obs);
        a.has_coupon = rq.coupon > 0.0 || rq.coupon_barrier > 0.0;
        a.ln_cb = rq.coupon_barrier > 0 ? static_cast<R>(std::log(rq.coupon_barrier)) : R(-1e30);
        a.ln_ki = rq.ki_barrier > 0 ? static_cast<R>(std::log(rq.ki_barrier)) : R(-1e30);
        a.coupon = rq.coupon, a.put_strike = rq.put_strike, a.memory = rq.memory, a.ki_daily = rq.ki_daily;
    }
    a.smem_blob = static_cast<int>((pk.bytes.size() + 15) & ~static_cast<size_t>(15));
    // The table goes into shared memory with the rest when the whole stays within 160 KB.
    const size_t table_bytes = table ? static_cast<size_t>(rq.n_rows) * rq.n_x * sizeof(R) : 0;
    const size_t acc_bytes = 8 * sizeof(double) * 2 * static_cast<size_t>(a.n_out);  // 8 warps
    a.table_in_smem = table && pk.bytes.size() + table_bytes + acc_bytes <= (160u << 10);
    if (a.table_in_smem) {
        a.off.table = pk.put<R>(rq.table, static_cast<size_t>(rq.n_rows) * rq.n_x);
        a.smem_blob = static_cast<int>((pk.bytes.size() + 15) & ~static_cast<size_t>(15));
    }
    if (static_cast<size_t>(a.smem_blob) + acc_bytes > (200u << 10)) invalid("request too large for shared memory");
    unsigned char* dblob = arena.alloc<unsigned char>(std::max<size_t>(16, pk.bytes.size()));
    check_cuda(cudaMemcpy(dblob, pk.bytes.data(), pk.bytes.size(), cudaMemcpyHostToDevice), "copy blob");
    a.blob = dblob;
    if (table && !a.table_in_smem) a.table_global = arena.put<R>(rq.table, static_cast<size_t>(rq.n_rows) * rq.n_x);
    smem_bytes = static_cast<size_t>(a.smem_blob) + acc_bytes;
    kernel = reinterpret_cast<const void*>(pick<R>(rq.model, rq.product, n));
    allow_smem(kernel, smem_bytes);
    blocks_per_sm = std::max(1, occupancy(kernel, block, smem_bytes));
}

template void McPlan::build<float>(const ob_mc_request&);
template void McPlan::build<double>(const ob_mc_request&);

void McPlan::create(const ob_mc_request& rq, int prec) {
    check_mc_request(rq);
    const char* generic = std::getenv("OPTLAB_B200_GENERIC");  // 1: the generic kernel even where fused.cu applies
    force_generic = generic && generic[0] == '1';
    sms = require_device();
    precision = prec;
    if (prec == OB_FP32) build<float>(rq);
    else build<double>(rq);
    max_blocks = sms * 64;
    d_partial = arena.alloc<double>(static_cast<size_t>(max_blocks) * 2 * n_out);
    d_sums = arena.alloc<double>(2 * OB_MAX_OUT);  // written by the first run's finalize
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
}

McPlan::~McPlan() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
}

// Block size and grid of a run. Among the plan's block and its halves down to 64 threads, the shape that keeps the
// most warps resident on the most SMs: a small batch (2^15 pairs of the QE ladder) then spreads over every SM in
// small blocks, while a large one keeps 512-thread blocks. The grid fills each SM once with resident blocks and the
// pairs are handed out grid-stride.
int McPlan::occupancy_at(int blk) {
    if (blk == block) return blocks_per_sm;
    for (int k = 0; k < 16; ++k)
        if (occ_block[k] == blk) return occ_blocks[k];
    const int per_sm = std::max(1, occupancy(kernel, blk, smem_bytes));
    for (int k = 0; k < 16; ++k)
        if (!occ_block[k]) {
            occ_block[k] = blk, occ_blocks[k] = per_sm;
            break;
        }
    return per_sm;
}

// Block size and grid of a launch. A warp works through its pairs in chunks of 32 lanes, every chunk the whole path,
// so the run lasts ceil(chunks / resident warps) rounds: the block size is chosen (multiples of 32 up to the plan's
// block) to keep that ceiling close to the exact quotient, with enough warps on each SM to keep its schedulers
// issuing (kIssueWarps; fewer count as proportionally slower).
int McPlan::launch_shape(long long n_pairs, int& blk) {
    constexpr double kIssueWarps = 24.0;
    const long long units = n_pairs * threads_per_pair;
    const long long chunks = (units + 31) / 32;
    double best = -1.0;
    int best_blk = block;
    for (int b = block; b >= 64; b -= 32) {
        const long long need = (units + b - 1) / b;
        const long long grid = std::min<long long>(need, static_cast<long long>(sms) * occupancy_at(b));
        const long long warps = grid * (b / 32);
        const long long rounds = (chunks + warps - 1) / warps;
        const double fill = static_cast<double>(chunks) / static_cast<double>(rounds * warps);
        const double per_sm = static_cast<double>(warps) / sms;
        const double score = fill * std::min(1.0, per_sm / kIssueWarps) * std::min(1.0, static_cast<double>(grid) / sms);
        if (score > best * 1.0001) best = score, best_blk = b;
    }
    blk = best_blk;
    const long long need = (units + blk - 1) / blk;
    const long long full = static_cast<long long>(sms) * occupancy_at(blk) * grid_waves;
    return static_cast<int>(std::max<long long>(1, std::min<long long>({need, full, max_blocks})));
}

void McPlan::run(long long n_pairs, long long first_pair, unsigned long long seed, cudaStream_t st) {
    if (n_pairs < 1 || first_pair < 0) invalid("n_pairs must be >= 1 and first_pair >= 0");
    int blk = block;
    const int grid = launch_shape(n_pairs, blk);
    const uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
    if (!timing) check_cuda(cudaEventRecord(e0, st), "cudaEventRecord"), timing = true;
    using FusedF = void (*)(FusedArgs<float>, long long, long long, uint32_t, uint32_t, double*);
    using FusedD = void (*)(FusedArgs<double>, long long, long long, uint32_t, uint32_t, double*);
    void* fn = const_cast<void*>(kernel);
    if (fused && precision == OB_FP32)
        reinterpret_cast<FusedF>(fn)<<<grid, blk, smem_bytes, st>>>(fa_f, n_pairs, first_pair, k0, k1, d_partial);
    else if (fused)
        reinterpret_cast<FusedD>(fn)<<<grid, blk, smem_bytes, st>>>(fa_d, n_pairs, first_pair, k0, k1, d_partial);
    else if (precision == OB_FP32)
        reinterpret_cast<KernelFn<float>>(fn)<<<grid, blk, smem_bytes, st>>>(args_f, n_pairs, first_pair, k0, k1,
                                                                              d_partial);
    else
        reinterpret_cast<KernelFn<double>>(fn)<<<grid, blk, smem_bytes, st>>>(args_d, n_pairs, first_pair, k0, k1,
                                                                               d_partial);
    check_cuda(cudaGetLastError(), "mc_kernel launch");
    mc_finalize<<<1, 1024, 0, st>>>(d_partial, grid, 2 * n_out, d_sums, pairs_run > 0);
    check_cuda(cudaGetLastError(), "mc_finalize launch");
    check_cuda(cudaEventRecord(e1, st), "cudaEventRecord");
    pairs_run += n_pairs;
    last_stream = st;
}

void McPlan::result(ob_mc_result& res) {
    double h[2 * OB_MAX_OUT] = {};
    if (pairs_run > 0) {  // (no run since the last result: empty sums)
        // the sums through the small pinned buffer: an asynchronous copy on the runs' stream, then one wait
        static_assert(sizeof h <= kSmallPinnedBytes, "the sums fit the pinned buffer");
        double* pin = static_cast<double*>(small_pinned());
        check_cuda(cudaMemcpyAsync(pin ? pin : h, d_sums, sizeof h, cudaMemcpyDeviceToHost, last_stream),
                   "copy sums");
        check_cuda(cudaStreamSynchronize(last_stream), "mc_kernel");
        if (pin) std::memcpy(h, pin, sizeof h);
    }
    float ms = 0.0f;
    if (timing) check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    std::memset(&res, 0, sizeof res);
    res.n_out = n_out;
    res.n_paths = 2 * pairs_run;
    const double nn = static_cast<double>(pairs_run);
    for (int k = 0; k < n_out; ++k) {
        const double mean = h[k] / nn, var = h[n_out + k] / nn - mean * mean;
        res.price[k] = mean;
        res.se[k] = pairs_run > 1 ? std::sqrt(std::fmax(var, 0.0) / (nn - 1.0)) : 0.0;
        res.sum_y[k] = h[k], res.sum_y2[k] = h[n_out + k];
    }
    res.kernel_ms = ms;
    pairs_run = 0;
    timing = false;
}

}  // namespace ob

struct ob_mc_plan {
    ob::McPlan impl;
};

extern "C" {

int ob_mc_plan_create(const ob_mc_request* rq, int precision, ob_mc_plan** plan) {
    return ob::guarded([&] {
        if (!rq || !plan) ob::invalid("null argument");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        *plan = nullptr;
        ob_mc_plan* p = new ob_mc_plan();
        try {
            p->impl.create(*rq, precision);
        } catch (...) {
            delete p;
            throw;
        }
        *plan = p;
    });
}

int ob_mc_run(ob_mc_plan* plan, long long n_pairs, long long first_pair, unsigned long long seed, void* stream) {
    return ob::guarded([&] {
        if (!plan) ob::invalid("null plan");
        plan->impl.run(n_pairs, first_pair, seed, static_cast<cudaStream_t>(stream));
    });
}

int ob_mc_result_get(ob_mc_plan* plan, ob_mc_result* res) {
    return ob::guarded([&] {
        if (!plan || !res) ob::invalid("null argument");
        plan->impl.result(*res);
    });
}

int ob_mc_plan_destroy(ob_mc_plan* plan) {
    return ob::guarded([&] { delete plan; });
}

int ob_mc_price(const ob_mc_request* rq, int precision, ob_mc_result* res) {
    return ob::guarded([&] {
        if (!rq || !res) ob::invalid("null argument");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        const auto t0 = std::chrono::steady_clock::now();
        ob::McPlan p;
        p.arena.recycle = true;  // the call reads its result back (synchronises) before p goes
        p.create(*rq, precision);
        p.run(rq->n_pairs, rq->first_pair, rq->seed, nullptr);
        p.result(*res);
        res->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
}

}  // extern "C"
