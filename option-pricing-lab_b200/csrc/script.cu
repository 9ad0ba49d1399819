// Payoff scripts on the device: ob_script_price simulates a request's paths (the path engine's step of model.cuh, or
// Andersen QE for one Heston name) and runs a compiled payoff script on both legs of every pair at its event steps,
// then reduces the pair-averaged present values into a price and its standard error.
//
// The script is the reference's payoff language (packages/structured/src/optlab/structured/script/), compiled on
// the host (optlab_b200/script.py) into instructions over a register file: the reference evaluates it on arrays of
// paths with conditions as masks (evaluator.py:123-231): inside an `if`, an assignment is x = m e + (1 - m) x, a
// payment adds m alive e to the flows, `terminate` multiplies alive by 1 - m, and both branches are evaluated. Read
// per path, that is straight-line code, so every lane of a warp runs the same instruction stream: the interpreter
// does not diverge. Each leg has its own register file (constants, variables, temporaries) in local memory; the
// registers are touched only at event steps, a few dozen times a path, against hundreds of path steps.
//
// Windows (lowest, highest, realised variance of one name's fixings) are kept as running states updated at their
// fixing steps, so nothing of the path is stored. Paths whose script is undefined (a payment that is not finite, a
// condition that is NaN where it matters, redemption weights that do not add up to one) are counted and reported;
// the host raises them as the reference does.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "exercise.cuh"
#include "mc.cuh"

namespace ob {

namespace {

constexpr int kMaxRegs = 128;
constexpr int kMaxWindows = 8;  // windows held in registers (kernels for up to 2 and up to 8)
constexpr double kAnnual = 252.0;  // realised variance: fixings a year (varswap.py:24)
constexpr int kMaxState = 4;       // state variables of an issuer's call
constexpr int kMaxPoly = 25, kMaxKnots = 25;  // a rule's polynomial terms and hinges

enum ScriptOp : int {
    kSpot, kWin, kMov, kAdd, kSub, kMul, kDiv, kNeg, kMin, kMax, kAbs, kExp, kLog, kSqrt,
    kGe, kGt, kLe, kLt, kEq, kAnd, kOr, kNot, kAssign, kPay, kTerm, kCond, kCall, kNumOps
};

template <typename R>
struct ScriptDev {
    ModelDev<R> m;
    int model, n_names, n_steps;
    const R* lf;        // n_names x (n_steps + 1): ln(F(t_i) / spot)
    R spot0[OB_MAX_NAMES];
    QeConsts<R> qe;
    const int4* code;
    const double* consts;
    int n_const, n_regs;
    const int* event_at;        // n_steps + 1: event index of each step end, or -1
    const int* event_code;      // n_events + 1
    const double* event_disc;
    const unsigned* fix_mask;   // n_steps + 1: windows fixing at each step end
    int n_windows;
    const int* win_name;
    const int* win_func;
    const int* win_nfix;
    const double* win_lo;
    const double* win_hi;
    const R* win_spot0;
    R eps;
    double red_tol;
    unsigned long long* bad;    // 3 counters: payments, conditions, redemptions
    // the issuer's call
    int n_events, n_calls, n_state, call_mode, rec_stride;
    const int* call_state;      // n_calls x 4 registers
    const double* rules;        // n_calls x OB_RULE_STRIDE
    double* record;             // call_mode 1: 2 n_pairs x rec_stride
    // branched continuations: up to step end branch_step, pair p follows outer path p / branch_pairs of an outer
    // simulation of branch_outer pairs on the key (bk0, bk1)
    int branch_step;
    long long branch_outer, branch_pairs;
    uint32_t bk0, bk1;
    double* pair_value;         // n_pairs: each pair's average present value, or null
};

// One leg's state between events (its register file lives in local memory: it is touched only at events).
template <typename R>
struct LegState {
    R reg[kMaxRegs];
    R alive;
    double pv, red;
    bool bad_pay, bad_cond;
};

// One leg's windows, read and written only by loops unrolled over NW so that they stay in registers: they change at
// every fixing, which is every step for a daily window. v: the lowest / highest ln(S / spot0) so far, or (variance)
// the last one (NaN before the first fixing); s: the variance's sum of squared log returns in its corridor.
template <typename R, int NW>
struct WinState {
    R v[NW];
    double s[NW];
};

template <typename R>
__device__ __forceinline__ R compare(int op, R a, R b, R eps) {
    if (isnan(a) || isnan(b)) return a + b;  // NaN stays NaN
    const bool h = op == kGe ? a >= b : op == kGt ? a > b : op == kLe ? a <= b : op == kLt ? a < b : a == b;
    const R hard = h ? R(1) : R(0);
    if (eps == R(0) || op == kEq) return hard;
    const R scale = eps * m_abs(b);
    if (!(scale > R(0))) return hard;
    const R d = (op == kGe || op == kGt) ? a - b : b - a;
    return m_min(m_max(d / scale + R(0.5), R(0)), R(1));
}

// What the interpreter reads besides a leg's state, passed by value so that no state of the kernel's step loop has
// its address taken (the step loop keeps its paths and windows in registers).
template <typename R>
struct EvCtx {
    const int4* code;
    const int* win_func;
    const int* win_nfix;
    const R* win_spot0;  // the spot of each window's name at the valuation date
    R eps;
    int call_mode, n_state, n_events, k;  // k: the event
    const int* call_state;
    const double* rules;
    double* rec;         // this leg's record (call_mode 1), or null
};

// A fitted rule's continuation of the state (exercise: the polynomial terms, then the hinges max(z_v - knot, 0), on
// the state normalised by the rule's mean and scale).
__device__ double continuation(const double* rule, const double* state, int n_state) {
    const int n_poly = static_cast<int>(rule[1]), n_knots = static_cast<int>(rule[2]);
    double z[kMaxState];
#pragma unroll
    for (int j = 0; j < kMaxState; ++j) z[j] = j < n_state ? (state[j] - rule[3 + j]) / rule[7 + j] : 0.0;
    const double* coef = rule + 161;
    double cont = 0.0;
    for (int t = 0; t < n_poly; ++t) {
        double term = 1.0;
        for (int j = 0; j < n_state; ++j) {
            const int p = static_cast<int>(rule[11 + 4 * t + j]);
            for (int e = 0; e < p; ++e) term *= z[j];
        }
        cont += coef[t] * term;
    }
    for (int q = 0; q < n_knots; ++q) {
        const double h = z[static_cast<int>(rule[111 + q])] - rule[136 + q];
        cont += coef[n_poly + q] * (h > 0.0 ? h : 0.0);
    }
    return cont;
}

// The script's instructions of one event on one leg: sp[a] is the leg's spot of name a at this step, win a copy of
// the leg's windows. Out of line: it runs a few dozen times a path, and inlined it would crowd the step loop.
// CALLS: the script has issuer calls; without them the interpreter keeps no call bookkeeping, whose registers would
// spill in the dispatch loop of every script (a third slower on the Phoenix).
template <typename R, int NW, bool CALLS>
__device__ __noinline__ void run_event(EvCtx<R> d, LegState<R>& s, WinState<R, NW> win, const R* sp, int c0, int c1,
                                       double disc) {
    R* r = s.reg;
    bool after = false;  // past this event's call statement
    double pre = 0.0, post = 0.0;
    for (int pc = c0; pc < c1; ++pc) {
        const int4 in = __ldg(d.code + pc);
        const int dst = in.y, a = in.z, b = in.w;
        switch (in.x) {
            case kSpot: r[dst] = sp[a]; break;
            case kWin: {
                R v = R(0);
                double sum = 0.0;
#pragma unroll
                for (int w = 0; w < NW; ++w)
                    if (w == a) v = win.v[w], sum = win.s[w];
                r[dst] = d.win_func[a] == 2 ? static_cast<R>(kAnnual / static_cast<double>(d.win_nfix[a] - 1) * sum)
                                            : d.win_spot0[a] * m_exp(v);
                break;
            }
            case kMov: r[dst] = r[a]; break;
            case kAdd: r[dst] = r[a] + r[b]; break;
            case kSub: r[dst] = r[a] - r[b]; break;
            case kMul: r[dst] = r[a] * r[b]; break;
            case kDiv: r[dst] = r[a] / r[b]; break;
            case kNeg: r[dst] = -r[a]; break;
            case kMin: case kMax: {  // NaN propagates, as NumPy's minimum and maximum
                const R x = r[a], y = r[b];
                r[dst] = (isnan(x) || isnan(y)) ? x + y : (in.x == kMin ? (x < y ? x : y) : (x > y ? x : y));
                break;
            }
            case kAbs: r[dst] = m_abs(r[a]); break;
            case kExp: r[dst] = m_exp(r[a]); break;
            case kLog: r[dst] = m_log(r[a]); break;
            case kSqrt: r[dst] = m_sqrt(r[a]); break;
            case kGe: case kGt: case kLe: case kLt: case kEq: r[dst] = compare(in.x, r[a], r[b], d.eps); break;
            case kAnd: {  // a certain false operand decides, even where the other one is undefined
                const R x = r[a], y = r[b];
                r[dst] = (x == R(0) || y == R(0)) ? R(0) : x * y;
                break;
            }
            case kOr: {
                const R x = r[a], y = r[b];
                r[dst] = (x == R(1) || y == R(1)) ? R(1) : x + y - x * y;
                break;
            }
            case kNot: r[dst] = R(1) - r[a]; break;
            case kAssign: {
                const R m = r[b], e = r[a], old = r[dst];
                r[dst] = m == R(1) ? e : (m == R(0) ? old : m * e + (R(1) - m) * old);
                break;
            }
            case kPay: {
                const R w = r[b] * s.alive, e = r[a];
                if (w != R(0)) {
                    if (!isfinite(e)) {
                        s.bad_pay = true;
                    } else {
                        const double paid = disc * (static_cast<double>(w) * static_cast<double>(e));
                        s.pv += paid;
                        if (CALLS) {
                            if (after) post += paid;
                            else pre += paid;
                        }
                    }
                }
                if (dst == 2) s.red += static_cast<double>(w);
                break;
            }
            case kCall:
                if (CALLS) {
                    double st[kMaxState];
#pragma unroll
                    for (int j = 0; j < kMaxState; ++j)
                        st[j] = j < d.n_state ? static_cast<double>(r[d.call_state[4 * dst + j]]) : 0.0;
                    const R m = r[b], amt = r[a];
                    if (d.call_mode == 1 && d.rec) {
                        double* c = d.rec + 2 * d.n_events + dst * (3 + d.n_state);
                        c[0] = static_cast<double>(m), c[1] = static_cast<double>(s.alive);
                        c[2] = static_cast<double>(amt);
                        for (int j = 0; j < d.n_state; ++j) c[3 + j] = st[j];
                        after = true;
                    } else if (d.call_mode == 2) {
                        const double* rule = d.rules + static_cast<long long>(dst) * OB_RULE_STRIDE;
                        const bool call =
                            rule[0] != 0.0 && continuation(rule, st, d.n_state) > static_cast<double>(amt);
                        const R md = call ? m : R(0), w = md * s.alive;
                        if (w != R(0)) {
                            if (!isfinite(amt)) s.bad_pay = true;
                            else s.pv += disc * (static_cast<double>(w) * static_cast<double>(amt));
                        }
                        s.red += static_cast<double>(w);
                        s.alive = s.alive * (R(1) - md);
                    }
                }
                break;
            case kTerm: s.alive = s.alive * (R(1) - r[a]); break;
            case kCond: {
                R c = r[a];
                if (isnan(c)) {
                    if (r[b] * s.alive != R(0)) s.bad_cond = true;
                    c = R(0);
                }
                r[dst] = c;
                break;
            }
            default: break;
        }
    }
    if (CALLS && d.call_mode == 1 && d.rec) d.rec[2 * d.k] = pre, d.rec[2 * d.k + 1] = post;
}

// The windows fixing at this step, on one leg. logp(a): ln(S_a / spot0_a) of name a at this step. A window keeps the
// extreme (or, for the variance, the last) of ln(S / spot0): S is increasing in it, so the lowest and highest spots
// are spot0 exp(extreme), and the log returns are differences of it; no exp or log is taken at the fixings.
// Each window's function and name, packed (function | name << 2), loaded once a thread into registers.
template <int NW>
struct WinMeta {
    int fn[NW];
};

template <typename R, int NW>
__device__ __forceinline__ WinMeta<NW> win_meta(const ScriptDev<R>& d) {
    WinMeta<NW> m;
#pragma unroll
    for (int w = 0; w < NW; ++w) m.fn[w] = w < d.n_windows ? (d.win_func[w] | (d.win_name[w] << 2)) : 0;
    return m;
}

// WF >= 0: the script's one window is a lowest (0) or a highest (1), known when the kernel is compiled, so a fixing
// is one comparison; WF < 0: any windows, each fixing dispatched on its function.
template <int WF = -1, typename R, int NW, typename LogFn>
__device__ __forceinline__ void fix_windows(const ScriptDev<R>& d, const WinMeta<NW>& meta, WinState<R, NW>& win,
                                            unsigned mask, LogFn logp) {
    if constexpr (WF >= 0) {
        if (mask & 1u) {
            const R y = logp(meta.fn[0] >> 2);
            win.v[0] = WF == 0 ? m_min(win.v[0], y) : m_max(win.v[0], y);
        }
        return;
    }
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        if (!((mask >> w) & 1u)) continue;
        const int f = meta.fn[w] & 3;
        const R y = logp(meta.fn[w] >> 2);
        if (f == 0) {
            win.v[w] = m_min(win.v[w], y);
        } else if (f == 1) {
            win.v[w] = m_max(win.v[w], y);
        } else {
            const R prev = win.v[w];
            if (!isnan(prev)) {
                const double lo = d.win_lo[w], hi = d.win_hi[w], pd = static_cast<double>(prev);
                const bool inside = (isnan(lo) || pd >= lo) && (isnan(hi) || pd <= hi);
                const double rr = static_cast<double>(y - prev);
                if (inside) win.s[w] += rr * rr;
            }
            win.v[w] = y;
        }
    }
}

template <typename R>
__device__ __forceinline__ EvCtx<R> ev_ctx(const ScriptDev<R>& d, int k, double* rec) {
    EvCtx<R> c;
    c.code = d.code, c.win_func = d.win_func, c.win_nfix = d.win_nfix, c.win_spot0 = d.win_spot0, c.eps = d.eps;
    c.call_mode = d.call_mode, c.n_state = d.n_state, c.n_events = d.n_events, c.k = k;
    c.call_state = d.call_state, c.rules = d.rules, c.rec = rec;
    return c;
}

// The record of one leg of one pair (pair p's legs are paths p and n_pairs + p), or null.
template <typename R>
__device__ __forceinline__ double* leg_record(const ScriptDev<R>& d, long long p, long long n_pairs, int l,
                                              bool active) {
    if (d.call_mode != 1 || !active) return nullptr;
    return d.record + static_cast<long long>(d.rec_stride) * (l ? n_pairs + p : p);
}

template <typename R, int NW>
__device__ __forceinline__ void win_init(const ScriptDev<R>& d, WinState<R, NW>& win) {
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const int f = w < d.n_windows ? d.win_func[w] : 0;
        win.v[w] = f == 0 ? R(INFINITY) : (f == 1 ? R(-INFINITY) : R(NAN));
        win.s[w] = 0.0;
    }
}

template <typename R>
__device__ void leg_init(const ScriptDev<R>& d, LegState<R>& s) {
    for (int k = 0; k < d.n_regs; ++k) s.reg[k] = k < d.n_const ? static_cast<R>(d.consts[k]) : R(0);
    s.alive = R(1), s.pv = 0.0, s.red = 0.0, s.bad_pay = s.bad_cond = false;
}

template <typename R, int N, int MODEL, int NW>
__global__ void __launch_bounds__(128) script_kernel(ScriptDev<R> d, long long n_pairs, uint32_t k0, uint32_t k1,
                                                     double* __restrict__ partial) {
    __shared__ double wacc[4][2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    if (threadIdx.x < 8) (&wacc[0][0])[threadIdx.x] = 0.0;
    __syncthreads();
    ModelDev<R> m = d.m;
    m.k0 = k0, m.k1 = k1;
    const int S = d.n_steps;
    const WinMeta<NW> meta = win_meta<R, NW>(d);
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < n_pairs;
         base += stride) {
        const bool active = base + lane < n_pairs;
        const uint64_t pair = static_cast<uint64_t>(active ? base + lane : n_pairs - 1);
        LegState<R> leg[2];
        leg_init(d, leg[0]), leg_init(d, leg[1]);
        WinState<R, NW> win[2];
        win_init(d, win[0]), win_init(d, win[1]);
        PairDev<R, N> st;
        NormalStream<R> qrng;
        R y[2] = {R(0), R(0)}, v[2] = {d.qe.v0, d.qe.v0};
        if (MODEL == OB_MODEL_HESTON_QE) qrng.init(pair, k0, k1, 0u);
        else pair_init<R, N>(m, st, pair);
        for (int i = 0; i <= S; ++i) {
            if (i > 0) {
                if (MODEL == OB_MODEL_HESTON_QE) {
                    const R zv = qrng.next(), zx = qrng.next();
                    qe_step(d.qe, y[0], v[0], zv, zx);
                    qe_step(d.qe, y[1], v[1], -zv, -zx);
                } else {
                    pair_step<R, N>(m, st, i);
                }
            }
            const unsigned fm = d.fix_mask[i];
            const int ev = d.event_at[i];
            if (!fm && ev < 0) continue;
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                auto logp = [&](int a) -> R {
                    if (MODEL == OB_MODEL_HESTON_QE) return y[l];
                    R x = R(0);
#pragma unroll
                    for (int n = 0; n < N; ++n)
                        if (n == a) x = st.x[l][n];
                    return d.lf[a * (S + 1) + i] + x;
                };
                if (fm) fix_windows(d, meta, win[l], fm, logp);
                if (ev >= 0) {
                    R sp[N];
#pragma unroll
                    for (int n = 0; n < N; ++n) sp[n] = n < d.n_names ? d.spot0[n] * m_exp(logp(n)) : R(0);
                    run_event<R, NW, true>(ev_ctx(d, ev, leg_record(d, base + lane, n_pairs, l, active)), leg[l], win[l], sp,
                                     d.event_code[ev], d.event_code[ev + 1], d.event_disc[ev]);
                }
            }
        }
        double y_pair = 0.0;
        if (active) {
            y_pair = 0.5 * (leg[0].pv + leg[1].pv);
            if (d.pair_value) d.pair_value[base + lane] = y_pair;
            unsigned long long bp = 0, bc = 0, br = 0;
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                bp += leg[l].bad_pay, bc += leg[l].bad_cond;
                br += !(fabs(leg[l].red - 1.0) <= d.red_tol);
            }
            if (bp) atomicAdd(&d.bad[0], bp);
            if (bc) atomicAdd(&d.bad[1], bc);
            if (br) atomicAdd(&d.bad[2], br);
        }
        const double s1 = warp_sum(y_pair), s2 = warp_sum(y_pair * y_pair);
        if (lane == 0) wacc[warp][0] += s1, wacc[warp][1] += s2;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int w = 0; w < n_warps; ++w) s += wacc[w][threadIdx.x];
        partial[2 * static_cast<long long>(blockIdx.x) + threadIdx.x] = s;
    }
}

// Every name local vol (kind 1), N names: the fused kernel's layout and stepping (fused.cuh) with the script at the
// step ends. Shared memory holds per step {-dt/2, sqrt(dt), dt}, per step and name {lo, inv_dx, log-forward, row},
// the correlation root, the table as (y, dy) pairs, and per step end the event to run and the windows fixing there.
// Normals come in batches of G steps of whole Philox blocks; the correlated z is computed once a pair and used with
// both signs. Block totals as in script_kernel.
struct LvOffsets {
    int step, name_step, root, table2, sched, lf0;
};

template <typename R>
struct LvArgs {
    LvOffsets off;
    const unsigned char* blob;
    int smem_blob;
    R top;
    const Pair2<R>* tab;  // the table in global memory when it does not fit the stage (kernels with GT), else unused
    int table_global;
};

// BRANCH: the pairs continue the paths of an outer simulation after step end d.branch_step (one leg per outer path:
// before the branch both legs take the outer path's normals, the outer antithetic leg's with the sign flipped).
// GT: the table is read from global memory (a.tab) instead of the stage.
template <typename R, int N, int NW, bool BRANCH, bool CALLS, bool GT = false, int WF = -1>
__global__ void __launch_bounds__(512, sizeof(R) == 4 ? 2 : 1)
    script_lv_kernel(ScriptDev<R> d, LvArgs<R> a, long long n_pairs, uint32_t k0, uint32_t k1,
                     double* __restrict__ partial) {
    constexpr int C = N;
    // One name, at most one window, no branch (the Phoenix and the barrier products): two Philox blocks a batch (8
    // steps, their independent multiply chains interleave), the full batches without the last-step test and the
    // batches without an event without its test, as in the fused kernel. Wider scripts keep one loop (its copies
    // would spill their window states).
    constexpr bool kLean = N == 1 && NW <= 1 && !BRANCH;
    constexpr int G = kLean ? 8 : (C % 4 == 0 ? 1 : (C % 2 == 0 ? 2 : 4));
    constexpr int NB = C * G / 4;
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ double wacc[16][2];
    {
        const int4* src = reinterpret_cast<const int4*>(a.blob);
        int4* dst = reinterpret_cast<int4*>(sm);
        for (int t = threadIdx.x; t < a.smem_blob / 16; t += blockDim.x) dst[t] = src[t];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    if (threadIdx.x < 32) (&wacc[0][0])[threadIdx.x] = 0.0;
    __syncthreads();
    const StepRec<R>* s_step = reinterpret_cast<const StepRec<R>*>(sm + a.off.step);
    const NameStep<R>* s_ns = reinterpret_cast<const NameStep<R>*>(sm + a.off.name_step);
    const R* s_root = reinterpret_cast<const R*>(sm + a.off.root);
    const Pair2<R>* s_tab = GT ? a.tab : reinterpret_cast<const Pair2<R>*>(sm + a.off.table2);
    const int2* s_sched = reinterpret_cast<const int2*>(sm + a.off.sched);  // (event, window mask) per step end
    const R* s_lf0 = reinterpret_cast<const R*>(sm + a.off.lf0);
    const int S = d.n_steps;
    const WinMeta<NW> meta = win_meta<R, NW>(d);
    // the correlation root: in registers for one or two names, read from shared memory for more (registers spill)
    constexpr bool kRootRegs = N <= 2;
    R rt[kRootRegs ? N * N : 1];
#pragma unroll
    for (int k = 0; k < (kRootRegs ? N * N : 0); ++k) rt[k] = s_root[k];
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < n_pairs;
         base += stride) {
        const bool active = base + lane < n_pairs;
        const uint64_t pair = static_cast<uint64_t>(active ? base + lane : n_pairs - 1);
        uint64_t opair = 0;
        R osign = R(1);
        if (BRANCH) {
            const long long o = static_cast<long long>(pair) / d.branch_pairs;  // the outer path continued
            opair = static_cast<uint64_t>(o < d.branch_outer ? o : o - d.branch_outer);
            osign = o < d.branch_outer ? R(1) : R(-1);
        }
        LegState<R> leg[2];
        leg_init(d, leg[0]), leg_init(d, leg[1]);
        WinState<R, NW> win[2];
        win_init(d, win[0]), win_init(d, win[1]);
        R x0[N], x1[N], y0[N], y1[N];
#pragma unroll
        for (int n = 0; n < N; ++n) x0[n] = x1[n] = R(0), y0[n] = y1[n] = s_lf0[n];
        // the step end i: its window fixings and (EV) its event; a batch whose steps hold no event runs with EV false
        auto observe = [&](int i, auto events) {
            constexpr bool EV = decltype(events)::value;
            const int2 sc = s_sched[i];
            if (!sc.y && (!EV || sc.x < 0)) return;
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                auto logp = [&](int nm) -> R {
                    if constexpr (N == 1) return l ? y1[0] : y0[0];
                    R v = R(0);
#pragma unroll
                    for (int n = 0; n < N; ++n)
                        if (n == nm) v = l ? y1[n] : y0[n];
                    return v;
                };
                if (sc.y) fix_windows<WF>(d, meta, win[l], static_cast<unsigned>(sc.y), logp);
                if (EV && sc.x >= 0) {
                    R sp[N];
#pragma unroll
                    for (int n = 0; n < N; ++n) sp[n] = d.spot0[n] * m_exp(l ? y1[n] : y0[n]);
                    run_event<R, NW, CALLS>(ev_ctx(d, sc.x, leg_record(d, base + lane, n_pairs, l, active)), leg[l], win[l],
                                     sp, d.event_code[sc.x], d.event_code[sc.x + 1], d.event_disc[sc.x]);
                }
            }
        };
        observe(0, std::true_type{});
        // One batch of G steps from step i0; only the tail batch (CHECK) may stop inside.
        auto run_batch = [&](int i0, int b, auto check, auto events) {
            constexpr bool CHECK = decltype(check)::value;
            R z[C * G];
            const bool own = !BRANCH || i0 + G - 1 > d.branch_step;  // a step of the batch draws its own normals
            if (own) {
#pragma unroll
                for (int k = 0; k < NB; ++k)
                    normals4<R>(pair, static_cast<uint64_t>(b) * NB + k, 0u, k0, k1, z[4 * k], z[4 * k + 1],
                                z[4 * k + 2], z[4 * k + 3]);
            }
            R zo[BRANCH ? C * G : 1];
            if (BRANCH && i0 <= d.branch_step) {  // a step of the batch follows the outer path
#pragma unroll
                for (int k = 0; k < NB; ++k)
                    normals4<R>(opair, static_cast<uint64_t>(b) * NB + k, 0u, d.bk0, d.bk1, zo[4 * k], zo[4 * k + 1],
                                zo[4 * k + 2], zo[4 * k + 3]);
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int i = i0 + g;
                if constexpr (CHECK && G > 1) {
                    if (i > S) break;
                }
                const StepRec<R> st = s_step[i - 1];
                const bool before = BRANCH && i <= d.branch_step;
                const R* zs = before ? &zo[g * C] : &z[g * C];
                const R sg0 = before ? osign : R(1), sg1 = before ? osign : R(-1);  // the legs' signs
                R zc[N];
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    R acc = R(0);
#pragma unroll
                    for (int m = 0; m < N; ++m) acc += (kRootRegs ? rt[n * N + m] : s_root[n * N + m]) * zs[m];
                    zc[n] = acc;
                }
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    const NameStep<R> ns = s_ns[(i - 1) * N + n];
                    int j0, j1;
                    R f0, f1;
                    table_cell(ns, a.top, x0[n], j0, f0), table_cell(ns, a.top, x1[n], j1, f1);
                    const Pair2<R> p0 = GT ? ldg_pair(s_tab + ns.row + j0) : s_tab[ns.row + j0];
                    const Pair2<R> p1 = GT ? ldg_pair(s_tab + ns.row + j1) : s_tab[ns.row + j1];
                    const R v0 = p0.a + f0 * p0.b, v1 = p1.a + f1 * p1.b;
                    // sqrt(dt) z with the legs' signs (+1, -1 but before a branch), the step's multiply-add written
                    // out: the same arithmetic in every instantiation, so a branch at step 0 is an ordinary run bit
                    // for bit
                    const R zd = st.sdt * zc[n], z0 = sg0 * zd, z1 = sg1 * zd;
                    x0[n] = lv_advance(x0[n], v0, st.hdt, z0);
                    x1[n] = lv_advance(x1[n], v1, st.hdt, z1);
                    y0[n] = x0[n] + ns.lf, y1[n] = x1[n] + ns.lf;
                }
                observe(i, events);
            }
        };
        // a step end without an event holds minus the steps to the next one: none in i0 .. i0 + G - 1 when step
        // i0's entry is at most -G
        if constexpr (kLean) {
            const int n_full = S / G;
            int i0 = 1, b = 0;
            for (; b < n_full; i0 += G, ++b) {
                if (s_sched[i0].x <= -G) run_batch(i0, b, std::false_type{}, std::false_type{});
                else run_batch(i0, b, std::false_type{}, std::true_type{});
            }
            if (i0 <= S) run_batch(i0, b, std::true_type{}, std::true_type{});
        } else {
            for (int i0 = 1, b = 0; i0 <= S; i0 += G, ++b) run_batch(i0, b, std::true_type{}, std::true_type{});
        }
        double y_pair = 0.0;
        if (active) {
            y_pair = 0.5 * (leg[0].pv + leg[1].pv);
            if (d.pair_value) d.pair_value[base + lane] = y_pair;
            unsigned long long bp = 0, bc = 0, br = 0;
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                bp += leg[l].bad_pay, bc += leg[l].bad_cond;
                br += !(fabs(leg[l].red - 1.0) <= d.red_tol);
            }
            if (bp) atomicAdd(&d.bad[0], bp);
            if (bc) atomicAdd(&d.bad[1], bc);
            if (br) atomicAdd(&d.bad[2], br);
        }
        const double s1 = warp_sum(y_pair), s2 = warp_sum(y_pair * y_pair);
        if (lane == 0) wacc[warp][0] += s1, wacc[warp][1] += s2;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int w = 0; w < n_warps; ++w) s += wacc[w][threadIdx.x];
        partial[2 * static_cast<long long>(blockIdx.x) + threadIdx.x] = s;
    }
}

template <typename R>
using ScriptLvFn = void (*)(ScriptDev<R>, LvArgs<R>, long long, uint32_t, uint32_t, double*);

template <typename R, int NW, bool CALLS, bool GT = false>
ScriptLvFn<R> pick_lv_calls(int n) {
    switch (n) {
        case 1: return script_lv_kernel<R, 1, NW, false, CALLS, GT>;
        case 2: return script_lv_kernel<R, 2, NW, false, CALLS, GT>;
        case 3: return script_lv_kernel<R, 3, NW, false, CALLS, GT>;
        case 4: return script_lv_kernel<R, 4, NW, false, CALLS, GT>;
        case 5: return script_lv_kernel<R, 5, NW, false, CALLS, GT>;
        default: return nullptr;
    }
}

template <typename R, int NW>
ScriptLvFn<R> pick_lv_nw(int n, bool branch, bool calls) {
    if (branch) return n == 1 ? script_lv_kernel<R, 1, NW, true, true> : nullptr;  // the dual bound: one name
    return calls ? pick_lv_calls<R, NW, true>(n) : pick_lv_calls<R, NW, false>(n);
}

// Kernels for one window (a knock-in barrier: its state alone stays in registers under the 64-register cap of two
// blocks an SM, where a second window's spills it to local memory, 3.11 -> 2.67 ms for the 3-year daily-window
// Phoenix), up to 2 and up to 8. A table in global memory (table_global) only comes with up to 2 windows, no call and
// no branch (pack_lv checks).
// One name whose one window is a lowest or a highest (a knock-in or knock-out barrier of a single-name note), no call
// and no branch: the window's function is compiled in (fix_windows, WF).
template <typename R, bool GT>
ScriptLvFn<R> pick_lv_single_window(int win_func) {
    return win_func == 0 ? script_lv_kernel<R, 1, 1, false, false, GT, 0> : script_lv_kernel<R, 1, 1, false, false, GT, 1>;
}

template <typename R>
ScriptLvFn<R> pick_lv(int n, int n_windows, int win_func0, bool branch, bool calls, bool table_global) {
    if (n == 1 && n_windows == 1 && !branch && !calls && (win_func0 == 0 || win_func0 == 1))
        return table_global ? pick_lv_single_window<R, true>(win_func0) : pick_lv_single_window<R, false>(win_func0);
    if (table_global) return n_windows <= 1 ? pick_lv_calls<R, 1, false, true>(n) : pick_lv_calls<R, 2, false, true>(n);
    if (n_windows <= 1 && !branch && !calls) return pick_lv_calls<R, 1, false>(n);
    return n_windows <= 2 ? pick_lv_nw<R, 2>(n, branch, calls) : pick_lv_nw<R, kMaxWindows>(n, branch, calls);
}

// The staged blob of the local-vol path, or false when it does not apply (a name not local vol, more than five
// names, or more than the shared-memory budget: 110 KB in float, 220 KB in double, without the table). The table
// goes into the stage when it fits beside the rest, else into global memory (L2-resident, read through the read-only
// cache) for scripts with up to two windows, no call and no branch.
template <typename R>
bool pack_lv(const ob_script_request& rq, const std::vector<int2>& sched, DeviceArena& arena, LvArgs<R>& a) {
    const ob_mc_request& q = rq.model;
    const int n = q.n_names, S = q.n_steps;
    if (q.model != OB_MODEL_PATHS || n > 5 || q.mixer) return false;
    for (int k = 0; k < n; ++k)
        if (q.kind[k] != 1) return false;
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
        steps[i].hdt = static_cast<R>(-0.5 * q.dt[i]), steps[i].sdt = static_cast<R>(std::sqrt(q.dt[i]));
        steps[i].dt = static_cast<R>(q.dt[i]), steps[i].obs = -1;
    }
    a.off.step = put(steps.data(), steps.size() * sizeof(StepRec<R>));
    a.top = static_cast<R>(q.n_x - 1) - static_cast<R>(1e-4);
    std::vector<NameStep<R>> ns(static_cast<size_t>(S) * n);
    for (int i = 1; i <= S; ++i)
        for (int k = 0; k < n; ++k) {
            NameStep<R>& r = ns[static_cast<size_t>(i - 1) * n + k];
            std::memset(&r, 0, sizeof r);
            const int row = q.step_row[static_cast<size_t>(k) * S + (i - 1)];
            r.lf = static_cast<R>(q.log_fwd[static_cast<size_t>(k) * (S + 1) + i]);
            set_cell_row(r, q.row_lo[row], q.row_inv_dx[row], a.top);
            r.row = row * (q.n_x - 1);
        }
    a.off.name_step = put(ns.data(), ns.size() * sizeof(NameStep<R>));
    std::vector<R> root(static_cast<size_t>(n) * n), lf0(n);
    for (size_t k = 0; k < root.size(); ++k) root[k] = static_cast<R>(q.root[k]);
    for (int k = 0; k < n; ++k) lf0[k] = static_cast<R>(q.log_fwd[static_cast<size_t>(k) * (S + 1)]);
    a.off.root = put(root.data(), root.size() * sizeof(R));
    a.off.lf0 = put(lf0.data(), lf0.size() * sizeof(R));
    a.off.sched = put(sched.data(), sched.size() * sizeof(int2));
    std::vector<Pair2<R>> tab(static_cast<size_t>(q.n_rows) * (q.n_x - 1));
    for (int r = 0; r < q.n_rows; ++r)
        for (int k = 0; k + 1 < q.n_x; ++k) {
            const double* row = q.table + static_cast<size_t>(r) * q.n_x;
            tab[static_cast<size_t>(r) * (q.n_x - 1) + k] = {static_cast<R>(row[k]), static_cast<R>(row[k + 1] - row[k])};
        }
    const size_t budget = sizeof(R) == 4 ? (110u << 10) : (220u << 10);
    if (blob.size() > budget) return false;
    a.table_global = ((blob.size() + 15) & ~static_cast<size_t>(15)) + tab.size() * sizeof(Pair2<R>) > budget;
    if (a.table_global && (rq.branch || rq.n_calls > 0 || rq.n_windows > 2)) return false;
    if (a.table_global) a.tab = arena.put_raw(tab.data(), tab.size());
    else a.off.table2 = put(tab.data(), tab.size() * sizeof(Pair2<R>));
    a.smem_blob = static_cast<int>((blob.size() + 15) & ~static_cast<size_t>(15));
    unsigned char* dblob = arena.alloc<unsigned char>(std::max<size_t>(16, blob.size()));
    check_cuda(cudaMemcpy(dblob, blob.data(), blob.size(), cudaMemcpyHostToDevice), "copy blob");
    a.blob = dblob;
    return true;
}

// The blocks' totals added in block order by one warp per sum (lane l adds blocks l, l + 32, ...).
__global__ void script_finalize(const double* __restrict__ partial, int n_blocks, double* __restrict__ sums) {
    const int lane = threadIdx.x & 31, t = threadIdx.x >> 5;
    if (t >= 2) return;
    double s = 0.0;
    for (int b = lane; b < n_blocks; b += 32) s += partial[2 * static_cast<long long>(b) + t];
    s = warp_sum(s);
    if (lane == 0) sums[t] = s;
}

template <typename R>
using ScriptFn = void (*)(ScriptDev<R>, long long, uint32_t, uint32_t, double*);

template <typename R, int NW>
ScriptFn<R> pick_script_nw(int model, int n) {
    if (model == OB_MODEL_HESTON_QE) return script_kernel<R, 1, OB_MODEL_HESTON_QE, NW>;
    if (n <= 1) return script_kernel<R, 1, OB_MODEL_PATHS, NW>;
    if (n <= 2) return script_kernel<R, 2, OB_MODEL_PATHS, NW>;
    if (n <= 4) return script_kernel<R, 4, OB_MODEL_PATHS, NW>;
    return script_kernel<R, 8, OB_MODEL_PATHS, NW>;
}

template <typename R>
ScriptFn<R> pick_script(int model, int n, int n_windows) {
    return n_windows <= 2 ? pick_script_nw<R, 2>(model, n) : pick_script_nw<R, kMaxWindows>(model, n);
}

// Every index the device will follow is checked here: registers, names, windows, tags, code ranges and steps.
void check_script(const ob_script_request& rq, bool record_needed = true) {
    check_mc_model(rq.model);
    const int S = rq.model.n_steps, n = rq.model.n_names;
    if (rq.n_regs < 1 || rq.n_regs > kMaxRegs) invalid("n_regs must be 1 to 128");
    if (rq.n_const < 1 || rq.n_const > rq.n_regs || !rq.consts) invalid("n_const must be 1 to n_regs");
    if (rq.n_code < 0 || (rq.n_code > 0 && !rq.code)) invalid("null code");
    if (rq.n_events < 1 || !rq.event_step || !rq.event_code || !rq.event_discount) invalid("a script needs events");
    if (rq.n_windows < 0 || rq.n_windows > kMaxWindows) invalid("n_windows must be 0 to 8");
    if (rq.n_windows && (!rq.win_name || !rq.win_func || !rq.win_fix0 || !rq.fix_step || !rq.win_lower ||
                         !rq.win_upper))
        invalid("null window arrays");
    if (!(rq.smoothing >= 0)) invalid("smoothing must be >= 0");
    for (int k = 0; k < rq.n_events; ++k) {
        if (rq.event_step[k] < 0 || rq.event_step[k] > S || (k && rq.event_step[k] <= rq.event_step[k - 1]))
            invalid("event steps must increase within 0 .. n_steps");
        if (!(rq.event_discount[k] >= 0)) invalid("event discounts must be >= 0");
    }
    for (int k = 0; k <= rq.n_events; ++k)
        if (rq.event_code[k] < 0 || rq.event_code[k] > rq.n_code || (k && rq.event_code[k] < rq.event_code[k - 1]))
            invalid("event code ranges must increase within the code");
    for (int w = 0; w < rq.n_windows; ++w) {
        if (rq.win_name[w] < 0 || rq.win_name[w] >= n) invalid("a window reads an unknown name");
        if (rq.win_func[w] < 0 || rq.win_func[w] > 2) invalid("win_func must be 0, 1 or 2");
        if (rq.win_fix0[w] < 0 || rq.win_fix0[w + 1] <= rq.win_fix0[w]) invalid("a window needs fixings");
        if (rq.win_func[w] == 2 && rq.win_fix0[w + 1] - rq.win_fix0[w] < 2)
            invalid("a variance window needs at least two fixings");
        for (int k = rq.win_fix0[w]; k < rq.win_fix0[w + 1]; ++k)
            if (rq.fix_step[k] < 0 || rq.fix_step[k] > S || (k > rq.win_fix0[w] && rq.fix_step[k] <= rq.fix_step[k - 1]))
                invalid("window fixing steps must increase within 0 .. n_steps");
    }
    if (rq.branch != 0 && rq.branch != 1) invalid("branch must be 0 or 1");
    if (rq.branch) {
        if (n != 1 || rq.model.model != OB_MODEL_PATHS || rq.model.kind[0] != 1)
            invalid("a branched run continues one local-vol name");
        if (rq.branch_step < 0 || rq.branch_step > S) invalid("branch_step must be within 0 .. n_steps");
        if (rq.branch_outer < 1 || rq.branch_pairs < 1 || rq.model.n_pairs != 2 * rq.branch_outer * rq.branch_pairs)
            invalid("a branched run has branch_pairs pairs for each of the 2 branch_outer outer paths");
    }
    if (rq.n_calls < 0 || rq.n_state < 0 || rq.n_state > kMaxState) invalid("n_calls >= 0 and n_state 0 to 4");
    if (rq.call_mode < 0 || rq.call_mode > 2) invalid("call_mode must be 0, 1 or 2");
    if (rq.n_calls && !rq.call_state) invalid("null call_state");
    if (record_needed && rq.call_mode == 1 && rq.n_calls && !rq.record) invalid("call_mode 1 needs a record array");
    if (rq.call_mode == 2 && rq.n_calls && !rq.rules) invalid("call_mode 2 needs rules");
    for (int c = 0; c < rq.n_calls; ++c)
        for (int j = 0; j < rq.n_state; ++j)
            if (rq.call_state[4 * c + j] < 0 || rq.call_state[4 * c + j] >= rq.n_regs)
                invalid("a call's state names a register beyond n_regs");
    if (rq.call_mode == 2)
        for (int c = 0; c < rq.n_calls; ++c) {
            const double* r = rq.rules + static_cast<long long>(c) * OB_RULE_STRIDE;
            if (r[0] == 0.0) continue;
            const double np = r[1], nk = r[2];
            if (!(np >= 0 && np <= kMaxPoly && nk >= 0 && nk <= kMaxKnots) || np != std::floor(np) ||
                nk != std::floor(nk))
                invalid("a rule has 0 to 25 polynomial terms and 0 to 25 hinges");
            for (int t = 0; t < static_cast<int>(np); ++t)
                for (int j = 0; j < rq.n_state; ++j) {
                    const double pw = r[11 + 4 * t + j];
                    if (!(pw >= 0 && pw <= 3) || pw != std::floor(pw)) invalid("rule powers must be 0 to 3");
                }
            for (int q = 0; q < static_cast<int>(nk); ++q) {
                const double v = r[111 + q];
                if (!(v >= 0 && v < rq.n_state) || v != std::floor(v)) invalid("a hinge names an unknown state");
            }
            for (int j = 0; j < rq.n_state; ++j)
                if (!(r[7 + j] != 0.0)) invalid("a rule's scales must not be 0");
        }
    auto reg = [&](int r) {
        if (r < 0 || r >= rq.n_regs) invalid("an instruction names a register beyond n_regs");
    };
    for (int pc = 0; pc < rq.n_code; ++pc) {
        const int* in = rq.code + 4 * pc;
        const int op = in[0], d = in[1], a = in[2], b = in[3];
        if (op < 0 || op >= kNumOps) invalid("unknown instruction");
        switch (op) {
            case kSpot:
                reg(d);
                if (a < 0 || a >= n) invalid("an instruction reads an unknown name");
                break;
            case kWin:
                reg(d);
                if (a < 0 || a >= rq.n_windows) invalid("an instruction reads an unknown window");
                break;
            case kPay:
                if (d < 0 || d > 2) invalid("a payment tag must be 0, 1 or 2");
                reg(a), reg(b);
                break;
            case kTerm: reg(a); break;
            case kCall:
                if (d < 0 || d >= rq.n_calls) invalid("a call instruction names an unknown call");
                reg(a), reg(b);
                break;
            case kMov: case kNeg: case kAbs: case kExp: case kLog: case kSqrt: case kNot: reg(d), reg(a); break;
            default:
                reg(d), reg(a), reg(b);
                if (op == kAssign && d < rq.n_const) invalid("an assignment to a constant register");
        }
    }
}

// Called with the pilot's record while it is in device memory (call_mode 1): rows of stride doubles, one a path, and
// the call's device arena.
using RecordHook = std::function<void(const double* record, long long n_paths, int stride, DeviceArena& arena)>;

template <typename R>
void run_script(const ob_script_request& rq, ob_script_result& res, const RecordHook* hook = nullptr) {
    const auto t_start = std::chrono::steady_clock::now();
    const int sms = require_device();
    DeviceArena arena;
    arena.recycle = true;  // the blocking copies of the sums and records end the call's device work
    const ob_mc_request& mq = rq.model;
    const int n = mq.n_names, S = mq.n_steps;
    ScriptDev<R> d{};
    d.model = mq.model, d.n_names = n, d.n_steps = S;
    for (int a = 0; a < n; ++a) d.spot0[a] = static_cast<R>(mq.spot[a]);
    Upload up;
    ModelDev<R>& m = d.m;
    m.n_names = n, m.n_steps = S, m.n_x = mq.n_x, m.same = mq.same, m.mixer = mq.mixer;
    up.add<R>(m.dt, mq.dt, S);
    up.add<R>(m.t0, mq.t0, S);
    if (mq.mixer) {  // local correlation: the generic interpreter kernel runs it (pack_lv declines)
        up.add<R>(m.low_root, mq.low_root, static_cast<size_t>(n) * n);
        for (int k = 0; k < 8; ++k) m.mix[k] = static_cast<R>(mq.mix[k]);
    }
    if (mq.model == OB_MODEL_PATHS) {
        bool table = false;
        for (int a = 0; a < n; ++a) {
            m.has_var |= mq.kind[a] == 2 || mq.kind[a] == 3;
            m.has_slv |= mq.kind[a] == 3;
            table |= mq.kind[a] == 1 || mq.kind[a] == 3;
        }
        up.add<R>(m.root, mq.root, static_cast<size_t>(n) * n);
        up.add<int>(m.kind, mq.kind, n);
        up.add<R>(m.cvar, mq.cvar, n);
        up.add<R>(m.hes, mq.heston, 5 * static_cast<size_t>(n));
        if (table) {
            up.add<int>(m.step_row, mq.step_row, static_cast<size_t>(n) * S);
            up.add<R>(m.lo, mq.row_lo, mq.n_rows);
            up.add<R>(m.inv_dx, mq.row_inv_dx, mq.n_rows);
            up.add<R>(m.table, mq.table, static_cast<size_t>(mq.n_rows) * mq.n_x);
        }
        up.add<R>(d.lf, mq.log_fwd, static_cast<size_t>(n) * (S + 1));
    } else {
        d.qe = make_qe_consts<R>(mq.heston, mq.r, mq.q, mq.dt[0]);
    }
    std::vector<int4> code(static_cast<size_t>(rq.n_code));  // (the caller's ints need not be 16-byte aligned)
    if (rq.n_code) std::memcpy(code.data(), rq.code, code.size() * sizeof(int4));
    up.add<int4>(d.code, code.data(), code.size());
    up.add<double>(d.consts, rq.consts, rq.n_const);
    d.n_const = rq.n_const, d.n_regs = rq.n_regs;
    std::vector<int> event_at(S + 1, -1);
    for (int k = 0; k < rq.n_events; ++k) event_at[rq.event_step[k]] = k;
    up.add<int>(d.event_at, event_at.data(), event_at.size());
    up.add<int>(d.event_code, rq.event_code, rq.n_events + 1);
    up.add<double>(d.event_disc, rq.event_discount, rq.n_events);
    std::vector<unsigned> fix_mask(S + 1, 0u);
    std::vector<int> nfix(std::max(1, rq.n_windows), 0);
    for (int w = 0; w < rq.n_windows; ++w) {
        for (int k = rq.win_fix0[w]; k < rq.win_fix0[w + 1]; ++k) fix_mask[rq.fix_step[k]] |= 1u << w;
        nfix[w] = rq.win_fix0[w + 1] - rq.win_fix0[w];
    }
    up.add<unsigned>(d.fix_mask, fix_mask.data(), fix_mask.size());
    d.n_windows = rq.n_windows;
    if (rq.n_windows) {
        up.add<int>(d.win_name, rq.win_name, rq.n_windows);
        up.add<int>(d.win_func, rq.win_func, rq.n_windows);
        up.add<int>(d.win_nfix, nfix.data(), rq.n_windows);
        // the corridor as bounds on ln(S / spot0) of the window's name (NaN: no bound)
        std::vector<double> llo(rq.n_windows), lhi(rq.n_windows);
        for (int w = 0; w < rq.n_windows; ++w) {
            const double s0 = mq.spot[rq.win_name[w]];
            auto bound = [&](double b) {
                return std::isnan(b) ? b : (b > 0 ? std::log(b / s0) : -INFINITY);  // no positive spot is <= 0
            };
            llo[w] = bound(rq.win_lower[w]), lhi[w] = bound(rq.win_upper[w]);
        }
        up.add<double>(d.win_lo, llo.data(), llo.size());
        up.add<double>(d.win_hi, lhi.data(), lhi.size());
        std::vector<double> ws0(rq.n_windows);
        for (int w = 0; w < rq.n_windows; ++w) ws0[w] = mq.spot[rq.win_name[w]];
        up.add<R>(d.win_spot0, ws0.data(), ws0.size());
    }
    d.n_events = rq.n_events, d.n_calls = rq.n_calls, d.n_state = rq.n_state, d.call_mode = rq.call_mode;
    d.rec_stride = 2 * rq.n_events + rq.n_calls * (3 + rq.n_state);
    if (rq.n_calls) {
        up.add<int>(d.call_state, rq.call_state, 4 * static_cast<size_t>(rq.n_calls));
        if (rq.call_mode == 2) up.add<double>(d.rules, rq.rules, static_cast<size_t>(rq.n_calls) * OB_RULE_STRIDE);
    }
    const size_t rec_count = rq.call_mode == 1 ? static_cast<size_t>(2 * mq.n_pairs) * d.rec_stride : 0;
    if (rec_count) {
        d.record = arena.alloc<double>(rec_count);
        check_cuda(cudaMemset(d.record, 0, rec_count * sizeof(double)), "cudaMemset");
    }
    d.branch_step = rq.branch ? rq.branch_step : -1;
    d.branch_outer = rq.branch_outer, d.branch_pairs = rq.branch_pairs;
    d.bk0 = static_cast<uint32_t>(rq.branch_seed), d.bk1 = static_cast<uint32_t>(rq.branch_seed >> 32);
    if (rq.pair_value) d.pair_value = arena.alloc<double>(static_cast<size_t>(mq.n_pairs));
    d.eps = static_cast<R>(rq.smoothing);
    d.red_tol = rq.smoothing == 0.0 ? 1e-12 : (sizeof(R) == 8 ? 1e-9 : 1e-5);
    // the run's outputs read back by one copy: the three counts (zeroed here), then the two sums (slots 4, 5)
    unsigned long long* outs = nullptr;
    up.zeros<unsigned long long>(outs, 8);
    // the inputs but the staged kernel's blob (pack_lv) in one copy
    up.commit(arena);
    d.bad = outs;

    // per step end (event, window mask); a step end without an event holds minus the number of steps to the next
    // one (past the last, more than any batch)
    std::vector<int2> sched(S + 1);
    for (int i = S, next = S + (1 << 20); i >= 0; --i) {
        if (event_at[i] >= 0) next = i;
        sched[i] = make_int2(event_at[i] >= 0 ? event_at[i] : i - next, static_cast<int>(fix_mask[i]));
    }
    LvArgs<R> lv{};
    const bool fast = pack_lv<R>(rq, sched, arena, lv);
    if (rq.branch && !fast) invalid("a branched run needs the staged local-vol kernel (its tables too large)");
    const void* fn = fast ? reinterpret_cast<const void*>(
                                pick_lv<R>(n, rq.n_windows, rq.n_windows ? rq.win_func[0] : -1, rq.branch != 0, rq.n_calls > 0,
                                          lv.table_global != 0))
                          : reinterpret_cast<const void*>(pick_script<R>(mq.model, n, rq.n_windows));
    const int block = fast ? 512 : 128;
    const size_t smem = fast ? static_cast<size_t>(lv.smem_blob) : 0;
    if (fast) allow_smem(fn, smem);
    const int per_sm = occupancy(fn, block, smem);
    const long long need = (mq.n_pairs + block - 1) / block;
    const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>(need, 1LL * sms * std::max(1, per_sm))));
    double* partial = arena.alloc<double>(2 * static_cast<size_t>(grid));
    double* sums = reinterpret_cast<double*>(outs + 4);
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    const uint32_t k0 = static_cast<uint32_t>(mq.seed), k1 = static_cast<uint32_t>(mq.seed >> 32);
    check_cuda(cudaEventRecord(e0), "cudaEventRecord");
    if (fast)
        reinterpret_cast<ScriptLvFn<R>>(const_cast<void*>(fn))<<<grid, block, smem>>>(d, lv, mq.n_pairs, k0, k1, partial);
    else
        reinterpret_cast<ScriptFn<R>>(const_cast<void*>(fn))<<<grid, block>>>(d, mq.n_pairs, k0, k1, partial);
    check_cuda(cudaGetLastError(), "script_kernel launch");
    script_finalize<<<1, 64>>>(partial, grid, sums);
    check_cuda(cudaGetLastError(), "script_finalize launch");
    check_cuda(cudaEventRecord(e1), "cudaEventRecord");
    unsigned long long out[8];
    void* pin = small_pinned();
    check_cuda(cudaMemcpyAsync(pin ? pin : out, outs, sizeof out, cudaMemcpyDeviceToHost), "copy sums and counts");
    check_cuda(cudaStreamSynchronize(nullptr), "script kernel");
    if (pin) std::memcpy(out, pin, sizeof out);
    double h[2];
    std::memcpy(h, out + 4, sizeof h);
    const unsigned long long* bad = out;
    if (rec_count && rq.record)
        check_cuda(cudaMemcpy(rq.record, d.record, rec_count * sizeof(double), cudaMemcpyDeviceToHost), "copy record");
    if (rec_count && hook) (*hook)(d.record, 2 * mq.n_pairs, d.rec_stride, arena);
    if (rq.pair_value)
        check_cuda(cudaMemcpy(rq.pair_value, d.pair_value, static_cast<size_t>(mq.n_pairs) * sizeof(double),
                              cudaMemcpyDeviceToHost),
                   "copy pair values");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0), cudaEventDestroy(e1);
    const double nn = static_cast<double>(mq.n_pairs), mean = h[0] / nn;
    res.price = mean;
    res.se = nn > 1 ? std::sqrt(std::fmax(h[1] / nn - mean * mean, 0.0) / (nn - 1.0)) : 0.0;
    res.n_paths = 2 * mq.n_pairs;
    res.bad_pay = static_cast<long long>(bad[0]), res.bad_cond = static_cast<long long>(bad[1]);
    res.bad_redemption = static_cast<long long>(bad[2]);
    res.kernel_ms = ms;
    (void)t_start;
}

}  // namespace
}  // namespace ob

extern "C" int ob_script_price(const ob_script_request* rq, int precision, ob_script_result* res) {
    return ob::guarded([&] {
        if (!rq || !res) ob::invalid("null argument");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        ob::check_script(*rq);
        *res = ob_script_result{};
        if (precision == OB_FP32) ob::run_script<float>(*rq, *res);
        else ob::run_script<double>(*rq, *res);
    });
}

extern "C" int ob_script_pilot_fit(const ob_script_request* rq, int precision, const int* call_event,
                                   const double* pay_discount, double* rules, double* in_sample, ob_script_result* res) {
    return ob::guarded([&] {
        if (!rq || !res || !call_event || !pay_discount || !rules || !in_sample) ob::invalid("null argument");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        if (rq->call_mode != 1 || rq->n_calls < 1) ob::invalid("the pilot fit runs a pilot (call_mode 1) of a script with calls");
        ob::check_script(*rq, false);
        std::vector<char> seen(rq->n_events, 0);
        for (int c = 0; c < rq->n_calls; ++c) {
            if (call_event[c] < 0 || call_event[c] >= rq->n_events || seen[call_event[c]])
                ob::invalid("call_event must name distinct events");
            seen[call_event[c]] = 1;
        }
        *res = ob_script_result{};
        bool fitted = false;
        const ob::RecordHook hook = [&](const double* record, long long n_paths, int stride, ob::DeviceArena& arena) {
            fitted = ob::fit_policy_on_device(record, n_paths, stride, rq->n_events, rq->n_calls, rq->n_state, call_event,
                                              pay_discount, rules, in_sample, arena);
        };
        if (precision == OB_FP32) ob::run_script<float>(*rq, *res, &hook);
        else ob::run_script<double>(*rq, *res, &hook);
        if (!fitted)
            throw ob::Error(OB_ESINGULAR, "pilot fit: a regression's terms are nearly collinear; fit it on the host");
    });
}
