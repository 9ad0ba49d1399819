// The per-pair step of the path engine on the device, in float or double.
//
// Semantics of RC/include/optlab_cuda/paths.hpp:190-276 (simulate_pair): each name in its log-forward x, a log-Euler
// spot step on the variance at the start of the step, full-truncation Euler for the variance:
//     var = c | T(t, x) | max(v, 0) | T(t, x) max(v, 0)     (kind 0 constant, 1 table, 2 Heston, 3 SLV)
//     v  += kappa (theta - v+) dt + xi sqrt(v+ dt) (rho z + sqrt(1 - rho^2) w)
//     x  += -var dt / 2 + sqrt(var dt) z
// with per step the spot normals, then the variance residuals (stream 0, or the aux stream when a name is SLV), then
// the mixer's common normal, and the two legs of a pair on (z, -z). Table rows are uniform in x, read by linear
// interpolation, clamped as paths.hpp:196-205. Andersen's QE-M step (RC/include/optlab_cuda/schemes.hpp:153-186) is
// here too, for the Heston model of the fixed products.
//
// The state of both legs of a pair lives in registers (N names each); the per-step inputs are read through plain
// pointers, which the fused kernel points at shared memory and the drop-in paths kernel at global memory.
#pragma once

#include "common.cuh"

namespace ob {

constexpr uint32_t kAuxStream = 0x80000000u;

template <typename R>
struct ModelDev {
    int n_names, n_steps, n_x, same, mixer;
    int has_var, has_slv;
    uint32_t k0, k1;
    const R* dt;        // n_steps
    const R* t0;        // n_steps
    const R* root;      // n x n
    const int* kind;    // n
    const R* cvar;      // n
    const R* hes;       // n x 5
    const int* step_row;  // n x n_steps
    const R* lo;        // per row
    const R* inv_dx;    // per row
    const R* table;     // rows x n_x
    const R* low_root;  // n x n
    R mix[8];
};

template <typename R>
__device__ __forceinline__ R table_value(const ModelDev<R>& m, int row, R x) {
    R u = (x - m.lo[row]) * m.inv_dx[row];
    const R top = static_cast<R>(m.n_x - 1) - static_cast<R>(1e-4);
    u = m_min(m_max(u, R(0)), top);
    const int i = static_cast<int>(u);
    const R w = u - static_cast<R>(i);
    const R* y = m.table + static_cast<long long>(row) * m.n_x;
    return y[i] * (R(1) - w) + y[i + 1] * w;
}

template <typename R, int N>
struct PairDev {
    R x[2][N], v[2][N];
    NormalStream<R> rng, aux;
};

template <typename R, int N>
__device__ __forceinline__ void pair_init(const ModelDev<R>& m, PairDev<R, N>& s, uint64_t pair) {
#pragma unroll
    for (int a = 0; a < N; ++a) {
        const bool hv = a < m.n_names && (m.kind[a] == 2 || m.kind[a] == 3);
        s.x[0][a] = s.x[1][a] = R(0);
        s.v[0][a] = s.v[1][a] = hv ? m.hes[a * 5] : R(0);
    }
    s.rng.init(pair, m.k0, m.k1, 0u);
    s.aux.init(pair, m.k0, m.k1, kAuxStream);
}

// Step i (1-based) of both legs, as paths.hpp:295-358.
template <typename R, int N>
__device__ __forceinline__ void pair_step(const ModelDev<R>& m, PairDev<R, N>& s, int i) {
    const int n = m.n_names;
    const R dt = m.dt[i - 1];
    R zs[N], zr[N], fresh = R(0);
#pragma unroll
    for (int a = 0; a < N; ++a)
        if (a < n) zs[a] = s.rng.next();
    if (m.has_var) {
#pragma unroll
        for (int a = 0; a < N; ++a)
            if (a < n) zr[a] = m.has_slv ? s.aux.next() : s.rng.next();
    }
    if (m.mixer) fresh = s.rng.next();
#pragma unroll
    for (int leg = 0; leg < 2; ++leg) {
        const R sign = leg ? R(-1) : R(1);
        R z[N], w[N];
        if (N == 1 && !m.mixer) {
            z[0] = sign * (m.root[0] * zs[0]);
        } else if (m.mixer) {
            // paths.hpp:304-322: a common factor whose weight depends on the level of the basket
            R mm = R(0);
#pragma unroll
            for (int a = 0; a < N; ++a)
                if (a < n) mm += m_exp(s.x[leg][a]);
            const R y = m_log(mm / static_cast<R>(n));
            const R t0 = m.t0[i - 1];
            const R u = y / (m.mix[4] * m_sqrt(m_max(t0, R(1.0 / 12))));
            R wt = m.mix[0] + m.mix[1] + m.mix[2] * m_max(-u, R(0)) - m.mix[3] * m_max(u, R(0));
            wt = m_min(m_max(wt, R(0)), R(1));
            const R market = m.mix[5] * sign * zs[n - 1], fr = sign * fresh;
            const R common = m.mix[6] * market + m.mix[7] * fr;
            R other[N];
#pragma unroll
            for (int a = 0; a < N; ++a) other[a] = a < n ? sign * zs[a] : R(0);
#pragma unroll
            for (int a = 0; a < N; ++a)
                if (a == n - 1) other[a] = m.mix[7] * market - m.mix[6] * fr;
            const R sw = m_sqrt(wt), sl = m_sqrt(R(1) - wt);
#pragma unroll
            for (int a = 0; a < N; ++a) {
                R acc = R(0);
#pragma unroll
                for (int b = 0; b < N; ++b)
                    if (a < n && b < n) acc += m.low_root[a * n + b] * other[b];
                z[a] = sw * common + sl * acc;
            }
        } else {
#pragma unroll
            for (int a = 0; a < N; ++a) {
                R acc = R(0);
#pragma unroll
                for (int b = 0; b < N; ++b)
                    if (a < n && b < n) acc += m.root[a * n + b] * zs[b];
                z[a] = sign * acc;
            }
        }
        if (m.has_var) {
#pragma unroll
            for (int a = 0; a < N; ++a) {
                if (m.same) {
                    R acc = R(0);
#pragma unroll
                    for (int b = 0; b < N; ++b)
                        if (a < n && b < n) acc += m.root[a * n + b] * zr[b];
                    w[a] = sign * acc;
                } else {
                    w[a] = a < n ? sign * zr[a] : R(0);
                }
            }
        }
#pragma unroll
        for (int a = 0; a < N; ++a) {
            if (a >= n) continue;
            const int k = m.kind[a];
            R var;
            const R vp = m_max(s.v[leg][a], R(0));
            if (k == 0) {
                var = m.cvar[a];
            } else if (k == 2) {
                var = vp;
            } else {
                const R t = table_value(m, m.step_row[a * m.n_steps + (i - 1)], s.x[leg][a]);
                var = k == 1 ? t : t * vp;
            }
            if (k == 2 || k == 3) {
                const R* h = m.hes + a * 5;
                const R zv = h[4] * z[a] + m_sqrt(R(1) - h[4] * h[4]) * w[a];
                s.v[leg][a] += h[1] * (h[2] - vp) * dt + h[3] * m_sqrt(vp * dt) * zv;
            }
            s.x[leg][a] += R(-0.5) * var * dt + m_sqrt(var * dt) * z[a];
        }
    }
}

// ------------------------------------------------------------------------------------------------ Andersen QE-M

// Constants of one step dt (schemes.hpp:107-141), computed on the host in double and cast once.
template <typename R>
struct QeConsts {
    R v0, theta, mu_dt, E, c1, c2, K1, K2, K3, K4, A, K0p;
};

template <typename R>
inline QeConsts<R> make_qe_consts(const double* h, double r, double q, double dt) {
    const double v0 = h[0], kappa = h[1], theta = h[2], xi = h[3], rho = h[4];
    const double E = std::exp(-kappa * dt), xi2 = xi * xi;
    const double k12 = 0.5 * dt * (kappa * rho / xi - 0.5);
    QeConsts<R> c;
    c.v0 = R(v0), c.theta = R(theta), c.mu_dt = R((r - q) * dt), c.E = R(E);
    c.c1 = R(xi2 * E * (1 - E) / kappa);
    c.c2 = R(theta * xi2 * (1 - E) * (1 - E) / (2 * kappa));
    c.K1 = R(k12 - rho / xi);
    c.K2 = R(k12 + rho / xi);
    c.K3 = R(0.5 * dt * (1 - rho * rho));
    c.K4 = c.K3;
    c.A = R((k12 + rho / xi) + 0.25 * dt * (1 - rho * rho));
    c.K0p = R(-rho * kappa * theta * dt / xi);
    return c;
}

// One QE-M step of (y, v) with independent normals zv (variance) and zx (log-spot), schemes.hpp:154-186. Andersen's
// scheme picks, per path and step, the quadratic branch (psi <= 3/2: v' = a (b + zv)^2) or the exponential one (mass
// p at zero, an exponential tail above it); lanes of a warp take both, so the warp executes both. Here the branches
// share their FP64 divisions: each division's numerator and denominator are selected per lane, so a warp whose lanes
// split runs three divisions (plus the exponential tail's inverse) where the two branches written apart ran seven,
// and psi is never divided out. With s2 = v c1 + c2 (the conditional variance of v') and D = s2 + m^2:
//   branch test    psi <= 3/2            as  s2 <= 3/2 m^2
//   division 1     quadratic: 2 / psi    exponential: 1 - p = 2 / (psi + 1)      (2 m^2 over s2 or D)
//   division 2     quadratic: a = m / (1 + b^2)    exponential: 1 / beta = m / (1 - p)
//   division 3     quadratic: the K0 term -A b^2 a / (1 - 2 A a)    exponential: (1 - p) / (1 - A / beta)
// with the exponential branch's K0 argument p + beta (1 - p) / (beta - A) written as p + (1 - p) / (1 - A / beta) and
// its finiteness A < beta as A / beta < 1 (beta > 0). The algebra is the reference's; only roundings differ.
// EXP: 0 each lane takes its own branch (a lane of the exponential branch runs the tail's CDF and logarithm after the
// step's divisions); 1 every lane evaluates the exponential tail, which each exponential lane keeps (straight-line
// code: the CDF, which depends on zv alone, overlaps the divisions); 2 no lane is exponential.
template <int EXP, typename R>
__device__ __forceinline__ void qe_step_body(const QeConsts<R>& c, R& y, R& v, R zv, R zx, R m, R m2, R s2,
                                             bool quad) {
    R one_minus_u = R(1);
    if (EXP == 1) one_minus_u = m_ncdf(-zv);  // 1 - U, exact in both tails
    const R r1 = (R(2) * m2) / (quad ? s2 : s2 + m2);  // quadratic: 2 / psi; exponential: q = 1 - p
    const R b2 = r1 - R(1) + m_sqrt(quad ? r1 * m_max(r1 - R(1), R(0)) : R(0));
    const R r2 = m / (quad ? R(1) + b2 : r1);  // quadratic: a; exponential: 1 / beta
    const R b = m_sqrt(quad ? b2 : R(0));
    R vn = r2 * (b + zv) * (b + zv);
    if (EXP == 0 && !quad) {
        one_minus_u = m_ncdf(-zv);
        vn = one_minus_u >= r1 ? R(0) : m_log(r1 / one_minus_u) * r2;
    }
    if (EXP == 1) {
        const R ve = one_minus_u >= r1 ? R(0) : m_log(r1 / one_minus_u) * r2;
        vn = quad ? vn : ve;
    }
    const R arg_q = R(1) - R(2) * c.A * r2;
    const R den_e = R(1) - c.A * r2;
    const R r3 = (quad ? -c.A * b2 * r2 : r1) / (quad ? arg_q : den_e);
    const R arg = quad ? arg_q : (R(1) - r1) + r3;
    const bool finite = quad ? arg_q > R(0) : den_e > R(0);
    const R lin = quad ? r3 : R(0);
    const R w = quad ? R(0.5) : R(-1);
    const R K0 = finite ? lin + w * m_log(arg) - (c.K1 + R(0.5) * c.K3) * v : c.K0p;
    y += c.mu_dt + K0 + c.K1 * v + c.K2 * vn + m_sqrt(m_max(c.K3 * v + c.K4 * vn, R(0))) * zx;
    v = vn;
}

template <typename R>
__device__ __forceinline__ void qe_step(const QeConsts<R>& c, R& y, R& v, R zv, R zx) {
    const R m = c.theta + (v - c.theta) * c.E;
    const R m2 = m * m, s2 = v * c.c1 + c.c2;
    qe_step_body<0>(c, y, v, zv, zx, m, m2, s2, s2 <= R(1.5) * m2);
}

// The same step for a warp whose 32 lanes all execute it together (none has left the loop): the warp votes. A warp
// with an exponential lane runs the straight-line copy in which every lane evaluates the exponential tail; a warp
// without one runs the quadratic step alone. The values are qe_step's bit for bit.
template <typename R>
__device__ __forceinline__ void qe_step_warp(const QeConsts<R>& c, R& y, R& v, R zv, R zx) {
    const R m = c.theta + (v - c.theta) * c.E;
    const R m2 = m * m, s2 = v * c.c1 + c.c2;
    const bool quad = s2 <= R(1.5) * m2;
    if (__any_sync(0xffffffffu, !quad)) qe_step_body<1>(c, y, v, zv, zx, m, m2, s2, quad);
    else qe_step_body<2>(c, y, v, zv, zx, m, m2, s2, true);
}

}  // namespace ob
