/* ORACLE — test infrastructure only. This file is a CPU restatement, in plain C and double precision, of the
 * reference's Monte Carlo path algorithms (Luca-CS/option-pricing-lab, packages/native/cuda = RC). Only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it, and only as the checker: the engine never calls
 * it and has no CPU fallback.
 *
 * Parity of this restatement is pinned two ways:
 *   - against the reference's own CPU engine, compiled from its sources by oracle/Makefile into oracle/_ref (tests in
 *     tests/test_oracle_vs_reference.py, run where the reference tree is present);
 *   - against the reference's golden vectors (tests/golden/native_cpu.json of the reference: Black-Scholes, Heston,
 *     local-vol and SLV path samples), restated as fixtures under tests/golden/ by tests/golden/make_fixtures.py.
 *
 * Each function cites the reference file:line it follows. Threads split the pairs into fixed blocks of 512 whose
 * partial sums are added in block order, so every result is independent of the thread count.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/optlab_b200.h"

#define OR_BLOCK 512

static char or_err[512];
const char* or_last_error(void) { return or_err; }
static int fail(const char* msg) {
    snprintf(or_err, sizeof or_err, "%s", msg);
    return OB_EINVAL;
}

/* ------------------------------------------------------------------------------------------- Philox4x32-10
 * RC/include/optlab_cuda/philox.hpp:22-44: ten rounds, multipliers 0xD2511F53 and 0xCD9E8D57, Weyl key bumps
 * 0x9E3779B9 and 0xBB67AE85. */
void or_philox(const uint32_t in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t x = in[0], y = in[1], z = in[2], w = in[3];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * x, p1 = (uint64_t)0xCD9E8D57u * z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t nx = hi1 ^ y ^ k0, nz = hi0 ^ w ^ k1;
        x = nx, y = lo1, z = nz, w = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = x, out[1] = y, out[2] = z, out[3] = w;
}

/* philox.hpp:45-49: u = (i + 1/2) 2^-32 */
static double to_unit(uint32_t i) { return (double)i * 2.3283064365386963e-10 + 1.1641532182693481e-10; }

/* philox.hpp:68-72 (the CPU branch): r = sqrt(-2 log u), angle 2 pi v */
static void box_muller(uint32_t a, uint32_t b, double* z0, double* z1) {
    const double u = to_unit(a), v = to_unit(b);
    const double r = sqrt(-2.0 * log(u));
    const double t = 6.283185307179586 * v;
    *z0 = r * cos(t), *z1 = r * sin(t);
}

/* paths.hpp:207-233: normals of one pair along one stream, block b -> normals 4b .. 4b+3; the aux stream sets the
 * top bit of the counter's last word. */
typedef struct {
    uint64_t pair;
    uint32_t k0, k1, tag;
    uint64_t block;
    double buf[4];
    int used;
} Stream;

static void stream_init(Stream* s, uint64_t pair, uint64_t seed, uint32_t tag) {
    s->pair = pair, s->k0 = (uint32_t)seed, s->k1 = (uint32_t)(seed >> 32), s->tag = tag, s->block = 0, s->used = 4;
}

static double stream_next(Stream* s) {
    if (s->used == 4) {
        const uint32_t c[4] = {(uint32_t)s->pair, (uint32_t)(s->pair >> 32), (uint32_t)s->block,
                               (uint32_t)(s->block >> 32) | s->tag};
        uint32_t r[4];
        or_philox(c, s->k0, s->k1, r);
        box_muller(r[0], r[1], &s->buf[0], &s->buf[1]);
        box_muller(r[2], r[3], &s->buf[2], &s->buf[3]);
        ++s->block, s->used = 0;
    }
    return s->buf[s->used++];
}

/* The known-answer surface of ob_philox_normals, on the CPU. */
int or_philox_normals(unsigned long long seed, long long first_pair, long long n_pairs, unsigned tag,
                      unsigned long long first_block, int n_blocks, unsigned* u32, double* z64) {
    for (long long p = 0; p < n_pairs; ++p)
        for (int b = 0; b < n_blocks; ++b) {
            const uint64_t pair = (uint64_t)(first_pair + p), blk = first_block + (uint64_t)b;
            const uint32_t c[4] = {(uint32_t)pair, (uint32_t)(pair >> 32), (uint32_t)blk, (uint32_t)(blk >> 32) | tag};
            uint32_t r[4];
            or_philox(c, (uint32_t)seed, (uint32_t)(seed >> 32), r);
            const long long o = (p * n_blocks + b) * 4;
            if (u32)
                for (int k = 0; k < 4; ++k) u32[o + k] = r[k];
            if (z64) {
                box_muller(r[0], r[1], &z64[o], &z64[o + 1]);
                box_muller(r[2], r[3], &z64[o + 2], &z64[o + 3]);
            }
        }
    return OB_OK;
}

/* ------------------------------------------------------------------------------------------- thread pool */

typedef void (*BlockFn)(const void* ctx, long long block, void* partial);

typedef struct {
    BlockFn fn;
    const void* ctx;
    long long n_blocks;
    char* partials;
    size_t partial_size;
    long long next;
    pthread_mutex_t mu;
} Pool;

static void* pool_worker(void* arg) {
    Pool* p = (Pool*)arg;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        const long long k = p->next++;
        pthread_mutex_unlock(&p->mu);
        if (k >= p->n_blocks) return NULL;
        p->fn(p->ctx, k, p->partials ? p->partials + (size_t)k * p->partial_size : NULL);
    }
}

static void run_blocks(BlockFn fn, const void* ctx, long long n_blocks, void* partials, size_t partial_size,
                       int n_threads) {
    Pool p = {fn, ctx, n_blocks, (char*)partials, partial_size, 0, PTHREAD_MUTEX_INITIALIZER};
    if (n_threads <= 1 || n_blocks <= 1) {
        pool_worker(&p);
        return;
    }
    if (n_threads > 256) n_threads = 256;
    pthread_t th[256];
    int started = 0;
    for (int t = 0; t < n_threads; ++t)
        if (pthread_create(&th[t], NULL, pool_worker, &p) == 0) ++started;
    if (!started) pool_worker(&p);
    for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------------------------- path engine
 * RC/include/optlab_cuda/paths.hpp:190-276 (simulate_pair) with the table read of :196-205 and the recording of
 * observations and windows of :241-272. Log-forward x per name, log-Euler spot step, full-truncation Euler
 * variance, correlation by `root`, an optional local-correlation mixer. */

typedef struct {
    int n_names, n_steps, n_x;
    uint64_t first_pair;
    uint64_t seed;
    const double *dt, *t0, *root, *cvar, *hes, *lo, *inv_dx, *table, *low_root;
    const int *kind, *step_row;
    int same, mixer;
    double mix[8];
} Model;

static double table_value(const Model* m, int row, double x) {
    double u = (x - m->lo[row]) * m->inv_dx[row];
    const double top = (double)(m->n_x - 1) - 1e-4;
    u = u > 0.0 ? u : 0.0;
    u = u < top ? u : top;
    const int i = (int)u;
    const double w = u - (double)i;
    const double* y = m->table + (long long)row * m->n_x;
    return y[i] * (1.0 - w) + y[i + 1] * w;
}

typedef struct {
    Stream rng, aux;
    double x[2][OB_MAX_NAMES], v[2][OB_MAX_NAMES];
    int has_var, has_slv;
} PairState;

static void pair_init(const Model* m, PairState* s, uint64_t pair) {
    s->has_var = s->has_slv = 0;
    for (int a = 0; a < m->n_names; ++a) {
        const int k = m->kind[a];
        const int hv = k == 2 || k == 3;
        s->has_var |= hv;
        s->has_slv |= k == 3;
        s->x[0][a] = s->x[1][a] = 0.0;
        s->v[0][a] = s->v[1][a] = hv ? m->hes[a * 5] : 0.0;
    }
    stream_init(&s->rng, pair, m->seed, 0u);
    stream_init(&s->aux, pair, m->seed, 0x80000000u);
}

/* paths.hpp:295-358: step i (1-based) of both legs */
static void pair_step(const Model* m, PairState* s, int i) {
    const int n = m->n_names;
    const double dt = m->dt[i - 1], t0 = m->t0[i - 1];
    double zs[OB_MAX_NAMES], zr[OB_MAX_NAMES], fresh = 0.0;
    for (int a = 0; a < n; ++a) zs[a] = stream_next(&s->rng);
    if (s->has_var)
        for (int a = 0; a < n; ++a) zr[a] = s->has_slv ? stream_next(&s->aux) : stream_next(&s->rng);
    if (m->mixer) fresh = stream_next(&s->rng);
    for (int leg = 0; leg < 2; ++leg) {
        const double sign = leg ? -1.0 : 1.0;
        double z[OB_MAX_NAMES], w[OB_MAX_NAMES];
        if (m->mixer) { /* paths.hpp:304-322 */
            double mm = 0.0;
            for (int a = 0; a < n; ++a) mm += exp(s->x[leg][a]);
            const double y = log(mm / (double)n);
            const double u = y / (m->mix[4] * sqrt(t0 > 1.0 / 12 ? t0 : 1.0 / 12));
            double wt = m->mix[0] + m->mix[1] + m->mix[2] * (-u > 0.0 ? -u : 0.0) - m->mix[3] * (u > 0.0 ? u : 0.0);
            wt = wt > 0.0 ? wt : 0.0;
            wt = wt < 1.0 ? wt : 1.0;
            const double market = m->mix[5] * sign * zs[n - 1], fr = sign * fresh;
            const double common = m->mix[6] * market + m->mix[7] * fr;
            double other[OB_MAX_NAMES];
            for (int a = 0; a < n; ++a) other[a] = sign * zs[a];
            other[n - 1] = m->mix[7] * market - m->mix[6] * fr;
            const double sw = sqrt(wt), sl = sqrt(1.0 - wt);
            for (int a = 0; a < n; ++a) {
                double acc = 0.0;
                for (int b = 0; b < n; ++b) acc += m->low_root[a * n + b] * other[b];
                z[a] = sw * common + sl * acc;
            }
        } else {
            for (int a = 0; a < n; ++a) {
                double acc = 0.0;
                for (int b = 0; b < n; ++b) acc += m->root[a * n + b] * zs[b];
                z[a] = sign * acc;
            }
        }
        if (s->has_var)
            for (int a = 0; a < n; ++a) {
                if (m->same) {
                    double acc = 0.0;
                    for (int b = 0; b < n; ++b) acc += m->root[a * n + b] * zr[b];
                    w[a] = sign * acc;
                } else {
                    w[a] = sign * zr[a];
                }
            }
        for (int a = 0; a < n; ++a) {
            const int k = m->kind[a];
            const double vp = s->v[leg][a] > 0.0 ? s->v[leg][a] : 0.0;
            double var;
            if (k == 0) var = m->cvar[a];
            else if (k == 2) var = vp;
            else {
                const double t = table_value(m, m->step_row[a * m->n_steps + (i - 1)], s->x[leg][a]);
                var = k == 1 ? t : t * vp;
            }
            if (k == 2 || k == 3) {
                const double* h = m->hes + a * 5;
                const double zv = h[4] * z[a] + sqrt(1.0 - h[4] * h[4]) * w[a];
                s->v[leg][a] += h[1] * (h[2] - vp) * dt + h[3] * sqrt(vp * dt) * zv;
            }
            s->x[leg][a] += -0.5 * var * dt + sqrt(var * dt) * z[a];
        }
    }
}

typedef struct {
    Model m;
    const ob_paths_request* rq;
} PathsCtx;

/* paths.hpp:241-272: spot columns and window extremes */
static void record(const ob_paths_request* rq, long long p, int j, const PairState* s, double lo[2][8][2],
                   double hi[2][8][2]) {
    const long long rows = 2 * rq->n_pairs;
    const long long r[2] = {p, rq->n_pairs + p};
    const int c = rq->col_of[j];
    for (int a = 0; a < rq->n_names; ++a) {
        const double f = rq->fwd[a * rq->n_obs + j];
        const double S[2] = {f * exp(s->x[0][a]), f * exp(s->x[1][a])};
        double* base = rq->out + (long long)a * rq->n_cols * rows;
        if (c >= 0) base[c * rows + r[0]] = S[0], base[c * rows + r[1]] = S[1];
        for (int w = 0; w < rq->n_windows; ++w) {
            if (j < rq->win_lo[w] || j > rq->win_hi[w]) continue;
            for (int leg = 0; leg < 2; ++leg) {
                if (j == rq->win_lo[w]) {
                    lo[leg][a][w] = hi[leg][a][w] = S[leg];
                } else {
                    lo[leg][a][w] = S[leg] < lo[leg][a][w] ? S[leg] : lo[leg][a][w];
                    hi[leg][a][w] = S[leg] > hi[leg][a][w] ? S[leg] : hi[leg][a][w];
                }
            }
            if (j == rq->win_hi[w]) {
                const long long cl = rq->n_keep + 2 * w, ch = cl + 1;
                for (int leg = 0; leg < 2; ++leg) {
                    base[cl * rows + r[leg]] = lo[leg][a][w];
                    base[ch * rows + r[leg]] = hi[leg][a][w];
                }
            }
        }
    }
}

static void paths_block(const void* vctx, long long blk, void* partial) {
    (void)partial;
    const PathsCtx* c = (const PathsCtx*)vctx;
    const ob_paths_request* rq = c->rq;
    const long long p0 = blk * OR_BLOCK, p1 = p0 + OR_BLOCK < rq->n_pairs ? p0 + OR_BLOCK : rq->n_pairs;
    for (long long p = p0; p < p1; ++p) {
        PairState s;
        double lo[2][8][2], hi[2][8][2];
        pair_init(&c->m, &s, c->m.first_pair + (uint64_t)p);
        int j = 0;
        while (j < rq->n_obs && rq->obs_step[j] == 0) record(rq, p, j++, &s, lo, hi);
        for (int i = 1; i <= rq->n_steps; ++i) {
            pair_step(&c->m, &s, i);
            while (j < rq->n_obs && rq->obs_step[j] == i) record(rq, p, j++, &s, lo, hi);
        }
    }
}

static Model model_of_paths(const ob_paths_request* rq) {
    Model m;
    memset(&m, 0, sizeof m);
    m.n_names = rq->n_names, m.n_steps = rq->n_steps, m.n_x = rq->n_x;
    m.first_pair = (uint64_t)rq->first_pair, m.seed = rq->seed;
    m.dt = rq->dt, m.t0 = rq->t0, m.root = rq->root, m.cvar = rq->cvar, m.hes = rq->heston;
    m.lo = rq->row_lo, m.inv_dx = rq->row_inv_dx, m.table = rq->table, m.low_root = rq->low_root;
    m.kind = rq->kind, m.step_row = rq->step_row, m.same = rq->same, m.mixer = rq->mixer;
    for (int k = 0; k < 8; ++k) m.mix[k] = rq->mix[k];
    return m;
}

/* Checks of RC/src/requests.cpp:168-207 (path_spec), restated. */
static int check_paths(const ob_paths_request* c) {
    if (c->n_names < 1 || c->n_names > OB_MAX_NAMES) return fail("n_names must be 1 to 8");
    if (c->n_pairs < 1 || c->first_pair < 0) return fail("n_pairs must be >= 1 and first_pair >= 0");
    if (c->n_steps < 0 || c->n_obs < 0) return fail("n_steps and n_obs must be >= 0");
    if (!c->out && c->n_obs > 0) return fail("null output");
    if (c->n_steps > 0 && (!c->dt || !c->t0)) return fail("null time grid");
    if (!c->root || !c->kind || !c->cvar || !c->heston || !c->fwd || (c->n_obs && !c->obs_step))
        return fail("null array");
    int table = 0;
    for (int a = 0; a < c->n_names; ++a) {
        const int k = c->kind[a];
        if (k < 0 || k > 3) return fail("kind must be 0 to 3");
        table |= k == 1 || k == 3;
        if ((k == 2 || k == 3) && !(c->heston[a * 5 + 1] > 0 && c->heston[a * 5 + 2] > 0 && c->heston[a * 5 + 3] >= 0 &&
                                    fabs(c->heston[a * 5 + 4]) <= 1))
            return fail("Heston parameters out of range");
    }
    if (table) {
        if (c->n_x < 2 || c->n_rows < 1 || !c->step_row || !c->row_lo || !c->row_inv_dx || !c->table)
            return fail("a tabulated variance needs n_x >= 2, rows and step_row");
        for (long long i = 0; i < (long long)c->n_names * c->n_steps; ++i) {
            const int k = c->kind[i / (c->n_steps ? c->n_steps : 1)];
            if ((k == 1 || k == 3) && (c->step_row[i] < 0 || c->step_row[i] >= c->n_rows))
                return fail("step_row out of range");
        }
    }
    int prev = 0;
    for (int j = 0; j < c->n_obs; ++j) {
        if (c->obs_step[j] < prev || c->obs_step[j] > c->n_steps)
            return fail("obs_step must be nondecreasing in [0, n_steps]");
        prev = c->obs_step[j];
    }
    if (c->mixer && (c->mixer != 1 || !c->low_root || !(c->mix[4] > 0))) return fail("bad local correlation");
    if (c->n_windows < 0 || c->n_windows > OB_MAX_WINDOWS || (c->n_windows && (!c->win_lo || !c->win_hi)))
        return fail("n_windows must be 0 to 2, with win_lo and win_hi");
    if (c->n_obs && !c->col_of) return fail("null col_of");
    if (c->n_keep < 0 || c->n_cols != c->n_keep + 2 * c->n_windows) return fail("n_cols must be n_keep + 2 n_windows");
    for (int j = 0; j < c->n_obs; ++j)
        if (c->col_of[j] < -1 || c->col_of[j] >= c->n_keep) return fail("col_of out of range");
    for (int w = 0; w < c->n_windows; ++w)
        if (c->win_lo[w] < 0 || c->win_hi[w] < c->win_lo[w] || c->win_hi[w] >= c->n_obs) return fail("bad window");
    return OB_OK;
}

int or_paths(ob_paths_request* rq, int n_threads) {
    const int st = check_paths(rq);
    if (st) return st;
    PathsCtx c = {model_of_paths(rq), rq};
    run_blocks(paths_block, &c, (rq->n_pairs + OR_BLOCK - 1) / OR_BLOCK, NULL, 0, n_threads);
    return OB_OK;
}

/* ------------------------------------------------------------------------------------------- Andersen QE-M
 * RC/include/optlab_cuda/schemes.hpp:107-141 (make_consts) and :153-186 (qe_step), for one step dt. */
typedef struct {
    double theta, mu_dt, E, c1, c2, K1, K2, K3, K4, A, K0p, v0;
} QeConsts;

static QeConsts qe_consts(const double* h, double r, double q, double dt) {
    const double v0 = h[0], kappa = h[1], theta = h[2], xi = h[3], rho = h[4];
    QeConsts c;
    const double E = exp(-kappa * dt), xi2 = xi * xi;
    const double k12 = 0.5 * dt * (kappa * rho / xi - 0.5);
    c.v0 = v0, c.theta = theta, c.mu_dt = (r - q) * dt, c.E = E;
    c.c1 = xi2 * E * (1 - E) / kappa;
    c.c2 = theta * xi2 * (1 - E) * (1 - E) / (2 * kappa);
    c.K1 = k12 - rho / xi;
    c.K2 = k12 + rho / xi;
    c.K3 = 0.5 * dt * (1 - rho * rho);
    c.K4 = c.K3;
    c.A = (k12 + rho / xi) + 0.25 * dt * (1 - rho * rho);
    c.K0p = -rho * kappa * theta * dt / xi;
    return c;
}

static double ncdf(double x) { return 0.5 * erfc(-x * 0.70710678118654752); }

static void qe_step(const QeConsts* c, double* y, double* v, double zv, double zx) {
    const double m = c->theta + (*v - c->theta) * c->E;
    const double psi = (*v * c->c1 + c->c2) / (m * m);
    double vn, lin, w, arg;
    int finite;
    if (psi <= 1.5) {
        const double inv = 2.0 / psi;
        const double b2 = inv - 1.0 + sqrt(inv) * sqrt(inv - 1.0 > 0.0 ? inv - 1.0 : 0.0);
        const double a = m / (1.0 + b2), b = sqrt(b2);
        vn = a * (b + zv) * (b + zv);
        arg = 1.0 - 2.0 * c->A * a;
        finite = c->A < 1.0 / (2.0 * a);
        lin = -c->A * b2 * a / arg;
        w = 0.5;
    } else {
        const double p = (psi - 1.0) / (psi + 1.0), beta = (1.0 - p) / m;
        const double one_minus_u = ncdf(-zv);
        vn = one_minus_u >= 1.0 - p ? 0.0 : log((1.0 - p) / one_minus_u) / beta;
        arg = p + beta * (1.0 - p) / (beta - c->A);
        finite = c->A < beta;
        lin = 0.0;
        w = -1.0;
    }
    const double K0 = finite ? lin + w * log(arg) - (c->K1 + 0.5 * c->K3) * *v : c->K0p;
    const double var = c->K3 * *v + c->K4 * vn;
    *y += c->mu_dt + K0 + c->K1 * *v + c->K2 * vn + sqrt(var > 0.0 ? var : 0.0) * zx;
    *v = vn;
}

/* ------------------------------------------------------------------------------------------- fused products
 * Ladder: payoffs at maturity, as RC/include/optlab_cuda/schemes.hpp:143-151 (leg_payoff) and
 * packages/core/src/optlab/core/products.py:82-102 (barrier_mc: hit = max S >= H up, min S <= H down, monitored at
 * every step end). Autocall: the script the term-sheet compiler writes for a Phoenix
 * (packages/structured/src/optlab/structured/compiler.py:114-127 coupon with memory, :141-161 knock-in redemption,
 * :271-280 call, :37-59 call dates = every coupon date but the last), for one name or the worst of several.
 * Each pair average y = (pay(z) + pay(-z)) / 2 goes into FP64 sums; price = mean, SE = the reference's
 * estimate_from_sums (RC/src/cpu_mc.cpp:8-12). */

#define N_SUMS (2 * OB_MAX_OUT)

typedef struct {
    const ob_mc_request* rq;
    Model m;
    QeConsts qe;
    int n_out;
    double ln_shift; /* a relative spot move ln(1 + move) on every performance, the start's included (0: none) */
    int sum_legs;    /* ladder: output 0 is the sum of the legs (the value of a trade made of them) */
} McCtx;

typedef struct {
    double s[N_SUMS];
} McPartial;

static double leg_payoff(int type, double S, double K) {
    switch (type) {
        case 1: return S > K ? S - K : 0.0;
        case 2: return K > S ? K - S : 0.0;
        case 3: return S - K;
        default: return 0.0;
    }
}

/* One leg of one pair through the product: the spot path of each name at grid point i is read through spot_at. */
typedef struct {
    double hi, lo;      /* ladder: running extremes of the underlying over step ends */
    double low_perf;    /* autocall: lowest worst-of performance over step ends */
    double pv, called, knocked, coupons;
    int missed, alive, next_obs;
} LegBook;

static void book_init(LegBook* b) {
    memset(b, 0, sizeof *b);
    b->hi = -INFINITY, b->lo = INFINITY, b->low_perf = 1.0, b->alive = 1;
}

/* Performance of the basket (worst of S_a / S0_a) at grid point i of one leg. */
static double worst_perf(const McCtx* c, const PairState* s, const double* y_qe, int leg, int i) {
    const ob_mc_request* rq = c->rq;
    if (rq->model == OB_MODEL_HESTON_QE) return exp(y_qe[leg] + c->ln_shift);
    double w = INFINITY;
    for (int a = 0; a < rq->n_names; ++a) {
        const double p = exp(rq->log_fwd[a * (rq->n_steps + 1) + i] + s->x[leg][a] + c->ln_shift);
        w = p < w ? p : w;
    }
    return w;
}

static void book_step(const McCtx* c, LegBook* b, double perf, int i) {
    const ob_mc_request* rq = c->rq;
    if (rq->product == OB_PRODUCT_LADDER) {
        const double U = rq->spot[0] * perf;
        b->hi = U > b->hi ? U : b->hi;
        b->lo = U < b->lo ? U : b->lo;
        return;
    }
    if (!b->alive) return;
    b->low_perf = perf < b->low_perf ? perf : b->low_perf;
    while (b->alive && b->next_obs < rq->n_obs && rq->obs_step[b->next_obs] == i) {
        const int j = b->next_obs++;
        const double D = rq->obs_discount[j];
        const int last = j == rq->n_obs - 1;
        if (rq->coupon > 0.0 || rq->coupon_barrier > 0.0) {
            if (perf >= rq->coupon_barrier) {
                const double k = rq->memory ? 1.0 + b->missed : 1.0;
                b->pv += D * rq->coupon * k, b->coupons += k, b->missed = 0;
            } else {
                ++b->missed;
            }
        }
        if (!last && rq->trigger[j] > 0.0 && perf >= rq->trigger[j]) {
            b->pv += D, b->called = 1.0, b->alive = 0;
        } else if (last) {
            const int ki = rq->ki_daily ? b->low_perf < rq->ki_barrier : perf < rq->ki_barrier;
            const double put = rq->put_strike - perf > 0.0 ? rq->put_strike - perf : 0.0;
            b->pv += D * (ki ? 1.0 - put : 1.0), b->knocked = ki, b->alive = 0;
        }
    }
}

static void book_outputs(const McCtx* c, const LegBook* b, double perf_T, double out[OB_MAX_OUT]) {
    const ob_mc_request* rq = c->rq;
    if (rq->product == OB_PRODUCT_LADDER) {
        const double U = rq->spot[0] * perf_T;
        for (int k = 0; k < rq->n_legs; ++k) {
            double pay = rq->discount * leg_payoff(rq->leg_type[k], U, rq->leg_strike[k]);
            const double H = rq->leg_level ? rq->leg_level[k] : 0.0;
            const int bt = rq->leg_barrier ? rq->leg_barrier[k] : 0;
            const int up_hit = b->hi >= H, down_hit = b->lo <= H;
            if (bt == OB_BARRIER_UP_OUT && up_hit) pay = 0.0;
            if (bt == OB_BARRIER_DOWN_OUT && down_hit) pay = 0.0;
            if (bt == OB_BARRIER_UP_IN && !up_hit) pay = 0.0;
            if (bt == OB_BARRIER_DOWN_IN && !down_hit) pay = 0.0;
            out[k] = pay;
        }
        out[rq->n_legs] = U;
        return;
    }
    out[0] = b->pv, out[1] = b->called, out[2] = b->knocked, out[3] = b->coupons;
}

static void mc_block(const void* vctx, long long blk, void* vpartial) {
    const McCtx* c = (const McCtx*)vctx;
    const ob_mc_request* rq = c->rq;
    McPartial* part = (McPartial*)vpartial;
    memset(part, 0, sizeof *part);
    const long long p0 = blk * OR_BLOCK, p1 = p0 + OR_BLOCK < rq->n_pairs ? p0 + OR_BLOCK : rq->n_pairs;
    for (long long p = p0; p < p1; ++p) {
        const uint64_t pair = (uint64_t)(rq->first_pair + p);
        PairState s;
        double y[2] = {0.0, 0.0}, v[2];
        LegBook book[2];
        book_init(&book[0]), book_init(&book[1]);
        book[0].low_perf = book[1].low_perf = exp(c->ln_shift);
        if (rq->model == OB_MODEL_HESTON_QE) {
            stream_init(&s.rng, pair, rq->seed, 0u);
            v[0] = v[1] = c->qe.v0;
        } else {
            pair_init(&c->m, &s, pair);
        }
        for (int i = 1; i <= rq->n_steps; ++i) {
            if (rq->model == OB_MODEL_HESTON_QE) {
                /* RC/include/optlab_cuda/schemes.hpp:212-227: zv then zx, both signs flipped on the second leg */
                const double zv = stream_next(&s.rng), zx = stream_next(&s.rng);
                qe_step(&c->qe, &y[0], &v[0], zv, zx);
                qe_step(&c->qe, &y[1], &v[1], -zv, -zx);
            } else {
                pair_step(&c->m, &s, i);
            }
            for (int leg = 0; leg < 2; ++leg) book_step(c, &book[leg], worst_perf(c, &s, y, leg, i), i);
        }
        double o0[OB_MAX_OUT], o1[OB_MAX_OUT];
        book_outputs(c, &book[0], worst_perf(c, &s, y, 0, rq->n_steps), o0);
        book_outputs(c, &book[1], worst_perf(c, &s, y, 1, rq->n_steps), o1);
        if (c->sum_legs && rq->product == OB_PRODUCT_LADDER) {
            double t0 = 0.0, t1 = 0.0;
            for (int k = 0; k < rq->n_legs; ++k) t0 += o0[k], t1 += o1[k];
            o0[0] = t0, o1[0] = t1;
        }
        for (int k = 0; k < c->n_out; ++k) {
            const double a = 0.5 * (o0[k] + o1[k]);
            part->s[k] += a, part->s[OB_MAX_OUT + k] += a * a;
        }
    }
}

static int check_mc(const ob_mc_request* rq) {
    if (rq->model != OB_MODEL_PATHS && rq->model != OB_MODEL_HESTON_QE) return fail("model must be 0 or 1");
    if (rq->n_names < 1 || rq->n_names > OB_MAX_NAMES) return fail("n_names must be 1 to 8");
    if (rq->model == OB_MODEL_HESTON_QE && rq->n_names != 1) return fail("the QE model has one name");
    if (rq->n_pairs < 2 || rq->first_pair < 0) return fail("n_pairs must be >= 2 and first_pair >= 0");
    if (rq->n_steps < 1 || !rq->dt || !rq->t0 || !rq->spot) return fail("null time grid or spot");
    if (rq->product == OB_PRODUCT_LADDER) {
        if (rq->n_legs < 1 || rq->n_legs > OB_MAX_OUT - 1 || !rq->leg_type || !rq->leg_strike)
            return fail("ladder: n_legs must be 1 to 31 with leg_type and leg_strike");
    } else if (rq->product == OB_PRODUCT_AUTOCALL) {
        if (rq->n_obs < 1 || !rq->obs_step || !rq->obs_discount || !rq->trigger) return fail("autocall: null schedule");
        for (int j = 0; j < rq->n_obs; ++j)
            if (rq->obs_step[j] < 1 || rq->obs_step[j] > rq->n_steps || (j && rq->obs_step[j] <= rq->obs_step[j - 1]))
                return fail("obs_step must be increasing in [1, n_steps]");
    } else {
        return fail("product must be 0 or 1");
    }
    if (rq->mixer && (rq->model != OB_MODEL_PATHS || rq->mixer != 1 || !rq->low_root || !(rq->mix[4] > 0)))
        return fail("bad local correlation");
    if (rq->model == OB_MODEL_PATHS) {
        if (!rq->root || !rq->kind || !rq->cvar || !rq->heston || !rq->log_fwd) return fail("null array");
        for (int a = 0; a < rq->n_names; ++a) {
            const int k = rq->kind[a];
            if (k < 0 || k > 3) return fail("kind must be 0 to 3");
            if ((k == 1 || k == 3) && (rq->n_x < 2 || rq->n_rows < 1 || !rq->step_row || !rq->table))
                return fail("a tabulated variance needs n_x >= 2, rows and step_row");
            if (k == 1 || k == 3)
                for (int i = 0; i < rq->n_steps; ++i)
                    if (rq->step_row[a * rq->n_steps + i] < 0 || rq->step_row[a * rq->n_steps + i] >= rq->n_rows)
                        return fail("step_row out of range");
        }
    } else {
        if (!rq->heston) return fail("null heston");
        for (int i = 1; i < rq->n_steps; ++i)
            if (fabs(rq->dt[i] - rq->dt[0]) > 1e-9 * rq->dt[0]) return fail("the QE model needs uniform steps");
    }
    return OB_OK;
}

static int mc_price_shifted(const ob_mc_request* rq, double ln_shift, int sum_legs, int n_threads,
                            ob_mc_result* res) {
    const int st = check_mc(rq);
    if (st) return st;
    McCtx c;
    memset(&c, 0, sizeof c);
    c.rq = rq;
    c.ln_shift = ln_shift;
    c.sum_legs = sum_legs;
    c.n_out = rq->product == OB_PRODUCT_LADDER ? rq->n_legs + 1 : 4;
    if (rq->model == OB_MODEL_HESTON_QE) {
        c.qe = qe_consts(rq->heston, rq->r, rq->q, rq->dt[0]);
    } else {
        c.m.n_names = rq->n_names, c.m.n_steps = rq->n_steps, c.m.n_x = rq->n_x, c.m.seed = rq->seed;
        c.m.dt = rq->dt, c.m.t0 = rq->t0, c.m.root = rq->root, c.m.cvar = rq->cvar, c.m.hes = rq->heston;
        c.m.lo = rq->row_lo, c.m.inv_dx = rq->row_inv_dx, c.m.table = rq->table, c.m.kind = rq->kind;
        c.m.step_row = rq->step_row, c.m.same = rq->same;
        c.m.mixer = rq->mixer, c.m.low_root = rq->low_root;
        for (int k = 0; k < 8; ++k) c.m.mix[k] = rq->mix[k];
    }
    const long long n_blocks = (rq->n_pairs + OR_BLOCK - 1) / OR_BLOCK;
    McPartial* parts = (McPartial*)calloc((size_t)n_blocks, sizeof(McPartial));
    if (!parts) return fail("out of memory");
    run_blocks(mc_block, &c, n_blocks, parts, sizeof(McPartial), n_threads);
    double tot[N_SUMS] = {0};
    for (long long b = 0; b < n_blocks; ++b)
        for (int k = 0; k < N_SUMS; ++k) tot[k] += parts[b].s[k];
    free(parts);
    memset(res, 0, sizeof *res);
    res->n_out = c.n_out;
    res->n_paths = 2 * rq->n_pairs;
    const double n = (double)rq->n_pairs;
    for (int k = 0; k < c.n_out; ++k) {
        const double mean = tot[k] / n, var = tot[OB_MAX_OUT + k] / n - mean * mean;
        res->price[k] = mean;
        res->se[k] = rq->n_pairs > 1 ? sqrt(fmax(var, 0.0) / (n - 1.0)) : 0.0;
        res->sum_y[k] = tot[k], res->sum_y2[k] = tot[OB_MAX_OUT + k];
    }
    return OB_OK;
}

int or_mc_price(const ob_mc_request* rq, int n_threads, ob_mc_result* res) {
    return mc_price_shifted(rq, 0.0, 0, n_threads, res);
}

/* ------------------------------------------------------------------------------------------- batched revaluation
 * One trade of an ob_batch_request under each of its scenarios, every scenario its own simulation on the trade's
 * seed: the trade as an ob_mc_request (spot 1, so that strikes and levels are fractions of the initial spot), a spot
 * move as a shift ln(1 + move) of every performance (the reference's path factors, packages/risk/src/optlab/risk/
 * engine.py:585-590), a vol move as the local-variance rows rebuilt as (max(sigma + shift + tilt k, 0.01))^2 at each
 * node k, the Heston model unmoved by it (its parameters do not depend on the surface,
 * packages/structured/src/optlab/structured/context.py:163-164), a carry move as the log-forward rebuilt with
 * r + carry_rate and q + carry_div and every payment at time t discounted by exp(-carry_rate t) more (the forward
 * ratio and discount move of packages/risk/src/optlab/risk/engine.py:8-11 and curves.py:109-112; a Heston trade's
 * drift moves the same way), a correlation move as the trade's moved root (multi-name local vol; the others do not
 * move). price and se: 1 + n_spot + n_carry + n_vol + n_corr values, in that order. */
int or_batch_trade(const ob_batch_request* b, int trade, int n_threads, double* price, double* se) {
    if (!b || trade < 0 || trade >= b->n_trades || !price || !se) return fail("bad batch trade");
    const ob_batch_trade* t = &b->trades[trade];
    const int S = t->n_steps, N = t->n_names, E = b->n_exp, X = b->n_x;
    const int lv = t->model == OB_MODEL_PATHS;
    double* dt = (double*)malloc(sizeof(double) * S);
    double* t0 = (double*)malloc(sizeof(double) * S);
    double* lf = (double*)malloc(sizeof(double) * N * (S + 1));
    int* step_row = (int*)malloc(sizeof(int) * N * S);
    double* odisc = (double*)malloc(sizeof(double) * (t->product == OB_PRODUCT_AUTOCALL ? t->n_obs : 1));
    double* table = (double*)malloc(sizeof(double) * (lv ? N * E * X : 1));
    double* lo = (double*)malloc(sizeof(double) * N * E);
    double* inv = (double*)malloc(sizeof(double) * N * E);
    double spot[OB_MAX_NAMES], cvar[OB_MAX_NAMES], hes[5 * OB_MAX_NAMES];
    int kind[OB_MAX_NAMES];
    if (!dt || !t0 || !lf || !step_row || !odisc || !table || !lo || !inv) return fail("out of memory");
    for (int i = 0; i < S; ++i) {
        dt[i] = b->dt, t0[i] = i * b->dt;
        int j = 0;
        while (j < E - 1 && b->horizon * (j + 1) / E <= t0[i] + 1e-12) ++j;
        for (int a = 0; a < N; ++a) step_row[a * S + i] = a * E + j;
    }
    for (int a = 0; a < N; ++a) {
        spot[a] = 1.0, cvar[a] = 0.0, kind[a] = 1;
        for (int k = 0; k < 5; ++k) hes[5 * a + k] = t->heston[k];
        for (int i = 0; i <= S; ++i) lf[a * (S + 1) + i] = (t->r - t->q) * (i * b->dt);
        if (lv)
            for (int e = 0; e < E; ++e) lo[a * E + e] = b->row_lo[t->table_row0 + a * E + e],
                                        inv[a * E + e] = b->row_inv_dx[t->table_row0 + a * E + e];
    }
    ob_mc_request rq;
    memset(&rq, 0, sizeof rq);
    rq.model = t->model, rq.n_names = N, rq.n_steps = S, rq.n_pairs = t->n_pairs, rq.seed = t->seed;
    rq.dt = dt, rq.t0 = t0, rq.spot = spot, rq.heston = hes, rq.r = t->r, rq.q = t->q;
    if (lv) {
        rq.root = b->root + t->root0, rq.kind = kind, rq.cvar = cvar, rq.same = 0, rq.log_fwd = lf;
        rq.n_x = X, rq.n_rows = N * E, rq.step_row = step_row, rq.row_lo = lo, rq.row_inv_dx = inv, rq.table = table;
    }
    rq.product = t->product;
    if (t->product == OB_PRODUCT_LADDER) {
        rq.n_legs = t->n_legs, rq.leg_type = b->leg_type + t->leg0, rq.leg_strike = b->leg_strike + t->leg0;
        rq.leg_barrier = b->leg_barrier + t->leg0, rq.leg_level = b->leg_level + t->leg0;
        rq.discount = t->discount;
    } else {
        rq.n_obs = t->n_obs, rq.obs_step = b->obs_step + t->obs0, rq.obs_discount = b->obs_discount + t->obs0;
        rq.trigger = b->obs_trigger + t->obs0, rq.coupon_barrier = t->coupon_barrier, rq.coupon = t->coupon;
        rq.ki_barrier = t->ki_barrier, rq.put_strike = t->put_strike, rq.memory = t->memory;
        rq.ki_daily = t->ki_daily;
    }
    int st = OB_OK;
    const int n_sc = 1 + b->n_spot + b->n_carry + b->n_vol + b->n_corr;
    for (int sc = 0; sc < n_sc && st == OB_OK; ++sc) {
        const int c0 = 1 + b->n_spot, v0 = c0 + b->n_carry, r0 = v0 + b->n_vol;
        const int carry = sc >= c0 && sc < v0 ? sc - c0 : -1;
        const int vol = sc >= v0 && sc < r0 ? sc - v0 : -1;
        const int corr = sc >= r0 ? sc - r0 : -1;
        if ((vol >= 0 && !lv) || (corr >= 0 && (!lv || N < 2))) { /* a move the trade's model does not see */
            price[sc] = price[0], se[sc] = se[0];
            continue;
        }
        const double dr = carry >= 0 ? b->carry_rate[carry] : 0.0, dq = carry >= 0 ? b->carry_div[carry] : 0.0;
        rq.r = t->r + dr, rq.q = t->q + dq;
        for (int a = 0; a < N; ++a)
            for (int i = 0; i <= S; ++i) lf[a * (S + 1) + i] = (rq.r - rq.q) * (i * b->dt);
        if (lv) rq.root = b->root + (corr >= 0 ? t->corr_root0 + corr * N * N : t->root0);
        if (t->product == OB_PRODUCT_LADDER) {
            rq.discount = t->discount * exp(-dr * S * b->dt);
        } else {
            for (int j = 0; j < t->n_obs; ++j)
                odisc[j] = b->obs_discount[t->obs0 + j] * exp(-dr * b->obs_step[t->obs0 + j] * b->dt);
            rq.obs_discount = odisc;
        }
        if (lv)
            for (int r = 0; r < N * E; ++r) {
                const double* src = b->table + (size_t)(t->table_row0 + r) * X;
                const double* moved = vol >= 0 ? b->vol_table + ((size_t)vol * b->n_rows + t->table_row0 + r) * X : src;
                for (int k = 0; k < X; ++k) table[(size_t)r * X + k] = moved[k];
            }
        const double shift = sc >= 1 && sc <= b->n_spot ? log1p(b->spot_shift[sc - 1]) : 0.0;
        ob_mc_result res;
        st = mc_price_shifted(&rq, shift, 1, n_threads, &res);
        if (st == OB_OK) price[sc] = res.price[0], se[sc] = res.se[0];
    }
    free(dt), free(t0), free(lf), free(step_row), free(odisc), free(table), free(lo), free(inv);
    return st;
}

/* ------------------------------------------------------------------------------------------- fixed products
 * RC/include/optlab_cuda/schemes.hpp:188-245 (bs_european_unit, path_unit) with the engine's Philox normals: unit
 * (antithetic pair) p reads stream 0 of pair p, one normal per step under Black-Scholes, (zv, zx) under Heston. */
typedef struct {
    const ob_request* rq;
    QeConsts qe;
    double S0, D, bs_drift, bs_vol, ln_h, inv_n;
} FixedCtx;

static void fixed_block(const void* vctx, long long blk, void* vpartial) {
    const FixedCtx* c = (const FixedCtx*)vctx;
    const ob_request* rq = c->rq;
    double* part = (double*)vpartial;
    memset(part, 0, 8 * sizeof(double));
    const long long n_units = rq->n_paths / 2;
    const long long p0 = blk * OR_BLOCK, p1 = p0 + OR_BLOCK < n_units ? p0 + OR_BLOCK : n_units;
    for (long long p = p0; p < p1; ++p) {
        Stream s;
        stream_init(&s, (uint64_t)p, rq->seed, 0u);
        double y[2] = {0, 0}, v[2] = {c->qe.v0, c->qe.v0}, sum_s[2] = {0, 0}, sum_y[2] = {0, 0};
        int alive[2] = {1, 1};
        const int steps = rq->product == 0 && rq->model == 0 ? 1 : rq->n_steps;
        for (int i = 0; i < steps; ++i) {
            double zv = 0.0, zx;
            if (rq->model == 1) zv = stream_next(&s);
            zx = stream_next(&s);
            for (int a = 0; a < 2; ++a) {
                const double sg = a ? -1.0 : 1.0;
                if (rq->model == 1) qe_step(&c->qe, &y[a], &v[a], sg * zv, sg * zx);
                else if (rq->product == 0) y[a] = c->bs_drift + c->bs_vol * sg * zx; /* one exact step, :188-198 */
                else y[a] += c->bs_drift + c->bs_vol * sg * zx;
                if (rq->product == 1) sum_s[a] += exp(y[a]), sum_y[a] += y[a];
                if (rq->product == 2) alive[a] = alive[a] && !(y[a] <= c->ln_h);
            }
        }
        double o[4] = {0, 0, 0, 0};
        for (int a = 0; a < 2; ++a) {
            const double S = c->S0 * exp(y[a]);
            if (rq->product == 0) {
                for (int k = 0; k < 3; ++k) o[k] += c->D * leg_payoff(rq->legs[k], S, rq->strikes[k]);
            } else if (rq->product == 1) {
                o[0] += c->D * leg_payoff(rq->legs[0], c->S0 * sum_s[a] * c->inv_n, rq->strikes[0]);
                o[1] += c->D * leg_payoff(rq->legs[0], c->S0 * exp(sum_y[a] * c->inv_n), rq->strikes[0]);
            } else {
                const double pay = c->D * leg_payoff(rq->legs[0], S, rq->strikes[0]);
                o[0] += alive[a] ? pay : 0.0;
                o[1] += pay;
            }
            o[3] += S;
        }
        for (int k = 0; k < 4; ++k) {
            const double yk = 0.5 * o[k];
            part[k] += yk, part[4 + k] += yk * yk;
        }
    }
}

/* RC/src/requests.cpp:140-165 (convert): the checks, restated. */
int or_price(const ob_request* rq, int n_threads, ob_result* res) {
    if (rq->model < 0 || rq->model > 1) return fail("model must be 0 (Black-Scholes) or 1 (Heston)");
    if (rq->product < 0 || rq->product > 2) return fail("product must be 0, 1 or 2");
    if (rq->n_steps < 1) return fail("n_steps must be >= 1");
    if (rq->n_paths < 4 || rq->n_paths % 2) return fail("n_paths must be even and >= 4");
    if (!(rq->S0 > 0 && rq->T > 0)) return fail("S0 and T must be positive");
    if (rq->model == 0 && !(rq->sigma > 0)) return fail("sigma must be positive");
    if (rq->model == 1 && !(rq->v0 >= 0 && rq->kappa > 0 && rq->theta > 0 && rq->xi > 0 && fabs(rq->rho) <= 1))
        return fail("Heston parameters out of range");
    if (rq->product == 2 && !(rq->H > 0 && rq->H < rq->S0)) return fail("barrier: need 0 < H < S0");
    for (int k = 0; k < 3; ++k)
        if (rq->legs[k] < 0 || rq->legs[k] > 3) return fail("legs must be 0 to 3");
    FixedCtx c;
    memset(&c, 0, sizeof c);
    c.rq = rq;
    const double dt = rq->T / rq->n_steps;
    const double h[5] = {rq->v0, rq->kappa, rq->theta, rq->xi, rq->rho};
    if (rq->model == 1) c.qe = qe_consts(h, rq->r, rq->q, dt);
    c.S0 = rq->S0, c.D = exp(-rq->r * rq->T);
    c.bs_drift = (rq->r - rq->q - 0.5 * rq->sigma * rq->sigma) * dt;
    c.bs_vol = rq->sigma * sqrt(dt);
    c.ln_h = log(rq->H / rq->S0);
    c.inv_n = 1.0 / rq->n_steps;
    const long long n_units = rq->n_paths / 2, n_blocks = (n_units + OR_BLOCK - 1) / OR_BLOCK;
    double* parts = (double*)calloc((size_t)n_blocks * 8, sizeof(double));
    if (!parts) return fail("out of memory");
    run_blocks(fixed_block, &c, n_blocks, parts, 8 * sizeof(double), n_threads);
    double tot[8] = {0};
    for (long long b = 0; b < n_blocks; ++b)
        for (int k = 0; k < 8; ++k) tot[k] += parts[b * 8 + k];
    free(parts);
    memset(res, 0, sizeof *res);
    const double n = (double)n_units;
    for (int k = 0; k < 4; ++k) {
        const double mean = tot[k] / n, var = tot[4 + k] / n - mean * mean;
        res->price[k] = mean, res->se[k] = sqrt(fmax(var, 0.0) / (n - 1.0));
    }
    res->n_paths = rq->n_paths;
    return OB_OK;
}

/* ------------------------------------------------------------------------------------------- SLV leverage
 * RC/src/leverage.cpp:17-97 (calibrate_leverage, quantile, interp_uniform) with the particle device of :109-159
 * (CpuParticles::bin and ::step) on one thread: the bins are summed in particle order, so the result is the
 * reference's on n_threads = 1. */

static double interp_uniform(double x, double a, double b, const double* y, int n) {
    double u = (x - a) / (b - a) * (n - 1);
    if (!(u > 0)) return y[0];
    if (u >= n - 1) return y[n - 1];
    const int i = (int)u;
    const double w = u - i;
    return y[i] * (1 - w) + y[i + 1] * w;
}

static double quantile(const long long* fine, int nf, double lo, double hi, double q) {
    long long total = 0;
    for (int k = 0; k < nf; ++k) total += fine[k];
    const double target = q * (double)total;
    const double width = (hi - lo) / (double)nf;
    double cum = 0;
    for (int k = 0; k < nf; ++k) {
        const double next = cum + (double)fine[k];
        if (next >= target && fine[k] > 0) return lo + ((double)k + (target - cum) / fine[k]) * width;
        cum = next;
    }
    return hi;
}

int or_leverage(ob_leverage_request* s) {
    if (!s->dt || !s->t0 || !s->lv_lo || !s->lv_inv_dx || !s->lv_rows || !s->x_grids || !s->values)
        return fail("null pointer");
    if (s->n_steps < 1 || s->n_pairs < 2 || s->n_x < 2 || s->n_bins < 2 || s->n_fine < 16 || s->n_lv < 2)
        return fail("n_steps, n_pairs, n_x, n_bins, n_fine or n_lv too small");
    if (!(s->kappa > 0 && s->theta > 0 && s->xi >= 0 && fabs(s->rho) <= 1 && s->v0 >= 0))
        return fail("Heston parameters out of range");
    const int nx = s->n_x, nb = s->n_bins, nf = s->n_fine;
    const long long np = s->n_pairs, n = 2 * np;
    const double n_particles = 2.0 * (double)np;
    double* x = (double*)calloc((size_t)n, sizeof(double));
    double* v = (double*)malloc((size_t)n * sizeof(double));
    long long* fine = (long long*)malloc((size_t)nf * sizeof(long long));
    double* acc = (double*)malloc((size_t)5 * nb * sizeof(double));
    double *x_eval = (double*)malloc(nx * sizeof(double)), *cond = (double*)malloc(nx * sizeof(double));
    double *lev = (double*)malloc(nx * sizeof(double)), *centres = (double*)malloc(nb * sizeof(double));
    if (!x || !v || !fine || !acc || !x_eval || !cond || !lev || !centres) {
        free(x), free(v), free(fine), free(acc), free(x_eval), free(cond), free(lev), free(centres);
        return fail("out of memory");
    }
    for (long long j = 0; j < n; ++j) v[j] = s->v0;
    const uint32_t k0 = (uint32_t)s->seed, k1 = (uint32_t)(s->seed >> 32);
    const double rc = sqrt(1 - s->rho * s->rho);
    double lo = 0, hi = 0;
    for (int i = 0; i < s->n_steps; ++i) {
        const double t0 = s->t0[i], h = s->dt[i];
        if (i == 0) {
            for (int g = 0; g < nx; ++g) {
                x_eval[g] = (-6.0 + 12.0 * g / (nx - 1)) * s->atm_vol * sqrt(h > 1e-4 ? h : 1e-4);
                cond[g] = s->v0;
            }
        } else {
            /* bin (leverage.cpp:164-187) */
            memset(fine, 0, (size_t)nf * sizeof(long long));
            memset(acc, 0, (size_t)5 * nb * sizeof(double));
            double v_sum = 0.0;
            const double wf = (hi - lo) / nf, we = (hi + 1e-12 - lo) / nb;
            for (long long j = 0; j < n; ++j) {
                const double xj = x[j], vj = s->positive_part ? (v[j] > 0.0 ? v[j] : 0.0) : v[j];
                int f = wf > 0 ? (int)((xj - lo) / wf) : 0;
                f = f < 0 ? 0 : (f > nf - 1 ? nf - 1 : f);
                fine[f] += 1;
                int k = (int)((xj - lo) / we);
                k = k < 0 ? 0 : (k > nb - 1 ? nb - 1 : k);
                acc[k] += 1, acc[nb + k] += vj, acc[2 * nb + k] += xj, acc[3 * nb + k] += xj * xj;
                acc[4 * nb + k] += xj * vj;
                v_sum += vj;
            }
            /* regression (leverage.cpp:116-139) */
            const double a = quantile(fine, nf, lo, hi, s->q_lo), b = quantile(fine, nf, lo, hi, s->q_hi);
            for (int g = 0; g < nx; ++g) x_eval[g] = a + (b - a) * g / (nx - 1);
            const double bw = s->bandwidth_scale * s->atm_vol * sqrt(t0 > 0.15 ? t0 : 0.15) * pow(n_particles, -0.2);
            const double wc = (hi + 1e-12 - lo) / nb;
            for (int k = 0; k < nb; ++k) centres[k] = lo + (k + 0.5) * wc;
            const double fallback = v_sum / n_particles;
            const double *cnt = acc, *sv = cnt + nb, *sx = sv + nb, *sxx = sx + nb, *sxv = sxx + nb;
            for (int g = 0; g < nx; ++g) {
                double S0 = 0, T0 = 0, Ax = 0, Axx = 0, Axv = 0;
                const double x0 = x_eval[g];
                for (int k = 0; k < nb; ++k) {
                    const double d = (x0 - centres[k]) / bw, w = exp(-0.5 * d * d);
                    S0 += w * cnt[k], T0 += w * sv[k];
                    if (s->local_linear) Ax += w * sx[k], Axx += w * sxx[k], Axv += w * sxv[k];
                }
                const double nw = S0 > 1e-8 ? T0 / (S0 > 1e-300 ? S0 : 1e-300) : fallback;
                cond[g] = nw;
                if (s->local_linear) {
                    const double S1 = Ax - x0 * S0, S2 = Axx - 2 * x0 * Ax + x0 * x0 * S0, T1 = Axv - x0 * T0;
                    const double det = S0 * S2 - S1 * S1;
                    const int ok = S0 >= 50 && det > 1e-12 * S0 * fabs(S2);
                    const double llv = ok ? (S2 * T0 - S1 * T1) / det : nw;
                    cond[g] = llv > 1e-8 ? llv : 1e-8;
                }
            }
        }
        /* leverage row (leverage.cpp:141-148) */
        const double* row = s->lv_rows + (long long)i * s->n_lv;
        const double lv_lo = s->lv_lo[i], lv_hi = lv_lo + (s->n_lv - 1) / s->lv_inv_dx[i];
        for (int g = 0; g < nx; ++g) {
            const double loc = interp_uniform(x_eval[g], lv_lo, lv_hi, row, s->n_lv);
            double L = sqrt(loc / (cond[g] > 1e-8 ? cond[g] : 1e-8));
            L = L > s->l_min ? L : s->l_min;
            L = L < s->l_max ? L : s->l_max;
            lev[g] = L;
            s->x_grids[(long long)i * nx + g] = x_eval[g];
            s->values[(long long)i * nx + g] = L;
        }
        /* step (leverage.cpp:189-214) */
        double mn = INFINITY, mx = -INFINITY;
        const double ea = x_eval[0], eb = x_eval[nx - 1];
        for (long long p = 0; p < np; ++p) {
            const uint32_t c[4] = {(uint32_t)p, (uint32_t)((uint64_t)p >> 32), (uint32_t)(i + 1), 0u};
            uint32_t r[4];
            double z[4];
            or_philox(c, k0, k1, r);
            box_muller(r[0], r[1], &z[0], &z[1]);
            box_muller(r[2], r[3], &z[2], &z[3]);
            for (int leg = 0; leg < 2; ++leg) {
                const long long j = leg ? np + p : p;
                const double sg = leg ? -1.0 : 1.0, z1 = sg * z[0], z2 = sg * z[1];
                const double L = interp_uniform(x[j], ea, eb, lev, nx);
                const double vp = v[j] > 0.0 ? v[j] : 0.0, var = L * L * vp;
                const double zx = s->rho * z2 + rc * z1;
                v[j] += s->kappa * (s->theta - vp) * h + s->xi * sqrt(vp * h) * z2;
                x[j] += -0.5 * var * h + sqrt(var * h) * zx;
                mn = x[j] < mn ? x[j] : mn, mx = x[j] > mx ? x[j] : mx;
            }
        }
        lo = mn, hi = mx;
    }
    free(x), free(v), free(fine), free(acc), free(x_eval), free(cond), free(lev), free(centres);
    return OB_OK;
}

/* ------------------------------------------------------------------------------------------- smoothed autocall
 * The autocall above with its digitals smoothed as the reference's script evaluator does for Greeks
 * (packages/structured/src/optlab/structured/script/evaluator.py:93-107, 185-220): a >= b becomes
 * clip((a - b) / (eps |b|) + 1/2, 0, 1), a < b clip((b - a) / (eps |b|) + 1/2, 0, 1); inside an `if` a payment is
 * weighted by the mask times the alive mass, an assignment becomes m e + (1 - m) old, and `terminate` multiplies the
 * alive mass by 1 - m. Price only, on the path engine's local vol (or any kind), for the adjoint's checks. */

static double ramp_ge(double a, double b, double eps) {
    if (eps <= 0.0) return a >= b ? 1.0 : 0.0;
    const double t = (a - b) / (eps * fabs(b)) + 0.5;
    return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
}
static double ramp_lt(double a, double b, double eps) {
    if (eps <= 0.0) return a < b ? 1.0 : 0.0;
    const double t = (b - a) / (eps * fabs(b)) + 0.5;
    return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
}

static double smooth_leg(const ob_mc_request* rq, double eps, const double* perf, double low) {
    double pv = 0.0, alive = 1.0, missed = 0.0;
    const int has_coupon = rq->coupon > 0.0 || rq->coupon_barrier > 0.0;
    for (int j = 0; j < rq->n_obs; ++j) {
        const double p = perf[j], D = rq->obs_discount[j];
        if (has_coupon) {
            const double c = ramp_ge(p, rq->coupon_barrier, eps);
            const double mult = rq->memory ? 1.0 + missed : 1.0;
            pv += D * rq->coupon * mult * c * alive;
            missed = rq->memory ? (1.0 - c) * (missed + 1.0) : 0.0;
        }
        if (j < rq->n_obs - 1) {
            const double q = rq->trigger[j] > 0.0 ? ramp_ge(p, rq->trigger[j], eps) : 0.0;
            pv += D * q * alive;
            alive *= 1.0 - q;
        } else {
            const double k = ramp_lt(rq->ki_daily ? low : p, rq->ki_barrier, eps);
            const double put = rq->put_strike - p > 0.0 ? rq->put_strike - p : 0.0;
            pv += D * alive * (1.0 - k * put);
        }
    }
    return pv;
}

typedef struct {
    const ob_mc_request* rq;
    Model m;
    double eps;
} SmoothCtx;

static void smooth_block(const void* vctx, long long blk, void* vpartial) {
    const SmoothCtx* c = (const SmoothCtx*)vctx;
    const ob_mc_request* rq = c->rq;
    double* part = (double*)vpartial;
    part[0] = part[1] = 0.0;
    const long long p0 = blk * OR_BLOCK, p1 = p0 + OR_BLOCK < rq->n_pairs ? p0 + OR_BLOCK : rq->n_pairs;
    double* perf = (double*)malloc((size_t)2 * rq->n_obs * sizeof(double));
    if (!perf) return;
    for (long long p = p0; p < p1; ++p) {
        PairState s;
        pair_init(&c->m, &s, (uint64_t)(rq->first_pair + p));
        double low[2] = {1.0, 1.0};
        int j = 0;
        for (int i = 1; i <= rq->n_steps; ++i) {
            pair_step(&c->m, &s, i);
            for (int leg = 0; leg < 2; ++leg) {
                double w = INFINITY;
                for (int a = 0; a < rq->n_names; ++a) {
                    const double q = exp(rq->log_fwd[a * (rq->n_steps + 1) + i] + s.x[leg][a]);
                    w = q < w ? q : w;
                }
                low[leg] = w < low[leg] ? w : low[leg];
                if (j < rq->n_obs && rq->obs_step[j] == i) perf[leg * rq->n_obs + j] = w;
            }
            if (j < rq->n_obs && rq->obs_step[j] == i) ++j;
        }
        const double y = 0.5 * (smooth_leg(rq, c->eps, perf, low[0]) + smooth_leg(rq, c->eps, perf + rq->n_obs, low[1]));
        part[0] += y, part[1] += y * y;
    }
    free(perf);
}

int or_autocall_smooth(const ob_mc_request* rq, double eps, int n_threads, ob_mc_result* res) {
    const int st = check_mc(rq);
    if (st) return st;
    if (rq->product != OB_PRODUCT_AUTOCALL || rq->model != OB_MODEL_PATHS) return fail("a path-engine autocall only");
    SmoothCtx c;
    memset(&c, 0, sizeof c);
    c.rq = rq, c.eps = eps;
    c.m.n_names = rq->n_names, c.m.n_steps = rq->n_steps, c.m.n_x = rq->n_x, c.m.seed = rq->seed;
    c.m.dt = rq->dt, c.m.t0 = rq->t0, c.m.root = rq->root, c.m.cvar = rq->cvar, c.m.hes = rq->heston;
    c.m.lo = rq->row_lo, c.m.inv_dx = rq->row_inv_dx, c.m.table = rq->table, c.m.kind = rq->kind;
    c.m.step_row = rq->step_row, c.m.same = rq->same;
    c.m.mixer = rq->mixer, c.m.low_root = rq->low_root;
    for (int k = 0; k < 8; ++k) c.m.mix[k] = rq->mix[k];
    const long long n_blocks = (rq->n_pairs + OR_BLOCK - 1) / OR_BLOCK;
    double* parts = (double*)calloc((size_t)n_blocks * 2, sizeof(double));
    if (!parts) return fail("out of memory");
    run_blocks(smooth_block, &c, n_blocks, parts, 2 * sizeof(double), n_threads);
    double s = 0.0, s2 = 0.0;
    for (long long b = 0; b < n_blocks; ++b) s += parts[2 * b], s2 += parts[2 * b + 1];
    free(parts);
    memset(res, 0, sizeof *res);
    const double n = (double)rq->n_pairs, mean = s / n;
    res->n_out = 1, res->n_paths = 2 * rq->n_pairs;
    res->price[0] = mean, res->se[0] = sqrt(fmax(s2 / n - mean * mean, 0.0) / (n - 1.0));
    res->sum_y[0] = s, res->sum_y2[0] = s2;
    return OB_OK;
}
