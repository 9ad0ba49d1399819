/* optlab_b200: a Monte Carlo path engine for NVIDIA B200 (sm_100a), reached through a C ABI.
 *
 * Every entry point returns an int status (OB_OK = 0) and never exits, aborts or traps: the engine runs inside the
 * caller's process. On an error, ob_last_error() gives a message for the calling thread. The status splits the
 * reference's exceptions: OB_EINVAL where it throws std::invalid_argument (a bad request), OB_ENODEV and OB_ECUDA
 * where it throws std::runtime_error (no device, a CUDA failure), OB_ETIMEOUT where a bounded device wait gave up,
 * OB_ESINGULAR where the device's pilot fit meets a regression it leaves to the host (ob_script_pilot_fit).
 *
 * Reference interfaces replaced (paths relative to the reference project, RC = packages/native/cuda):
 *   optlab::api::paths     RC/include/optlab_cuda/requests.hpp:105-106, request layout :36-63   -> ob_paths
 *   optlab::api::leverage  RC/include/optlab_cuda/requests.hpp:107-108, request layout :76-93   -> ob_leverage
 *   optlab::api::price     RC/include/optlab_cuda/requests.hpp:103-104, layouts :12-29         -> ob_price
 *   optlab::api::{gpu_count,has_cuda,cpu_threads,device_info}  requests.hpp:97-101            -> ob_gpu_count, ...
 * The request structs below keep the reference's field order and types, so a binding written for the reference's
 * structs binds these unchanged. The fused, adjoint and batched entry points (ob_mc_*, ob_adjoint_*, ob_batch_*) have
 * no counterpart in the reference ABI: they replace the host NumPy evaluation and bump-and-revalue loops that sit on
 * top of optlab::api::paths (packages/structured/src/optlab/structured/engine.py:143-153,260-330 and
 * packages/risk/src/optlab/risk/engine.py:382-425).
 *
 * Precision argument: OB_FP32 evolves the paths in float (sums in double), OB_FP64 in double throughout.
 * Threading: one caller thread at a time per process (an internal mutex serialises calls), as the reference's
 * "not thread-safe on the GPU" (requests.hpp:103).
 */
#ifndef OPTLAB_B200_H
#define OPTLAB_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define OB_OK 0
#define OB_EINVAL 1
#define OB_ENODEV 2
#define OB_ECUDA 3
#define OB_ETIMEOUT 4
#define OB_ENOMEM 5
#define OB_ESINGULAR 6

#define OB_FP32 0
#define OB_FP64 1

#define OB_MAX_NAMES 8
#define OB_MAX_WINDOWS 2
#define OB_MAX_OUT 32

/* ---------------------------------------------------------------------------------------------- requests (mirrors) */

/* Same layout as optlab_request (RC/include/optlab_cuda/requests.hpp:12-23). model: 0 Black-Scholes, 1 Heston (QE);
   product: 0 European, 1 Asian, 2 down-and-out barrier; legs: 0 none, 1 call, 2 put, 3 forward. */
typedef struct {
    int model, product;
    int legs[3];
    double strikes[3];
    double H;
    int n_steps;
    double S0, r, q, T;
    double sigma;
    double v0, kappa, theta, xi, rho;
    long long n_paths;
    unsigned long long seed;
} ob_request;

/* Same layout as optlab_result (requests.hpp:25-29). */
typedef struct {
    double price[4], se[4];
    long long n_paths;
    double kernel_ms, total_ms;
} ob_result;

/* Same layout as optlab_paths_request (requests.hpp:36-63): host pointers, double, row major. out holds
   n_names x n_cols columns of 2 n_pairs rows, column (a, c) at out + (a * n_cols + c) * 2 n_pairs. */
typedef struct {
    int n_names, n_steps, n_obs, n_x, n_rows;
    long long n_pairs, first_pair;
    unsigned long long seed;
    const double* dt;
    const double* t0;
    const int* obs_step;
    const double* root;
    const int* kind;
    const double* cvar;
    const double* heston;
    int same;
    const int* step_row;
    const double* row_lo;
    const double* row_inv_dx;
    const double* table;
    const double* fwd;
    int mixer;
    double mix[8];
    const double* low_root;
    int n_cols, n_keep;
    const int* col_of;
    int n_windows;
    const int* win_lo;
    const int* win_hi;
    double* out;
    double kernel_ms, total_ms;
} ob_paths_request;

/* Same layout as optlab_device (requests.hpp:66-71). */
typedef struct {
    char name[256];
    int major, minor, sm_count, clock_mhz;
    long long total_mem, free_mem;
    int integrated, kernel_timeout;
} ob_device;

/* Same layout as optlab_leverage_request (requests.hpp:76-93). */
typedef struct {
    int n_steps;
    const double* dt;
    const double* t0;
    long long n_pairs;
    unsigned long long seed;
    double v0, kappa, theta, xi, rho;
    int n_x, n_bins, n_fine;
    double atm_vol, bandwidth_scale, l_min, l_max, q_lo, q_hi;
    int local_linear, positive_part;
    int n_lv;
    const double* lv_lo;
    const double* lv_inv_dx;
    const double* lv_rows;
    double* x_grids;
    double* values;
    double total_ms;
} ob_leverage_request;

/* ---------------------------------------------------------------------------------------------- fused pricing */

#define OB_MODEL_PATHS 0     /* the log-Euler step of paths.hpp, per name kind (constant, table, Heston, SLV) */
#define OB_MODEL_HESTON_QE 1 /* Andersen QE-M for one Heston name (schemes.hpp:154-187), uniform steps */

#define OB_PRODUCT_LADDER 0   /* payoffs at maturity, each with an optional barrier monitored at every step end */
#define OB_PRODUCT_AUTOCALL 1 /* Phoenix / worst-of autocall with coupon memory and a knock-in put */

#define OB_BARRIER_NONE 0
#define OB_BARRIER_UP_OUT 1
#define OB_BARRIER_DOWN_OUT 2
#define OB_BARRIER_UP_IN 3
#define OB_BARRIER_DOWN_IN 4

/* A simulation plus a product, priced in one launch: path, payoff and the FP64 sums of the pair averages.
   The model part reads as ob_paths_request; the spot of name a at grid point i is spot[a] * exp(log_fwd[a, i] + x)
   under OB_MODEL_PATHS and spot[0] * exp(y) under OB_MODEL_HESTON_QE (y = ln S / S0, drift (r - q) dt).
   Ladder: output k = leg k's discounted payoff at maturity; then E[S_T] of name 0 (undiscounted).
   Autocall: output 0 = price (notional 1); 1 = probability of an early redemption; 2 = probability of a knock-in;
   3 = the expected number of coupons paid. */
typedef struct {
    int model;
    int n_names, n_steps;
    long long n_pairs, first_pair;
    unsigned long long seed;
    const double* dt;          /* n_steps */
    const double* t0;          /* n_steps */
    const double* root;        /* n_names x n_names */
    const int* kind;           /* n_names: 0 constant, 1 table, 2 Heston (Euler), 3 SLV */
    const double* cvar;        /* n_names */
    const double* heston;      /* n_names x 5: v0, kappa, theta, xi, rho */
    int same;                  /* variance residuals correlated like the spots */
    int n_x, n_rows;
    const int* step_row;       /* n_names x n_steps */
    const double* row_lo;      /* n_rows */
    const double* row_inv_dx;  /* n_rows */
    const double* table;       /* n_rows x n_x */
    const double* spot;        /* n_names */
    const double* log_fwd;     /* n_names x (n_steps + 1): ln(F(t_i) / S0), t_0 = 0 */
    double r, q;               /* OB_MODEL_HESTON_QE: flat rates */
    int product;
    /* ladder */
    int n_legs;                /* <= OB_MAX_OUT - 1 */
    const int* leg_type;       /* 1 call, 2 put, 3 forward */
    const double* leg_strike;
    const int* leg_barrier;    /* OB_BARRIER_* */
    const double* leg_level;   /* barrier level (spot units) */
    double discount;           /* D(T) */
    /* autocall */
    int n_obs;
    const int* obs_step;       /* n_obs, increasing, in 1..n_steps: observation j after step obs_step[j] */
    const double* obs_discount;/* n_obs: discount factor of the payment of observation j */
    const double* trigger;     /* n_obs: autocall level of perf (<= 0: no call on that date; never on the last) */
    double coupon_barrier, coupon, ki_barrier, put_strike;
    int memory;                /* coupons missed are paid at the next coupon */
    int ki_daily;              /* 1: knock-in on the lowest close of every step end; 0: at maturity only */
    /* local correlation (OB_MODEL_PATHS, 2 names or more; paths.hpp:219-237): with mixer 1 every step draws one more
       normal after the names' and mixes a common factor into the names' normals, with a weight that moves with the
       level of the basket at the step's start. mix = (w0, level, down, up, sigma, sign, cos, sin), low_root the root
       of the low correlation aligned to the factor: the reference plan's mix and low_root (localcorr.py:47-83). */
    int mixer;
    double mix[8];
    const double* low_root;    /* n_names x n_names */
} ob_mc_request;

typedef struct {
    int n_out;
    double price[OB_MAX_OUT], se[OB_MAX_OUT];
    long long n_paths;
    double kernel_ms, total_ms;
    /* the FP64 sums the estimate comes from, over the n_paths / 2 pair values y of output k: sum y and sum y^2
       (price = sum_y / n, se = sqrt((sum_y2 / n - price^2) / (n - 1))); what ranks pool to combine shards */
    double sum_y[OB_MAX_OUT], sum_y2[OB_MAX_OUT];
} ob_mc_result;

typedef struct ob_mc_plan ob_mc_plan;

/* ---------------------------------------------------------------------------------------------- adjoint Greeks */

#define OB_ADJ_BATCHES 32 /* batches of pairs of the gradient (standard errors by batch means) */

/* An autocall under the path engine's local vol (every name kind 1, 1 to 4 names, pairs 0 .. n_pairs - 1) with its
   digitals smoothed as ramps of relative width `smoothing` (the reference's risk engine uses 0.005 for Greeks,
   packages/risk/src/optlab/risk/greeks.py:430; 0 gives the exact payoff). checkpoint: the steps between the states
   the forward pass keeps for the backward one: 1 (every step: the backward recomputes nothing), 4 (every fourth:
   the backward recomputes each 4-step segment, a quarter of the memory), 0 (every step while those states take at
   most 24 GiB, else every fourth). */
typedef struct {
    ob_mc_request base;
    double smoothing;
    int checkpoint;
} ob_adjoint_request;

typedef struct {
    double price, price_se;                              /* smoothed price, notional 1 */
    double delta[OB_MAX_NAMES], delta_se[OB_MAX_NAMES];  /* dV/dS_a, local vol moving with the spot (log-moneyness) */
    long long n_paths;
    int n_batches;
    double forward_ms, backward_ms;
} ob_adjoint_result;

typedef struct ob_adjoint_plan ob_adjoint_plan;

/* ---------------------------------------------------------------------------------------------- batched risk */

/* One trade of a revaluation batch. Local-vol trades (model OB_MODEL_PATHS) have 1 to 5 names, each a block of
   n_exp table rows of the batch's pool starting at table_row0 + a n_exp; Heston trades (OB_MODEL_HESTON_QE) one name.
   Ladder legs and autocall schedules are read from the pools at leg0 / obs0; strikes, barrier levels, triggers and
   the knock-in are fractions of the initial spot, applied to the worst performance of the names. */
typedef struct {
    int model, product, n_names, n_steps;
    long long n_pairs;
    unsigned long long seed;
    int table_row0, root0;
    double heston[5];
    double r, q;
    int n_legs, leg0;
    int n_obs, obs0;
    double coupon_barrier, coupon, ki_barrier, put_strike;
    int memory, ki_daily;
    double discount;
    int corr_root0; /* local vol, 2 to 5 names: the first of its n_corr moved roots in the root pool, n_names^2 each */
} ob_batch_trade;

/* The batch: trades, pools and scenarios. Every trade steps by dt; a local-vol table row j of a trade is the
   expiry horizon (j + 1) / n_exp, read by steps starting before it (the first expiry after a step's start). The
   scenarios of each trade: the base, then n_spot relative spot moves (evaluated on the base simulation: the local vol
   is in log-moneyness, so a spot move scales the paths), then n_vol moves of the implied volatilities, each a
   simulation on the same random numbers with the pool's local variance under that move (vol_table: the host moves
   each surface's implied vols as the reference's risk scenarios do, packages/risk/src/optlab/risk/shocks.py:63-108,
   and re-tabulates Dupire on the same points; vol_shift and vol_tilt record each move's parallel shift and skew);
   Heston trades do not move under them, as the reference's Heston model ignores the surface. After those, n_carry (at most 4) moves of the carry on the base
   simulation: carry_rate moves the rate in the forward and the discounting, carry_div the dividend yield (with repo)
   in the forward only, so that a path moves by exp((carry_rate - carry_div) t) at time t and a payment at t
   (the ladder's last step, an autocall's observation step) is discounted by exp(-carry_rate t) more
   (packages/risk/src/optlab/risk/engine.py:8-11). Last, n_corr moves of the correlation, each a simulation of the
   multi-name local-vol trades on the moved root at corr_root0 (single-name and Heston trades do not move). The
   outputs of a trade: base, spot moves, carry moves, vol moves, correlation moves; the base simulation holds at most
   32 of them (1 + n_spot + n_carry). */
typedef struct {
    int n_trades;
    const ob_batch_trade* trades;
    double dt, horizon;
    int n_exp, n_x;
    int n_rows;                /* rows of the pool (table, row_lo, row_inv_dx and each vol scenario's table) */
    const double* table;       /* pool rows x n_x: local variance */
    const double* row_lo;      /* pool rows */
    const double* row_inv_dx;  /* pool rows */
    const double* root;        /* pool of correlation roots */
    const int* leg_type;
    const double* leg_strike;
    const int* leg_barrier;
    const double* leg_level;
    const int* obs_step;
    const double* obs_trigger;
    const double* obs_discount;
    int n_spot;
    const double* spot_shift;
    int n_vol;
    const double* vol_shift;   /* n_vol: the parallel implied-vol move of each scenario (a record) */
    const double* vol_tilt;    /* n_vol: the skew move (90 % - 110 % vol gap at one year) of each scenario (a record) */
    const double* vol_table;   /* n_vol x pool rows x n_x: the pool's local variance under each vol scenario */
    int n_carry;
    const double* carry_rate;
    const double* carry_div;
    int n_corr;
} ob_batch_request;

#define OB_BATCH_MAX_CARRY 4 /* carry moves of a batch */

typedef struct ob_batch ob_batch;

/* ---------------------------------------------------------------------------------------------- payoff scripts */

/* A payoff script of the reference's language (packages/structured/src/optlab/structured/script/), compiled on the
   host into register bytecode (optlab_b200/script.py) and run on every path while it is simulated. `model` is the
   simulation (its product fields are unused); names follow the script's underlyings. Registers 0 .. n_const - 1
   hold `consts` (register 0 is 1.0, the top-level mask), the next ones the variables (0 at the start of a path),
   then temporaries; n_regs <= 128. `code` is n_code instructions of 4 ints (op, d, a, b), event k running
   instructions event_code[k] .. event_code[k + 1] - 1 at step end event_step[k] (0: the valuation date) with the
   discount factor event_discount[k] of its payment date (0: no payment counted). Window w (lowest, highest or
   realised variance, win_func 0, 1, 2) reads name win_name[w] at the step ends fix_step[win_fix0[w] ..
   win_fix0[w + 1] - 1]; a variance corridor is [win_lower[w], win_upper[w]] (NaN: no bound). smoothing: the
   relative width of the comparison ramps (0: hard comparisons). */
typedef struct {
    ob_mc_request model;
    int n_code;
    const int* code;
    int n_const;
    const double* consts;
    int n_regs;
    int n_events;
    const int* event_step;
    const int* event_code;     /* n_events + 1 */
    const double* event_discount;
    int n_windows;             /* <= 8 */
    const int* win_name;
    const int* win_func;
    const int* win_fix0;       /* n_windows + 1 */
    const int* fix_step;
    const double* win_lower;
    const double* win_upper;
    double smoothing;
    /* The issuer's call (`call pay`, instruction "call" with d = call index, a = amount, b = mask): call_mode 0 never
       calls; 1 records a pilot: for every path (pair p's legs at p and n_pairs + p), per event its discounted flows
       before and after its call statement, then per call its mask, the alive mass, the amount and the n_state state
       values, into the host array `record` (2 n_pairs x (2 n_events + n_calls (3 + n_state)) doubles); 2 applies
       fitted rules: the issuer calls where the rule's continuation of the state is above the amount. A rule is
       OB_RULE_STRIDE doubles: valid, n_poly, n_knots, mean[4], scale[4], powers[25][4], knot variable[25],
       knot[25], coefficients[50] (the polynomials', then the hinges'). */
    int n_calls;
    const int* call_state;     /* n_calls x 4: registers of each call's state */
    int n_state;               /* <= 4 */
    int call_mode;
    const double* rules;
    double* record;
    /* Branched continuations (the inner paths of the issuer's dual bound, packages/structured/src/optlab/structured/
       exercise.py:294-380): with branch = 1, one local-vol name and the staged local-vol kernel, pair p continues
       outer path o = p / branch_pairs: up to step end branch_step both its legs follow that path's draws (path o of
       an outer simulation of branch_outer pairs on branch_seed: pair o of it for o < branch_outer, else the
       antithetic leg of pair o - branch_outer), after it the pair draws its own on the model's seed. pair_value
       (host, n_pairs doubles, may be NULL; also without branch) receives each pair's average present value. */
    int branch;
    int branch_step;
    long long branch_outer;
    long long branch_pairs;
    unsigned long long branch_seed;
    double* pair_value;
} ob_script_request;

#define OB_RULE_STRIDE 224

/* price and se of the pair-averaged present value; the paths (legs) on which a payment was not finite, a condition
   undefined where it mattered, or the redemption weights did not add up to one. */
typedef struct {
    double price, se;
    long long n_paths;
    long long bad_pay, bad_cond, bad_redemption;
    double kernel_ms;
} ob_script_result;

/* ---------------------------------------------------------------------------------------------- entry points */

const char* ob_last_error(void);
int ob_version(void);
/* requests.hpp:97: CUDA devices, 0 without device or driver (never an error). */
int ob_gpu_count(void);
/* requests.hpp:98: 1, this library always has its CUDA backend. */
int ob_has_cuda(void);
/* requests.hpp:99: hardware threads of the host. */
int ob_cpu_threads(void);
/* requests.hpp:101: properties of a device; OB_ENODEV without it. */
int ob_device_info(int device, ob_device* out);
/* No counterpart in the reference (it allocates and frees per call). The one-shot calls (ob_price, ob_mc_price,
   ob_paths, ob_script_price, ob_leverage, ob_philox_normals) keep their device buffers for the next call, at most
   512 MB over all devices, and ob_paths keeps 64 MB of pinned host memory through which it copies its columns (the
   result reads 16 KB more); this frees them and forgets the kernels' occupancy answers and shared-memory limits the
   plans cached. Call it before cudaDeviceReset or before destroying a context the library has used: cached buffers
   and attributes belong to the context that made them. */
int ob_release_buffers(void);

/* The engine's random numbers for RNG parity: for pairs first_pair .. first_pair + n_pairs - 1 of key seed, blocks
   first_block .. first_block + n_blocks - 1 of the stream tagged `tag` (0 or 0x80000000, paths.hpp:207-233),
   the Philox4x32-10 outputs (4 u32 per block) and their Box-Muller normals in double and float. Host outputs of
   n_pairs x n_blocks x 4 values, pair-major; any output may be NULL. */
int ob_philox_normals(unsigned long long seed, long long first_pair, long long n_pairs, unsigned tag,
                      unsigned long long first_block, int n_blocks, unsigned* u32, double* z64, float* z32);

/* Drop-in for optlab::api::paths(rq, 1, 0) (requests.hpp:105-106): fills rq->out and the timings. */
int ob_paths(ob_paths_request* rq, int precision);

/* Drop-in for optlab::api::leverage(rq, 1, 0) (requests.hpp:107-108): fills x_grids, values and total_ms.
   The whole calibration runs on the device as one persistent kernel (grid barriers between its phases); the host
   reads the two output tables once. OB_ETIMEOUT: a grid barrier gave up waiting (see ob_set_wait_limit). */
int ob_leverage(ob_leverage_request* rq, int precision);

/* No counterpart in the reference (its calibration synchronises through the host). The polls a persistent kernel's
   grid barrier makes before it gives up and the call returns OB_ETIMEOUT; a barrier completes within microseconds,
   and the default (about a second) is far above that. A negative value restores the default; returns the previous
   limit. Process-wide; read at each call. */
long long ob_set_wait_limit(long long polls);

/* Drop-in for optlab::api::price(rq, 1, 0) (requests.hpp:103-104): the fixed products of the reference's study,
   with the engine's Philox normals (pair p reads stream 0 of pair p) instead of cuRAND. */
int ob_price(const ob_request* rq, ob_result* res, int precision);

/* ob_price without any device allocation, for callers that own all device memory through another allocator or
   must not call cudaMalloc/cudaFree while pricing. No counterpart in the reference: it has no allocation-free path.
   Its scratch (the per-block and final sums) is a fixed array in the library, about 256 KiB on every device that
   loads it, kept until exit; launches needing more than 4096 blocks are refused (OB_EINVAL; a B200 launch takes at
   most 148 x 8). Every call looks up the array's address in the current device's context; the first call on a
   device also loads the library's device code there and should come before any stream capture. Calls share the
   array: calls that overlap on the GPU race and must not be made (within one process the library's lock and the
   blocking read-back of the sums keep its own calls apart). */
int ob_price_noalloc(const ob_request* rq, ob_result* res, int precision);

/* Fused pricing, end to end: host request in, result out (copies and allocations included). */
int ob_mc_price(const ob_mc_request* rq, int precision, ob_mc_result* res);

/* The same in three steps, for callers that keep the inputs resident on the device: create validates the request
   and uploads it; run launches n_pairs pairs from first_pair on `stream` (a cudaStream_t, NULL: the legacy stream)
   without waiting; result waits for the stream and reads the sums of every run since the last result. */
int ob_mc_plan_create(const ob_mc_request* rq, int precision, ob_mc_plan** plan);
int ob_mc_run(ob_mc_plan* plan, long long n_pairs, long long first_pair, unsigned long long seed, void* stream);
int ob_mc_result_get(ob_mc_plan* plan, ob_mc_result* res);
int ob_mc_plan_destroy(ob_mc_plan* plan);

/* Adjoint (pathwise) Greeks: no counterpart in the reference ABI; it replaces the bump-and-revalue loop of
   packages/risk/src/optlab/risk/engine.py:382-425 and greeks.py:199-244 for local-vol autocalls. create uploads the
   request; run makes one forward pass on `stream` (d_table: a device n_rows x n_x double table of local variance
   replacing the current one, NULL keeps it) and, with d_grad non-null, the backward pass, filling d_grad (device,
   OB_ADJ_BATCHES x n_rows x n_x doubles) with each batch's sum over its pairs of d(pair value)/d(table entry);
   result waits, returns price and deltas with standard errors, and the pairs of each batch (batch_pairs may be
   NULL). Without d_grad, run is the smoothed revaluation of a bump-and-revalue. */
int ob_adjoint_plan_create(const ob_adjoint_request* rq, int precision, ob_adjoint_plan** plan);
int ob_adjoint_run(ob_adjoint_plan* plan, const double* d_table, double* d_grad, void* stream);
int ob_adjoint_result_get(ob_adjoint_plan* plan, ob_adjoint_result* res, long long* batch_pairs);
int ob_adjoint_plan_destroy(ob_adjoint_plan* plan);

/* Batched risk revaluation: no counterpart in the reference ABI; it replaces the per-shock simulations of
   packages/risk/src/optlab/risk/engine.py:382-425,563-644 for a book of trades. create checks and uploads the batch;
   tune times candidate tiles (pairs per work item) and block sizes on a sample of each trade class's work and keeps
   the fastest (budget_ms bounds its time; 0: the defaults); capture records one run (every class's persistent kernel
   on its own stream, then the reduction) as a CUDA graph; launch replays it on `stream` (or runs the kernels directly
   without a capture); run_per_trade runs the same work as one launch per trade simulation, the comparison; result
   waits and writes price and se (n_trades x (1 + n_spot + n_carry + n_vol + n_corr), row-major) and the last run's
   device time. */
int ob_batch_create(const ob_batch_request* rq, int precision, ob_batch** batch);
int ob_batch_tune(ob_batch* batch, int budget_ms);
int ob_batch_capture(ob_batch* batch, void* stream);
int ob_batch_launch(ob_batch* batch, void* stream);
int ob_batch_run_per_trade(ob_batch* batch, void* stream);
int ob_batch_result(ob_batch* batch, double* price, double* se, double* device_ms);
/* The trade classes (one persistent kernel each) and their current shapes: *n_classes, and for the first
   max_classes of them 8 ints each in info: model, names, product, trades, tile (pairs per work item), block, and
   after ob_batch_tune the time in microseconds of the tuner's sample of the class at its shape before tuning and at
   the kept one (0 before tuning). */
int ob_batch_classes(const ob_batch* batch, int max_classes, int* n_classes, int* info);
int ob_batch_destroy(ob_batch* batch);

/* Payoff scripts: no counterpart in the reference ABI; it replaces the evaluation of a script on paths brought to
   the host (packages/structured/src/optlab/structured/engine.py:143-153 with script/evaluator.py:123-231): the
   paths are simulated and the script evaluated on the device, and only the price and its SE come back. */
int ob_script_price(const ob_script_request* rq, int precision, ob_script_result* res);

/* The issuer's Longstaff-Schwartz policy fitted on the device: replaces the reference's pilot and fit
   (packages/structured/src/optlab/structured/exercise.py:212-252 with the basis of :125-140, run from
   structured/engine.py:342-370). Runs the pilot `rq` (call_mode 1; rq->record may be NULL, and the record then stays
   on the device) and fits the rules backward over its calls on the device: call_event[c] is the event of call c,
   pay_discount[k] the discount factor of event k's payment (0: none counted). rules receives n_calls rows of
   OB_RULE_STRIDE doubles in the layout call_mode 2 reads (a call no path reaches: a row of zeros), in_sample the
   pilot's value under its own policy, res the pilot's own result (never called). OB_ESINGULAR: a regression's terms
   were nearly collinear (a pivot of its normal equations below 1e-13 of its diagonal), where the reference's SVD solve
   and the device's refined normal equations may part; the caller fits that pilot on the host. */
int ob_script_pilot_fit(const ob_script_request* rq, int precision, const int* call_event, const double* pay_discount,
                        double* rules, double* in_sample, ob_script_result* res);

#ifdef __cplusplus
}
#endif

#endif /* OPTLAB_B200_H */
