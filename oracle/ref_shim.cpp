// ORACLE — test infrastructure only. An extern "C" face over the reference's own CPU engine, compiled from the
// reference's sources where they lie (oracle/Makefile, output oracle/_ref/libref_optlab.so). It lets the tests and the
// CPU baseline call the reference directly, as its nanobind module would (RC/bindings/ext.cpp:57-179), and it
// composes the reference's Andersen QE-M step with the reference's Philox normal stream, which the reference itself
// never does (its QE reads cuRAND on the GPU and std::normal_distribution on the CPU).
//
// Reference pieces used (RC = packages/native/cuda):
//   optlab::api::paths / leverage / price    RC/include/optlab_cuda/requests.hpp:103-108
//   optlab::NormalStream<double>             RC/include/optlab_cuda/paths.hpp:213-233
//   optlab::make_consts<double>, qe_step     RC/include/optlab_cuda/schemes.hpp:107-186
//   optlab::philox4x32_10, box_muller        RC/include/optlab_cuda/philox.hpp:33-73
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "optlab_cuda/params.hpp"
#include "optlab_cuda/paths.hpp"
#include "optlab_cuda/philox.hpp"
#include "optlab_cuda/requests.hpp"
#include "optlab_cuda/schemes.hpp"

namespace {

thread_local char g_err[512];

int caught(const std::exception& e) {
    std::snprintf(g_err, sizeof g_err, "%s", e.what());
    return 1;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err; }

int ref_paths(optlab_paths_request* rq, int n_threads) {
    try {
        optlab::api::paths(*rq, 0, n_threads);
        return 0;
    } catch (const std::exception& e) {
        return caught(e);
    }
}

int ref_leverage(optlab_leverage_request* rq, int n_threads) {
    try {
        optlab::api::leverage(*rq, 0, n_threads);
        return 0;
    } catch (const std::exception& e) {
        return caught(e);
    }
}

int ref_price(const optlab_request* rq, int n_threads, optlab_result* out) {
    try {
        *out = optlab::api::price(*rq, 0, n_threads);
        return 0;
    } catch (const std::exception& e) {
        return caught(e);
    }
}

// Philox blocks and normals of the reference (double, the CPU branch of box_muller).
int ref_philox_normals(unsigned long long seed, long long first_pair, long long n_pairs, unsigned tag,
                       unsigned long long first_block, int n_blocks, unsigned* u32, double* z64) {
    for (long long p = 0; p < n_pairs; ++p)
        for (int b = 0; b < n_blocks; ++b) {
            const std::uint64_t pair = static_cast<std::uint64_t>(first_pair + p), blk = first_block + b;
            const optlab::U4 r = optlab::philox4x32_10(
                {static_cast<std::uint32_t>(pair), static_cast<std::uint32_t>(pair >> 32),
                 static_cast<std::uint32_t>(blk), static_cast<std::uint32_t>(blk >> 32) | tag},
                static_cast<std::uint32_t>(seed), static_cast<std::uint32_t>(seed >> 32));
            const long long o = (p * n_blocks + b) * 4;
            if (u32) u32[o] = r.x, u32[o + 1] = r.y, u32[o + 2] = r.z, u32[o + 3] = r.w;
            if (z64) {
                optlab::box_muller<double>(r.x, r.y, z64[o], z64[o + 1]);
                optlab::box_muller<double>(r.z, r.w, z64[o + 2], z64[o + 3]);
            }
        }
    return 0;
}

// Heston QE-M (the reference's make_consts<double> and qe_step<double>) on the reference's NormalStream<double>,
// stream 0 of each pair: per step zv then zx, both negated on the antithetic leg (schemes.hpp:212-227). Payoffs of
// one pair: n_legs calls or puts at maturity, each optionally knocked out by an up barrier monitored at every step
// end (hit = max S >= H, packages/core/src/optlab/core/products.py:98-100), plus E[S_T]. Sums of the pair averages
// are added in pair order on each thread's contiguous slice, then in slice order.
int ref_qe_ladder(double S0, double r, double q, double T, int n_steps, const double* heston, long long n_pairs,
                  long long first_pair, unsigned long long seed, int n_legs, const int* leg_type,
                  const double* leg_strike, const int* leg_up_out, const double* leg_level, int n_threads,
                  double* price, double* se) {
    try {
        optlab::McRequest rq;
        rq.model = optlab::Model::Heston;
        rq.market = {S0, r, q, T};
        rq.heston = {heston[0], heston[1], heston[2], heston[3], heston[4]};
        rq.product.n_steps = n_steps;
        const optlab::PathConsts<double> c = optlab::make_consts<double>(rq);
        const double D = std::exp(-r * T);
        const int n_out = n_legs + 1;
        if (n_threads <= 0) n_threads = static_cast<int>(std::thread::hardware_concurrency());
        if (n_threads < 1) n_threads = 1;
        std::vector<std::vector<double>> parts(n_threads, std::vector<double>(2 * n_out, 0.0));
        auto work = [&](int t) {
            const long long a = n_pairs * t / n_threads, b = n_pairs * (t + 1) / n_threads;
            std::vector<double>& acc = parts[t];
            for (long long p = a; p < b; ++p) {
                optlab::NormalStream<double> rng{static_cast<std::uint64_t>(first_pair + p),
                                                 static_cast<std::uint32_t>(seed),
                                                 static_cast<std::uint32_t>(seed >> 32)};
                double y[2] = {0.0, 0.0}, v[2] = {c.v0, c.v0}, hi[2] = {-INFINITY, -INFINITY};
                for (int i = 0; i < n_steps; ++i) {
                    const double zv = rng.next(), zx = rng.next();
                    for (int leg = 0; leg < 2; ++leg) {
                        const double sg = leg ? -1.0 : 1.0;
                        optlab::qe_step<double>(c, y[leg], v[leg], sg * zv, sg * zx);
                        const double S = S0 * std::exp(y[leg]);
                        hi[leg] = S > hi[leg] ? S : hi[leg];
                    }
                }
                for (int k = 0; k < n_out; ++k) {
                    double o = 0.0;
                    for (int leg = 0; leg < 2; ++leg) {
                        const double S = S0 * std::exp(y[leg]);
                        if (k == n_legs) {
                            o += S;
                        } else {
                            const double pay = D * optlab::leg_payoff<double>(leg_type[k], S, leg_strike[k]);
                            o += leg_up_out[k] && hi[leg] >= leg_level[k] ? 0.0 : pay;
                        }
                    }
                    const double yk = 0.5 * o;
                    acc[k] += yk, acc[n_out + k] += yk * yk;
                }
            }
        };
        std::vector<std::thread> pool;
        for (int t = 0; t < n_threads; ++t) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
        for (int k = 0; k < n_out; ++k) {
            double s = 0.0, s2 = 0.0;
            for (const auto& pt : parts) s += pt[k], s2 += pt[n_out + k];
            const optlab::Estimate e = optlab::estimate_from_sums(s, s2, n_pairs);
            price[k] = e.price, se[k] = e.se;
        }
        return 0;
    } catch (const std::exception& e) {
        return caught(e);
    }
}

int ref_cpu_threads() { return optlab::api::cpu_threads(); }

}  // extern "C"
