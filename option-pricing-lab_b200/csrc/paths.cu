// ob_paths: the drop-in for optlab::api::paths(rq, 1, 0) (RC/include/optlab_cuda/requests.hpp:105-106,
// RC/src/paths_gpu.cu:76-167). One thread per antithetic pair, state in registers, the spot columns and window
// extremes written in the reference's layout (out[(a n_cols + c) 2 n_pairs + row], pair p at row p, its antithetic
// at n_pairs + p), in float or double. The request is checked as RC/src/requests.cpp:168-207 does.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "model.cuh"

namespace ob {

namespace {

template <typename R>
struct PathsDev {
    ModelDev<R> m;
    int n_obs, n_cols, n_keep, n_win;
    long long n_pairs, first_pair, rows;
    const int* obs_step;
    const int* col_of;
    const int* win_lo;
    const int* win_hi;
    const R* fwd;  // n x n_obs
    double* out;
};

template <typename R, int N>
__device__ __forceinline__ void record(const PathsDev<R>& s, long long p, int j, const PairDev<R, N>& st,
                                       R (&lo)[2][N][2], R (&hi)[2][N][2]) {
    const long long r0 = p, r1 = s.n_pairs + p;
    const int c = s.col_of[j];
#pragma unroll
    for (int a = 0; a < N; ++a) {
        if (a >= s.m.n_names) continue;
        const R f = s.fwd[a * s.n_obs + j];
        const R S0 = f * m_exp(st.x[0][a]), S1 = f * m_exp(st.x[1][a]);
        double* base = s.out + static_cast<long long>(a) * s.n_cols * s.rows;
        if (c >= 0) {
            base[c * s.rows + r0] = static_cast<double>(S0);
            base[c * s.rows + r1] = static_cast<double>(S1);
        }
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            if (w >= s.n_win || j < s.win_lo[w] || j > s.win_hi[w]) continue;
            if (j == s.win_lo[w]) {
                lo[0][a][w] = hi[0][a][w] = S0;
                lo[1][a][w] = hi[1][a][w] = S1;
            } else {
                lo[0][a][w] = m_min(lo[0][a][w], S0), hi[0][a][w] = m_max(hi[0][a][w], S0);
                lo[1][a][w] = m_min(lo[1][a][w], S1), hi[1][a][w] = m_max(hi[1][a][w], S1);
            }
            if (j == s.win_hi[w]) {
                const long long cl = s.n_keep + 2 * w, ch = cl + 1;
                base[cl * s.rows + r0] = static_cast<double>(lo[0][a][w]);
                base[ch * s.rows + r0] = static_cast<double>(hi[0][a][w]);
                base[cl * s.rows + r1] = static_cast<double>(lo[1][a][w]);
                base[ch * s.rows + r1] = static_cast<double>(hi[1][a][w]);
            }
        }
    }
}

template <typename R, int N>
__global__ void __launch_bounds__(256) paths_kernel(PathsDev<R> s) {
    const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= s.n_pairs) return;
    PairDev<R, N> st;
    pair_init<R, N>(s.m, st, static_cast<uint64_t>(s.first_pair + p));
    R lo[2][N][2], hi[2][N][2];
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
        for (int w = 0; w < 2; ++w) lo[0][a][w] = lo[1][a][w] = hi[0][a][w] = hi[1][a][w] = R(0);
    int j = 0;
    while (j < s.n_obs && s.obs_step[j] == 0) record<R, N>(s, p, j++, st, lo, hi);
    for (int i = 1; i <= s.m.n_steps; ++i) {
        pair_step<R, N>(s.m, st, i);
        while (j < s.n_obs && s.obs_step[j] == i) record<R, N>(s, p, j++, st, lo, hi);
    }
}

void check_request(const ob_paths_request& c) {
    if (c.n_names < 1 || c.n_names > OB_MAX_NAMES) invalid("n_names must be 1 to 8");
    if (c.n_pairs < 1 || c.first_pair < 0) invalid("n_pairs must be >= 1 and first_pair >= 0");
    if (c.n_steps < 0 || c.n_obs < 0) invalid("n_steps and n_obs must be >= 0");
    if (!c.out && c.n_obs > 0) invalid("null output");
    if (c.n_steps > 0 && (!c.dt || !c.t0)) invalid("null time grid");
    if (!c.root || !c.kind || !c.cvar || !c.heston || !c.fwd || (c.n_obs && !c.obs_step)) invalid("null array");
    bool table = false;
    for (int a = 0; a < c.n_names; ++a) {
        const int k = c.kind[a];
        if (k < 0 || k > 3) invalid("kind must be 0 to 3");
        table |= k == 1 || k == 3;
        if ((k == 2 || k == 3) && !(c.heston[a * 5 + 1] > 0 && c.heston[a * 5 + 2] > 0 && c.heston[a * 5 + 3] >= 0 &&
                                    std::fabs(c.heston[a * 5 + 4]) <= 1))
            invalid("Heston parameters out of range");
    }
    if (table) {
        if (c.n_x < 2 || c.n_rows < 1 || !c.step_row || !c.row_lo || !c.row_inv_dx || !c.table)
            invalid("a tabulated variance needs n_x >= 2, rows and step_row");
        for (long long i = 0; i < static_cast<long long>(c.n_names) * c.n_steps; ++i) {
            const int k = c.kind[i / (c.n_steps ? c.n_steps : 1)];
            if ((k == 1 || k == 3) && (c.step_row[i] < 0 || c.step_row[i] >= c.n_rows)) invalid("step_row out of range");
        }
    }
    int prev = 0;
    for (int j = 0; j < c.n_obs; ++j) {
        if (c.obs_step[j] < prev || c.obs_step[j] > c.n_steps) invalid("obs_step must be nondecreasing in [0, n_steps]");
        prev = c.obs_step[j];
    }
    if (c.mixer && (c.mixer != 1 || !c.low_root || !(c.mix[4] > 0))) invalid("bad local correlation");
    if (c.n_windows < 0 || c.n_windows > OB_MAX_WINDOWS || (c.n_windows && (!c.win_lo || !c.win_hi)))
        invalid("n_windows must be 0 to 2, with win_lo and win_hi");
    if (c.n_obs && !c.col_of) invalid("null col_of");
    if (c.n_keep < 0 || c.n_cols != c.n_keep + 2 * c.n_windows) invalid("n_cols must be n_keep + 2 n_windows");
    for (int j = 0; j < c.n_obs; ++j)
        if (c.col_of[j] < -1 || c.col_of[j] >= c.n_keep) invalid("col_of out of range");
    for (int w = 0; w < c.n_windows; ++w)
        if (c.win_lo[w] < 0 || c.win_hi[w] < c.win_lo[w] || c.win_hi[w] >= c.n_obs) invalid("bad window");
}

template <typename R>
void run_paths(ob_paths_request& h) {
    const auto t_start = std::chrono::steady_clock::now();
    require_device();
    const int n = h.n_names;
    bool table = false, has_var = false, has_slv = false;
    for (int a = 0; a < n; ++a) {
        table |= h.kind[a] == 1 || h.kind[a] == 3;
        has_var |= h.kind[a] == 2 || h.kind[a] == 3;
        has_slv |= h.kind[a] == 3;
    }
    DeviceArena arena;
    PathsDev<R> s{};
    ModelDev<R>& m = s.m;
    m.n_names = n, m.n_steps = h.n_steps, m.n_x = h.n_x, m.same = h.same, m.mixer = h.mixer;
    m.has_var = has_var, m.has_slv = has_slv;
    m.k0 = static_cast<uint32_t>(h.seed), m.k1 = static_cast<uint32_t>(h.seed >> 32);
    m.dt = arena.put<R>(h.dt, h.n_steps);
    m.t0 = arena.put<R>(h.t0, h.n_steps);
    m.root = arena.put<R>(h.root, static_cast<size_t>(n) * n);
    m.kind = arena.put<int>(h.kind, n);
    m.cvar = arena.put<R>(h.cvar, n);
    m.hes = arena.put<R>(h.heston, 5 * static_cast<size_t>(n));
    if (table) {
        m.step_row = arena.put<int>(h.step_row, static_cast<size_t>(n) * h.n_steps);
        m.lo = arena.put<R>(h.row_lo, h.n_rows);
        m.inv_dx = arena.put<R>(h.row_inv_dx, h.n_rows);
        m.table = arena.put<R>(h.table, static_cast<size_t>(h.n_rows) * h.n_x);
    }
    if (h.mixer) m.low_root = arena.put<R>(h.low_root, static_cast<size_t>(n) * n);
    for (int k = 0; k < 8; ++k) m.mix[k] = static_cast<R>(h.mix[k]);
    s.n_obs = h.n_obs, s.n_cols = h.n_cols, s.n_keep = h.n_keep, s.n_win = h.n_windows;
    s.obs_step = arena.put<int>(h.obs_step, h.n_obs);
    s.col_of = arena.put<int>(h.col_of, h.n_obs);
    s.win_lo = arena.put<int>(h.win_lo, h.n_windows);
    s.win_hi = arena.put<int>(h.win_hi, h.n_windows);
    s.fwd = arena.put<R>(h.fwd, static_cast<size_t>(n) * h.n_obs);

    // Chunks of pairs: the output of one chunk within a quarter of the free memory (at most 4 GB).
    const long long cols = static_cast<long long>(n) * h.n_cols;
    size_t free_mem = 0, total_mem = 0;
    check_cuda(cudaMemGetInfo(&free_mem, &total_mem), "cudaMemGetInfo");
    const long long budget = std::min<long long>(static_cast<long long>(free_mem) / 4, 4LL << 30);
    long long chunk = h.n_pairs;
    if (cols > 0) chunk = std::min(chunk, std::max<long long>(1024, budget / (cols * 2 * 8)));
    double* dout = arena.alloc<double>(std::max<long long>(1, cols * 2 * chunk));
    cudaEvent_t ev0, ev1;
    check_cuda(cudaEventCreate(&ev0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev1), "cudaEventCreate");
    const size_t host_bytes = static_cast<size_t>(cols) * 2 * h.n_pairs * sizeof(double);
    const bool pinned = host_bytes >= (8u << 20) &&
                        cudaHostRegister(h.out, host_bytes, cudaHostRegisterDefault) == cudaSuccess;
    if (!pinned) cudaGetLastError();
    float kernel_ms = 0.0f;
    try {
        for (long long c0 = 0; c0 < h.n_pairs; c0 += chunk) {
            const long long mcount = std::min(chunk, h.n_pairs - c0);
            PathsDev<R> part = s;
            part.n_pairs = mcount, part.first_pair = h.first_pair + c0, part.rows = 2 * mcount, part.out = dout;
            const int block = 256;
            const unsigned grid = static_cast<unsigned>((mcount + block - 1) / block);
            check_cuda(cudaEventRecord(ev0), "cudaEventRecord");
            if (n <= 1) paths_kernel<R, 1><<<grid, block>>>(part);
            else if (n <= 2) paths_kernel<R, 2><<<grid, block>>>(part);
            else if (n <= 4) paths_kernel<R, 4><<<grid, block>>>(part);
            else paths_kernel<R, 8><<<grid, block>>>(part);
            check_cuda(cudaGetLastError(), "paths_kernel launch");
            check_cuda(cudaEventRecord(ev1), "cudaEventRecord");
            if (cols > 0) {
                const size_t width = static_cast<size_t>(mcount) * sizeof(double);
                const size_t spitch = static_cast<size_t>(2 * mcount) * sizeof(double);
                const size_t dpitch = static_cast<size_t>(2 * h.n_pairs) * sizeof(double);
                check_cuda(cudaMemcpy2D(h.out + c0, dpitch, dout, spitch, width, cols, cudaMemcpyDeviceToHost),
                           "cudaMemcpy2D (leg 0)");
                check_cuda(cudaMemcpy2D(h.out + h.n_pairs + c0, dpitch, dout + mcount, spitch, width, cols,
                                        cudaMemcpyDeviceToHost),
                           "cudaMemcpy2D (leg 1)");
            }
            check_cuda(cudaEventSynchronize(ev1), "paths_kernel");
            float ms = 0.0f;
            check_cuda(cudaEventElapsedTime(&ms, ev0, ev1), "cudaEventElapsedTime");
            kernel_ms += ms;
        }
    } catch (...) {
        if (pinned) cudaHostUnregister(h.out);
        cudaEventDestroy(ev0), cudaEventDestroy(ev1);
        throw;
    }
    if (pinned) cudaHostUnregister(h.out);
    cudaEventDestroy(ev0), cudaEventDestroy(ev1);
    h.kernel_ms = kernel_ms;
    h.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
}

}  // namespace
}  // namespace ob

extern "C" int ob_paths(ob_paths_request* rq, int precision) {
    return ob::guarded([&] {
        if (!rq) ob::invalid("null request");
        if (precision != OB_FP32 && precision != OB_FP64) ob::invalid("precision must be OB_FP32 or OB_FP64");
        ob::check_request(*rq);
        if (precision == OB_FP32) ob::run_paths<float>(*rq);
        else ob::run_paths<double>(*rq);
    });
}
