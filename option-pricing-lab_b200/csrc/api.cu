// Status, device queries and the random-number surface of the C ABI (include/optlab_b200.h).
// Reference counterparts: optlab::api::{gpu_count, has_cuda, cpu_threads, device_info}
// (RC/include/optlab_cuda/requests.hpp:97-101, RC/src/requests.cpp:225-325).
#include <algorithm>
#include <cstdarg>
#include <map>
#include <thread>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "host_copy.cuh"

namespace ob {

namespace {
thread_local char g_err[1024] = "";
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

std::mutex& api_mutex() {
    static std::mutex m;
    return m;
}

int require_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        throw Error(OB_ENODEV, "no CUDA device");
    }
    int dev = 0, sms = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    return sms;
}

namespace {
struct OccKey {
    const void* kernel;
    int device, block;
    size_t smem;
    bool operator<(const OccKey& o) const {
        return std::tie(kernel, device, block, smem) < std::tie(o.kernel, o.device, o.block, o.smem);
    }
};
// What the launch caches hold: occupancy answers, and the shared-memory limit set on each kernel of each device.
struct LaunchCaches {
    std::mutex m;
    std::map<OccKey, int> occ;
    std::map<std::pair<const void*, int>, size_t> smem_set;
    static LaunchCaches& get() {
        static LaunchCaches* c = new LaunchCaches();
        return *c;
    }
};
}  // namespace

int occupancy(const void* kernel, int block, size_t smem) {
    LaunchCaches& c = LaunchCaches::get();
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    const OccKey key{kernel, dev, block, smem};
    {
        std::lock_guard<std::mutex> lock(c.m);
        const auto it = c.occ.find(key);
        if (it != c.occ.end()) return it->second;
    }
    int per_sm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem), "occupancy");
    std::lock_guard<std::mutex> lock(c.m);
    c.occ[key] = per_sm;
    return per_sm;
}

void allow_smem(const void* kernel, size_t smem) {
    LaunchCaches& c = LaunchCaches::get();
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(c.m);
    size_t& have = c.smem_set[{kernel, dev}];
    if (have >= smem && have > 0) return;
    check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
               "cudaFuncSetAttribute");
    have = smem;
}

void clear_launch_caches() {
    LaunchCaches& c = LaunchCaches::get();
    std::lock_guard<std::mutex> lock(c.m);
    c.occ.clear(), c.smem_set.clear();
}

namespace {
std::mutex g_pin_m;
void* g_pin = nullptr;
bool g_pin_tried = false;
}  // namespace

void* small_pinned() {
    std::lock_guard<std::mutex> lock(g_pin_m);
    if (!g_pin_tried) {
        g_pin_tried = true;
        if (cudaHostAlloc(&g_pin, kSmallPinnedBytes, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            g_pin = nullptr;
        }
    }
    return g_pin;
}

void release_small_pinned() {
    std::lock_guard<std::mutex> lock(g_pin_m);
    if (g_pin) cudaFreeHost(g_pin);
    cudaGetLastError();
    g_pin = nullptr, g_pin_tried = false;
}

namespace {

// One thread per (pair, block): the Philox outputs and both normal precisions, pair-major.
__global__ void philox_kernel(uint32_t k0, uint32_t k1, long long first_pair, long long n_pairs, uint32_t tag,
                              unsigned long long first_block, int n_blocks, unsigned* u32, double* z64, float* z32) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n_pairs * n_blocks) return;
    const long long p = t / n_blocks;
    const int b = static_cast<int>(t % n_blocks);
    const uint64_t pair = static_cast<uint64_t>(first_pair + p), blk = first_block + static_cast<uint64_t>(b);
    uint32_t x = static_cast<uint32_t>(pair), y = static_cast<uint32_t>(pair >> 32);
    uint32_t z = static_cast<uint32_t>(blk), w = static_cast<uint32_t>(blk >> 32) | tag;
    philox4x32_10(x, y, z, w, k0, k1);
    const long long o = t * 4;
    u32[o] = x, u32[o + 1] = y, u32[o + 2] = z, u32[o + 3] = w;
    box_muller(x, y, z64[o], z64[o + 1]);
    box_muller(z, w, z64[o + 2], z64[o + 3]);
    box_muller(x, y, z32[o], z32[o + 1]);
    box_muller(z, w, z32[o + 2], z32[o + 3]);
}

}  // namespace
}  // namespace ob

extern "C" {

const char* ob_last_error(void) { return ob::g_err; }

int ob_version(void) { return 10000; }

int ob_gpu_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int ob_has_cuda(void) { return 1; }

int ob_release_buffers(void) {
    return ob::guarded([&] {
        ob::BufferCache::get().drain();
        ob::PinnedStage::get().release();
        ob::clear_launch_caches();
        ob::release_small_pinned();
    });
}

int ob_cpu_threads(void) {
    const unsigned n = std::thread::hardware_concurrency();
    return n ? static_cast<int>(n) : 1;
}

int ob_device_info(int device, ob_device* out) {
    return ob::guarded([&] {
        if (!out) ob::invalid("null output");
        std::memset(out, 0, sizeof *out);
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
            cudaGetLastError();
            throw ob::Error(OB_ENODEV, "no such CUDA device");
        }
        cudaDeviceProp p{};
        ob::check_cuda(cudaGetDeviceProperties(&p, device), "cudaGetDeviceProperties");
        std::snprintf(out->name, sizeof out->name, "%s", p.name);
        out->major = p.major, out->minor = p.minor, out->sm_count = p.multiProcessorCount;
        int khz = 0;
        cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device);
        out->clock_mhz = khz / 1000;
        out->total_mem = static_cast<long long>(p.totalGlobalMem);
        out->integrated = p.integrated;
        int timeout = 0;
        cudaDeviceGetAttribute(&timeout, cudaDevAttrKernelExecTimeout, device);
        out->kernel_timeout = timeout;
        int prev = 0;
        cudaGetDevice(&prev);
        size_t fr = 0, tot = 0;
        if (cudaSetDevice(device) == cudaSuccess && cudaMemGetInfo(&fr, &tot) == cudaSuccess)
            out->free_mem = static_cast<long long>(fr);
        cudaSetDevice(prev);
        cudaGetLastError();
    });
}

int ob_philox_normals(unsigned long long seed, long long first_pair, long long n_pairs, unsigned tag,
                      unsigned long long first_block, int n_blocks, unsigned* u32, double* z64, float* z32) {
    return ob::guarded([&] {
        if (n_pairs < 0 || n_blocks < 0 || first_pair < 0) ob::invalid("negative size");
        if (tag != 0u && tag != 0x80000000u) ob::invalid("tag must be 0 or 0x80000000");
        const long long n = n_pairs * n_blocks;
        if (n == 0) return;
        if (n > (1LL << 28)) ob::invalid("at most 2^28 blocks per call");
        ob::require_device();
        ob::DeviceArena arena;
        arena.recycle = true;  // the blocking copies below end the call's device work
        unsigned* du = arena.alloc<unsigned>(4 * n);
        double* dz = arena.alloc<double>(4 * n);
        float* df = arena.alloc<float>(4 * n);
        const int block = 256;
        ob::philox_kernel<<<static_cast<unsigned>((n + block - 1) / block), block>>>(
            static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), first_pair, n_pairs, tag, first_block,
            n_blocks, du, dz, df);
        ob::check_cuda(cudaGetLastError(), "philox_kernel launch");
        if (u32) ob::check_cuda(cudaMemcpy(u32, du, 4 * n * sizeof(unsigned), cudaMemcpyDeviceToHost), "copy u32");
        if (z64) ob::check_cuda(cudaMemcpy(z64, dz, 4 * n * sizeof(double), cudaMemcpyDeviceToHost), "copy z64");
        if (z32) ob::check_cuda(cudaMemcpy(z32, df, 4 * n * sizeof(float), cudaMemcpyDeviceToHost), "copy z32");
        ob::check_cuda(cudaDeviceSynchronize(), "philox_kernel");
    });
}

}  // extern "C"
