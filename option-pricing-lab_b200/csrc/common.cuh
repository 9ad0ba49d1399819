// Shared device code of the engine: status handling, the counter-based normals, and small math helpers.
//
// Normals follow the reference's definition (RC = packages/native/cuda of Luca-CS/option-pricing-lab):
//   Philox4x32-10 on counter {pair_lo, pair_hi, block_lo, block_hi | tag}, key {seed_lo, seed_hi}
//     (RC/include/optlab_cuda/philox.hpp:22-44, RC/include/optlab_cuda/paths.hpp:207-233);
//   u = (i + 1/2) 2^-32 (philox.hpp:45-49); Box-Muller r = sqrt(-2 ln u), (cos, sin)(2 pi v) by sincospi
//     (philox.hpp:51-66).
// The integer stream is bit-exact with the reference; in double the normals differ from its CPU's only by libm
// rounding, in float by the hardware sine and cosine of the angle (below) as well.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <functional>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/optlab_b200.h"

namespace ob {

// ------------------------------------------------------------------------------------------------ status

void set_error(const char* fmt, ...);

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(OB_ECUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
inline void invalid(const char* msg) { throw Error(OB_EINVAL, msg); }

// Runs f, turning exceptions into a status and the thread's last error. Serialised by one process-wide mutex.
std::mutex& api_mutex();
template <typename F>
int guarded(F&& f) {
    std::lock_guard<std::mutex> lock(api_mutex());
    try {
        f();
        return OB_OK;
    } catch (const Error& e) {
        set_error("%s", e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_error("out of host memory");
        return OB_ENOMEM;
    } catch (const std::exception& e) {
        set_error("%s", e.what());
        return OB_ECUDA;
    }
}

// Device 0 must exist; returns its SM count.
int require_device();

// Resident blocks an SM of kernel at block threads and smem bytes of dynamic shared memory on the current device (0:
// it cannot launch so). Cached for the process: a query costs microseconds and a one-shot call builds a plan that
// asks for each candidate block size.
int occupancy(const void* kernel, int block, size_t smem);
// Raises kernel's dynamic shared-memory limit on the current device to at least smem bytes (once per kernel and
// size: the attribute is a maximum, so a larger setting serves smaller launches).
void allow_smem(const void* kernel, size_t smem);
// Forgets both (ob_release_buffers: after a device reset the kernels' attributes are gone).
void clear_launch_caches();

// A small pinned host buffer (kSmallPinnedBytes) for the read-back of results, allocated at its first use and kept;
// null where pinned memory cannot be had. The library's calls are serialised, so one buffer serves them all.
constexpr size_t kSmallPinnedBytes = 16384;
void* small_pinned();
void release_small_pinned();  // (ob_release_buffers)

// ------------------------------------------------------------------------------------------------ device memory

// A non-blocking stream owned by one call, destroyed with it.
struct Stream {
    cudaStream_t s = nullptr;
    Stream() { check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate"); }
    ~Stream() {
        if (s) cudaStreamDestroy(s);
    }
    Stream(const Stream&) = delete;
    Stream& operator=(const Stream&) = delete;
    cudaStream_t get() const { return s; }
};

// Device buffers that finished calls handed back, for the next call of the process: a one-shot call's cudaMalloc and
// cudaFree (a few hundred microseconds together, and cudaFree waits for the whole device) become a lookup. At most
// kBytes are held over all devices; a buffer is reused for a request of at least half its size. The cache is never
// destroyed: its buffers go with the process.
class BufferCache {
  public:
    static constexpr size_t kBytes = size_t(512) << 20;
    static BufferCache& get() {
        static BufferCache* c = new BufferCache();
        return *c;
    }
    // The smallest held buffer of device dev with bytes <= size <= 2 bytes (its size in got), or null.
    void* take(int dev, size_t bytes, size_t& got) {
        std::lock_guard<std::mutex> lock(m_);
        int best = -1;
        for (int i = 0; i < n_; ++i)
            if (e_[i].dev == dev && e_[i].bytes >= bytes && e_[i].bytes <= 2 * bytes &&
                (best < 0 || e_[i].bytes < e_[best].bytes))
                best = i;
        if (best < 0) return nullptr;
        void* p = e_[best].p;
        got = e_[best].bytes;
        held_ -= got;
        e_[best] = e_[--n_];
        return p;
    }
    // Frees every held buffer (each on its own device) and returns how many there were. Buffers belong to the
    // context that allocated them: a caller that resets a device (cudaDeviceReset) or destroys its context must
    // empty the cache first, or the next call could be handed memory of a context that is gone.
    int drain() {
        std::lock_guard<std::mutex> lock(m_);
        int prev = 0;
        cudaGetDevice(&prev);
        const int n = n_;
        for (int i = 0; i < n_; ++i) {
            cudaSetDevice(e_[i].dev);
            cudaFree(e_[i].p);
        }
        cudaSetDevice(prev);
        cudaGetLastError();
        n_ = 0, held_ = 0;
        return n;
    }
    // Keeps a buffer no kernel uses any more; false when the cache is full (the caller frees it).
    bool give(int dev, void* p, size_t bytes) {
        std::lock_guard<std::mutex> lock(m_);
        if (n_ == kSlots || held_ + bytes > kBytes) return false;
        e_[n_++] = {dev, p, bytes};
        held_ += bytes;
        return true;
    }

  private:
    static constexpr int kSlots = 256;
    struct Entry {
        int dev;
        void* p;
        size_t bytes;
    };
    std::mutex m_;
    Entry e_[kSlots];
    int n_ = 0;
    size_t held_ = 0;
};

// Owns device allocations for one call or one plan. With `recycle` (set by calls that synchronise their work before
// returning, never by plans, whose callers may destroy them with kernels in flight) the buffers come from and go back
// to the BufferCache; on an error path they are freed as usual, since kernels may still be using them.
struct DeviceArena {
    void* ptrs[64] = {};
    size_t sizes[64] = {};
    int n = 0;
    int dev = -1;
    bool recycle = false;
    ~DeviceArena() { release(); }
    void release() {
        const bool keep = recycle && std::uncaught_exceptions() == 0;
        for (int i = 0; i < n; ++i)
            if (!keep || !BufferCache::get().give(dev, ptrs[i], sizes[i])) cudaFree(ptrs[i]);
        n = 0;
    }
    void* raw(size_t bytes) {
        if (n == 64) throw Error(OB_ENOMEM, "too many device buffers");
        const size_t want = bytes ? bytes : 16;
        size_t got = want;
        void* d = nullptr;
        if (recycle) {
            if (dev < 0) check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
            d = BufferCache::get().take(dev, want, got);
        }
        if (!d) {
            got = want;
            const cudaError_t e = cudaMalloc(&d, want);
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw Error(OB_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
            }
        }
        ptrs[n] = d, sizes[n] = got, ++n;
        return d;
    }
    template <typename T>
    T* alloc(size_t count) {
        return static_cast<T*>(raw(count * sizeof(T)));
    }
    // Host array of count elements of T, already in the device's layout, to a new device buffer in one copy.
    template <typename T>
    T* put_raw(const T* host, size_t count) {
        T* d = alloc<T>(count);
        check_cuda(cudaMemcpy(d, host, count * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy (inputs)");
        return d;
    }
    // Host array of count elements (converted to T) to a new device buffer; null or empty gives null. An array already
    // of T is copied as it is (no host copy to convert into).
    template <typename T, typename S>
    T* put(const S* host, size_t count, cudaStream_t st = nullptr) {
        if (!host || !count) return nullptr;
        T* d = alloc<T>(count);
        if constexpr (std::is_same_v<T, S>) {
            check_cuda(cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync (inputs)");
            check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize (inputs)");
            return d;
        }
        T* tmp = static_cast<T*>(std::malloc(count * sizeof(T)));
        if (!tmp) throw std::bad_alloc();
        for (size_t i = 0; i < count; ++i) tmp[i] = static_cast<T>(host[i]);
        const cudaError_t e = cudaMemcpyAsync(d, tmp, count * sizeof(T), cudaMemcpyHostToDevice, st);
        const cudaError_t e2 = cudaStreamSynchronize(st);
        std::free(tmp);
        check_cuda(e, "cudaMemcpyAsync (inputs)");
        check_cuda(e2, "cudaStreamSynchronize (inputs)");
        return d;
    }
};

// A call's inputs gathered into one host buffer and copied to the device in one transfer by commit(): a call with
// many small inputs pays one copy's driver work instead of one for each (a few microseconds apiece). add() converts
// to T as DeviceArena::put does (null or empty gives a null pointer) and names the pointer that receives the device
// address; the pointers hold their addresses once commit() has returned.
class Upload {
  public:
    template <typename T, typename S, typename P>
    void add(P*& field, const S* host, size_t count) {
        static_assert(std::is_same_v<std::remove_const_t<P>, T>, "the field points to T");
        if (!host || !count) {
            field = nullptr;
            return;
        }
        const size_t off = (bytes_.size() + 15) & ~static_cast<size_t>(15);
        bytes_.resize(off + count * sizeof(T));
        T* out = reinterpret_cast<T*>(bytes_.data() + off);
        if constexpr (std::is_same_v<T, S>) std::memcpy(out, host, count * sizeof(T));
        else
            for (size_t i = 0; i < count; ++i) out[i] = static_cast<T>(host[i]);
        fixes_.push_back({off, [&field](unsigned char* base) { field = reinterpret_cast<P*>(base); }});
    }
    // count zero-filled elements of T
    template <typename T, typename P>
    void zeros(P*& field, size_t count) {
        static_assert(std::is_same_v<std::remove_const_t<P>, T>, "the field points to T");
        const size_t off = (bytes_.size() + 15) & ~static_cast<size_t>(15);
        bytes_.resize(off + count * sizeof(T), 0);
        fixes_.push_back({off, [&field](unsigned char* base) { field = reinterpret_cast<P*>(base); }});
    }
    void commit(DeviceArena& arena) {
        if (bytes_.empty()) return;
        unsigned char* d = arena.alloc<unsigned char>(bytes_.size());
        check_cuda(cudaMemcpy(d, bytes_.data(), bytes_.size(), cudaMemcpyHostToDevice), "cudaMemcpy (inputs)");
        for (const Fix& f : fixes_) f.set(d + f.off);
    }

  private:
    struct Fix {
        size_t off;
        std::function<void(unsigned char*)> set;
    };
    std::vector<unsigned char> bytes_;
    std::vector<Fix> fixes_;
};

// ------------------------------------------------------------------------------------------------ normals

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t& x, uint32_t& y, uint32_t& z, uint32_t& w,
                                                       uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        // one 32 x 32 -> 64-bit product gives both halves (a single wide multiply on the device)
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * x, p1 = static_cast<uint64_t>(0xCD9E8D57u) * z;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        const uint32_t nx = hi1 ^ y ^ k0, nz = hi0 ^ w ^ k1;
        x = nx, y = lo1, z = nz, w = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

template <typename R>
__device__ __forceinline__ R to_unit(uint32_t i);
template <>
__device__ __forceinline__ float to_unit<float>(uint32_t i) {
    return static_cast<float>(i) * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
}
template <>
__device__ __forceinline__ double to_unit<double>(uint32_t i) {
    return static_cast<double>(i) * 2.3283064365386963e-10 + 1.1641532182693481e-10;
}

// Float: the radius with the precise logarithm (near u = 1 an approximate one's absolute error would be a large part
// of the small radius); the angle 2 pi v taken as 2 pi (v - 1/2) + pi, inside [-pi, pi), where the hardware sine and
// cosine keep an absolute error near 1e-6 (a normal moves by a few 1e-6 at most, |z| <= 6.7: inside the reference's
// float-against-double criteria), the shift by pi flipping both signs. The angle 2 pi (b + 1/2) 2^-32 - pi is one
// multiply-add from b in float (b's conversion rounds as v's does, the sum once: within 3.9e-7 of the exact angle,
// as 2 pi (v - 1/2) computed in steps is).
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, float& z0, float& z1) {
    const float r = sqrtf(-2.0f * logf(to_unit<float>(a)));
    float s, c;
    // 2 pi 2^-32 and pi 2^-32 - pi, rounded to float
    __sincosf(fmaf(static_cast<float>(b), 1.46291807926715968e-09f, -3.14159265285070240f), &s, &c);
    z0 = -r * c, z1 = -r * s;
}
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, double& z0, double& z1) {
    const double r = sqrt(-2.0 * log(to_unit<double>(a)));
    double s, c;
    sincospi(2.0 * to_unit<double>(b), &s, &c);
    z0 = r * c, z1 = r * s;
}

// The four normals of block `block` of one pair's stream.
template <typename R>
__device__ __forceinline__ void normals4(uint64_t pair, uint64_t block, uint32_t tag, uint32_t k0, uint32_t k1,
                                         R& z0, R& z1, R& z2, R& z3) {
    uint32_t x = static_cast<uint32_t>(pair), y = static_cast<uint32_t>(pair >> 32);
    uint32_t z = static_cast<uint32_t>(block), w = static_cast<uint32_t>(block >> 32) | tag;
    philox4x32_10(x, y, z, w, k0, k1);
    box_muller(x, y, z0, z1);
    box_muller(z, w, z2, z3);
}

// Normals of one pair along one stream, read in order (block b gives normals 4b .. 4b+3). The buffer stays in
// registers: the slot is picked by selects, never by a dynamic index.
template <typename R>
struct NormalStream {
    uint64_t pair;
    uint64_t block;
    uint32_t k0, k1, tag;
    int used;
    R b0, b1, b2, b3;

    __device__ __forceinline__ void init(uint64_t p, uint32_t key0, uint32_t key1, uint32_t t) {
        pair = p, block = 0, k0 = key0, k1 = key1, tag = t, used = 4;
        b0 = b1 = b2 = b3 = R(0);
    }
    __device__ __forceinline__ R next() {
        if (used == 4) {
            normals4<R>(pair, block, tag, k0, k1, b0, b1, b2, b3);
            ++block, used = 0;
        }
        const R z = used == 0 ? b0 : used == 1 ? b1 : used == 2 ? b2 : b3;
        ++used;
        return z;
    }
};

// ------------------------------------------------------------------------------------------------ math helpers

__device__ __forceinline__ float m_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double m_abs(double x) { return fabs(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double m_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_log(float x) { return logf(x); }
__device__ __forceinline__ double m_log(double x) { return log(x); }
__device__ __forceinline__ float m_ncdf(float x) { return normcdff(x); }
__device__ __forceinline__ double m_ncdf(double x) { return normcdf(x); }
template <typename R>
__device__ __forceinline__ R m_max(R a, R b) { return a > b ? a : b; }
template <typename R>
__device__ __forceinline__ R m_min(R a, R b) { return a < b ? a : b; }

// Warp sum of a double.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

}  // namespace ob
