// The specialised fused kernel: every name of one kind (Black-Scholes, local vol, Heston by Euler, SLV, or one Heston
// name by QE), N names known at compile time, everything a step reads staged in shared memory.
//
// Per step and name one 16-byte record {lo, inv_dx, log-forward at the step end, table row} (32 bytes in double)
// is read as a warp-wide broadcast; the local-variance table is stored as (y_i, y_i+1) pairs so that an
// interpolation is one 8-byte shared load. Normals are drawn in batches of G steps whose count is a multiple of four,
// so each Philox block fills registers by constant indices; the correlated normal root z is computed once per pair
// and step and used with both signs (the reference's two legs read the same z with opposite signs,
// RC/include/optlab_cuda/paths.hpp:301-329). Each leg's step is the reference's arithmetic up to reassociation:
// x += var (-dt / 2) + sqrt(var) sqrt(dt) z with -dt / 2 and sqrt(dt) precomputed per step, and the table read as
// y + w dy.
#pragma once

#include "model.cuh"

namespace ob {

// org and inv_dx locate x in the step's row: in the cell form (set_cell_row, the fused, script and path kernels) or in
// the form of u = table_u(step, x) (the adjoint): -lo inv_dx in float (u = x inv_dx + org, one multiply-add), lo in
// double (u = (x - lo) inv_dx, the reference's order).
template <typename R>
struct alignas(16) NameStep;
template <>
struct alignas(16) NameStep<float> {
    float org, inv_dx, lf;
    int row;  // first (y_i, y_i+1) pair of the step's table row
};
template <>
struct alignas(16) NameStep<double> {
    double org, inv_dx, lf;
    int row, pad;
};

__host__ __device__ inline float name_step_org(double lo, double inv_dx, float*) {
    return static_cast<float>(-lo * inv_dx);
}
__host__ __device__ inline double name_step_org(double lo, double, double*) { return lo; }
// The origin to store for a row starting at lo with 1 / dx = inv_dx.
template <typename R>
__host__ __device__ inline R name_step_org(double lo, double inv_dx) {
    return name_step_org(lo, inv_dx, static_cast<R*>(nullptr));
}

__device__ __forceinline__ float table_u(float org, float inv_dx, float x) { return fmaf(x, inv_dx, org); }
__device__ __forceinline__ double table_u(double org, double inv_dx, double x) { return (x - org) * inv_dx; }
template <typename R>
__device__ __forceinline__ R table_u(const NameStep<R>& s, R x) {
    return table_u(s.org, s.inv_dx, x);
}

// The cell form of a row, for the kernels that need only a coordinate's interval and weight (the fused, script and
// path kernels; the adjoint keeps table_u's form for its derivative). In float the coordinate is stored divided by
// top, so that its clamp to [0, top] is the saturation of its multiply-add: u / top = sat(x inv_dx / top - lo inv_dx
// / top). In double the row keeps table_u's form.
inline void cell_row(double lo, double inv_dx, float top, float& org, float& inv) {
    org = static_cast<float>(-lo * inv_dx / top), inv = static_cast<float>(inv_dx / top);
}
inline void cell_row(double lo, double inv_dx, double, double& org, double& inv) { org = lo, inv = inv_dx; }
template <typename R>
inline void set_cell_row(NameStep<R>& r, double lo, double inv_dx, R top) {
    cell_row(lo, inv_dx, top, r.org, r.inv_dx);
}

// The interval j = floor(u) and the weight f = u - j of x's coordinate u, clamped to [0, top], in a row of the cell
// form. Float: s = sat(x inv_dx' + org') = u / top; s top + 2^23 rounded toward zero is a float in [2^23, 2^24)
// whose low mantissa bits hold floor(u) exactly (u < 2^23), and f = s top - floor(u) in one more multiply-add (the
// subtraction 2^23 - that float is exact). Four FMA-pipe instructions where the clamp, the conversion to an integer
// and back and the subtraction take six, two of them on the MUFU pipe. Double: the clamp and the conversions.
__device__ __forceinline__ void table_cell(float org, float inv, float top, float x, int& j, float& f) {
    float s;
    asm("fma.rn.ftz.sat.f32 %0, %1, %2, %3;" : "=f"(s) : "f"(x), "f"(inv), "f"(org));
    const float big = __fmaf_rz(s, top, 8388608.0f);
    j = __float_as_int(big) - 0x4B000000;
    f = fmaf(s, top, 8388608.0f - big);
}
__device__ __forceinline__ void table_cell(double org, double inv, double top, double x, int& j, double& f) {
    const double u = fmin(fmax(table_u(org, inv, x), 0.0), top);
    j = static_cast<int>(u);
    f = u - static_cast<double>(j);
}
template <typename R>
__device__ __forceinline__ void table_cell(const NameStep<R>& r, R top, R x, int& j, R& f) {
    table_cell(r.org, r.inv_dx, top, x, j, f);
}

// One leg's log-spot step, x + var (-dt / 2) + sqrt(var) (sqrt(dt) z): in float as two multiply-adds (the drift into
// x, then the diffusion), in double in the reference's grouping (the two terms summed, then added to x).
__device__ __forceinline__ float lv_advance(float x, float var, float hdt, float zd) {
    return fmaf(sqrtf(var), zd, fmaf(var, hdt, x));
}
__device__ __forceinline__ double lv_advance(double x, double var, double hdt, double zd) {
    return x + fma(sqrt(var), zd, var * hdt);
}

// One table interval: the value at its left point and the increment to the right one, so that an interpolation is
// one multiply-add (y + w dy, the reference's y_i (1 - w) + y_i+1 w up to rounding).
template <typename R>
struct alignas(2 * sizeof(R)) Pair2 {
    R a, b;
};

// An interval of a table left in global memory (too large for the shared-memory stage): one 8- or 16-byte load
// through the read-only data cache.
__device__ __forceinline__ Pair2<float> ldg_pair(const Pair2<float>* p) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return {v.x, v.y};
}
__device__ __forceinline__ Pair2<double> ldg_pair(const Pair2<double>* p) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return {v.x, v.y};
}

// A record of whole 16-byte words (StepRec, NameStep) read from global memory through the read-only data cache: the
// compiler may then issue the load ahead of the kernel's stores and reductions, which a plain load could alias.
template <typename T>
__device__ __forceinline__ T ldg_rec(const T* p) {
    static_assert(sizeof(T) % 16 == 0 && alignof(T) >= 16, "a record of whole 16-byte words");
    T out;
    const int4* src = reinterpret_cast<const int4*>(p);
    int4* dst = reinterpret_cast<int4*>(&out);
#pragma unroll
    for (int k = 0; k < static_cast<int>(sizeof(T) / 16); ++k) dst[k] = __ldg(src + k);
    return out;
}

// Per step: -dt / 2, sqrt(dt), dt, and the index of the observation taken at the step's end (negative: none; in an
// autocall minus the number of steps to the next observation).
template <typename R>
struct alignas(16) StepRec {
    R hdt, sdt, dt;
    int obs;
};

// Byte offsets inside the staged blob.
struct FusedOffsets {
    int step, name_step, root, hes, table2, ln_trig, obs_disc, leg_type, leg_strike, leg_barrier, ln_level;
    int mix_den, low_root;  // local correlation: per step sigma sqrt(max(t0, 1/12)); the aligned low root
};

template <typename R>
struct FusedArgs {
    FusedOffsets off;
    const unsigned char* blob;
    int smem_blob;
    int n_steps, n_obs, n_out, n_legs, n_x, same;
    R top;  // n_x - 1 - 1e-4, the clamp of the table interpolation
    QeConsts<R> qe;
    R spot0;
    double discount;
    int has_coupon, memory, ki_daily;
    R ln_cb, ln_ki;
    double coupon, put_strike;
    const Pair2<R>* tab;  // the table in global memory when it does not fit the stage (kernels with GT), else unused
    // local correlation (kernels with MIX): w0 + level, down, up, sign, cos, sin of the mixer (paths.hpp:219-237)
    R mix_base, mix_down, mix_up, mix_sign, mix_cos, mix_sin;
};

}  // namespace ob
