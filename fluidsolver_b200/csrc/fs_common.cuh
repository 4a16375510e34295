// Shared device definitions of the B200 hot path: precision-generic vector
// math, the cubic spline kernel, compensated neighbor accumulators, and the
// status word every kernel checks.
//
// Operation order. The FP32 precision mode reproduces the reference's float
// arithmetic operation by operation (glm's scalar code path, compiled without
// FMA contraction; this library is built with -fmad=false), so that with the
// reference's neighbor order the results are bit-identical. The comments name
// the reference expression each helper evaluates.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fluidsolver_b200.h"

// Pointer qualifiers of the search and solver code. FSB_R is __restrict__
// and FSB_LDG a read-only-cache load, except in a translation unit that
// defines FSB_COHERENT_LOADS first: there kernels read data that earlier
// phases of the same kernel wrote (the small-scene step kernel), which the
// non-coherent read-only path must not serve, so both become plain.
#ifdef FSB_COHERENT_LOADS
#define FSB_R
#define FSB_LDG(p) (*(p))
#else
#define FSB_R __restrict__
#define FSB_LDG(p) __ldg(p)
#endif

namespace fsb {

// ---------------------------------------------------------------------------
// precision-generic 3-vectors (2D runs through the same code with z == 0: every
// z product and sum is then exactly +-0 and leaves x/y results bit-identical)
// ---------------------------------------------------------------------------
template <typename R> struct V3 {
    R x, y, z;
};

template <typename R> struct Vec4T;
template <> struct Vec4T<float> { using type = float4; };
template <> struct Vec4T<double> { using type = double4; };
template <typename R> using V4 = typename Vec4T<R>::type;

template <typename R> __host__ __device__ __forceinline__ V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> xyz(const V4<R>& a) { return {a.x, a.y, a.z}; }
template <typename R> __host__ __device__ __forceinline__ V4<R> v4(const V3<R>& a, R w) {
    V4<R> r;
    r.x = a.x; r.y = a.y; r.z = a.z; r.w = w;
    return r;
}
template <typename R> __host__ __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
// glm::dot: (a.x*b.x + a.y*b.y) + a.z*b.z
template <typename R> __host__ __device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// FLT_EPSILON, the reference's "is zero" threshold (LibFluidMath.hpp:238-244)
constexpr float kFltEps = 1.19209290e-07f;

// ---------------------------------------------------------------------------
// cubic spline kernel (CubicSplineKernel.cpp:9-63, CubicSplineKernel3D.cpp:7-66)
// ---------------------------------------------------------------------------
template <typename R> struct SplineKernel {
    R h;      // kernel_support / 2
    R alpha;  // 5/(14 pi h^2) in 2D, 1/(4 pi h^3) in 3D

    // GetKernelValue(position - neighborPosition); d = x_i - x_j
    __device__ __forceinline__ R W(V3<R> d) const {
        R q = sqrt_(dot(d, d)) / h;
        R ret = R(0);
        if (q < R(1)) {
            R a = R(2) - q, b = R(1) - q;
            ret = ((a * a) * a) - R(4) * ((b * b) * b);
        } else if (q < R(2)) {
            R a = R(2) - q;
            ret = (a * a) * a;
        }
        return alpha * ret;
    }

    // GetKernelDerivativeReversedValue(x_j, x_i), i.e. the gradient of W at
    // x_i - x_j: alpha * ((h * d_c) / |d|) * poly(q); zero for |d| <= FLT_EPSILON.
    __device__ __forceinline__ V3<R> gradW(V3<R> d) const {
        R len = sqrt_(dot(d, d));
        R q = len / h;
        V3<R> pre = v3<R>(0, 0, 0);
        if (len > R(kFltEps)) pre = v3<R>((h * d.x) / len, (h * d.y) / len, (h * d.z) / len);
        if (q < R(1)) {
            R a = R(2) - q, b = R(1) - q;
            R poly = R(-3) * (a * a) + R(12) * (b * b);
            return v3<R>(alpha * (pre.x * poly), alpha * (pre.y * poly), alpha * (pre.z * poly));
        } else if (q < R(2)) {
            R a = R(2) - q;
            R poly = R(-3) * (a * a);
            return v3<R>(alpha * (pre.x * poly), alpha * (pre.y * poly), alpha * (pre.z * poly));
        }
        return v3<R>(0, 0, 0);
    }

    static __device__ __forceinline__ R sqrt_(R x);

    // ---- fast evaluation (compensated-sum mode): one rsqrt, no divisions,
    // fused multiply-adds. The same piecewise cubic; rounding differs from the
    // reference's by a few ulp per pair.
    R inv_h;     // 1 / h
    R alpha_h;   // alpha * h

    __device__ __forceinline__ R Wf(V3<R> d) const {
        const R r2 = fma_(d.z, d.z, fma_(d.y, d.y, d.x * d.x));
        const R q = sqrt_fast(r2) * inv_h;
        const R a = R(2) - q, b = R(1) - q;
        if (q < R(1)) return alpha * fma_(R(-4) * b * b, b, a * a * a);
        if (q < R(2)) return alpha * (a * a * a);
        return R(0);
    }
    __device__ __forceinline__ V3<R> gradWf(V3<R> d) const {
        const R r2 = fma_(d.z, d.z, fma_(d.y, d.y, d.x * d.x));
        if (!(r2 > R(kFltEps) * R(kFltEps))) return v3<R>(0, 0, 0);
        const R inv = rsqrt_fast(r2);
        const R q = r2 * inv * inv_h;
        const R a = R(2) - q, b = R(1) - q;
        R poly;
        if (q < R(1)) poly = fma_(R(12) * b, b, R(-3) * a * a);
        else if (q < R(2)) poly = R(-3) * a * a;
        else return v3<R>(0, 0, 0);
        const R f = alpha_h * poly * inv;
        return v3<R>(f * d.x, f * d.y, f * d.z);
    }
    template <bool FAST> __device__ __forceinline__ R w(V3<R> d) const { return FAST ? Wf(d) : W(d); }
    template <bool FAST> __device__ __forceinline__ V3<R> grad(V3<R> d) const { return FAST ? gradWf(d) : gradW(d); }

    static __device__ __forceinline__ R fma_(R a, R b, R c);
    static __device__ __forceinline__ R rsqrt_fast(R x);
    static __device__ __forceinline__ R sqrt_fast(R x);
};
template <> __device__ __forceinline__ float SplineKernel<float>::fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <> __device__ __forceinline__ double SplineKernel<double>::fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
template <> __device__ __forceinline__ float SplineKernel<float>::rsqrt_fast(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double SplineKernel<double>::rsqrt_fast(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float SplineKernel<float>::sqrt_fast(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }
template <> __device__ __forceinline__ double SplineKernel<double>::sqrt_fast(double x) { return sqrt(x); }

// dot product: glm's (x*x' + y*y') + z*z' in the exact modes, fused in the fast mode
template <bool FAST, typename R> __device__ __forceinline__ R dotf(V3<R> a, V3<R> b) {
    if (FAST) return SplineKernel<R>::fma_(a.z, b.z, SplineKernel<R>::fma_(a.y, b.y, a.x * b.x));
    return dot(a, b);
}

// division: exact (reference order) or reciprocal-based (fast mode)
template <bool FAST> __device__ __forceinline__ float fdiv(float a, float b) { return FAST ? __fdividef(a, b) : a / b; }
template <bool FAST> __device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
template <> __device__ __forceinline__ float SplineKernel<float>::sqrt_(float x) { return __fsqrt_rn(x); }
template <> __device__ __forceinline__ double SplineKernel<double>::sqrt_(double x) { return __dsqrt_rn(x); }

// ---------------------------------------------------------------------------
// neighbor-sum accumulators: plain (reference order) or Kahan-compensated
// ---------------------------------------------------------------------------
template <typename R, bool KAHAN> struct Acc {
    R s = R(0), c = R(0);
    __device__ __forceinline__ void add(R v) {
        if (KAHAN) {
            R y = v - c;
            R t = s + y;
            c = (t - s) - y;
            s = t;
        } else {
            s = s + v;
        }
    }
    __device__ __forceinline__ void sub(R v) {
        if (KAHAN) add(-v);
        else s = s - v;
    }
    __device__ __forceinline__ R get() const { return s; }
};

template <typename R, bool KAHAN> struct Acc3 {
    Acc<R, KAHAN> x, y, z;
    __device__ __forceinline__ void add(V3<R> v) { x.add(v.x); y.add(v.y); z.add(v.z); }
    __device__ __forceinline__ void sub(V3<R> v) { x.sub(v.x); y.sub(v.y); z.sub(v.z); }
    __device__ __forceinline__ V3<R> get() const { return {x.get(), y.get(), z.get()}; }
};

// ---------------------------------------------------------------------------
// neighbor list entries: sorted particle index, top bit set for boundary
// ---------------------------------------------------------------------------
constexpr uint32_t kBoundaryBit = 0x80000000u;
constexpr uint32_t kIndexMask = 0x7fffffffu;

// device status word (first error wins)
__device__ __forceinline__ void raise_status(int* status, int code) { atomicCAS(status, 0, code); }

// Programmatic dependent launch (a kernel launched with programmatic stream
// serialization may start while the kernel before it still runs):
// grid_dependency_wait blocks until that kernel has completed and its writes
// are visible (at once when launched without the attribute);
// launch_dependents lets the next such kernel start early.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// One scene's cell grid: dims, this step's origin (cell coordinates) and the
// offset of its cells in the concatenated cell tables.
struct SceneGrid {
    int d0, d1, d2;
    int o0, o1, o2;
    long long base;
};

// per-step device scalars shared by the kernels of one step (one set per scene)
struct StepScalars {
    float desired_dt;        // Timepoint::desired_time_step
    float dt;                // current_timestep (after the CFL clamp: actual)
    int iteration;           // IISPH iterations done
    int done;                // IISPH early-exit flag
    double err_sum;          // FP64 residual sum of this iteration
    unsigned long long err_count;
    unsigned int max_err_bits;  // non-negative float maxima as ordered bits
    unsigned int max_a2_bits;
    unsigned int max_v2_bits;
    float avg_err;           // stat_last_average_predicted_density_error
    double avg_err64;
    float max_err;
    float final_max_a2;      // of the last iteration (CFL input)
    float final_max_v2;
    int max_neighbors;
    int loop_guard;          // executions of the pressure-loop body this step
    unsigned int gen_v2_bits;   // dynamic time step generator: largest |v|^2, |a|^2 at the step's start
    unsigned int gen_a2_bits;
};

}  // namespace fsb
