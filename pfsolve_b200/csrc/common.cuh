// common.cuh -- device helpers shared by the JW-step kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dd.cuh"

namespace pfb {

constexpr unsigned FULL = 0xffffffffu;

// ---- value types: real systems use double, complex systems double2 (re, im
// of one complex right-hand side share the real matrix).
template <class V> struct VOps;

template <> struct VOps<double> {
    static __device__ __forceinline__ double zero() { return 0.0; }
    static __device__ __forceinline__ double mul(double a, double v) { return a * v; }
    // a*v + w
    static __device__ __forceinline__ double fma(double a, double v, double w) { return __fma_rn(a, v, w); }
    static __device__ __forceinline__ double add(double v, double w) { return v + w; }
    static __device__ __forceinline__ double shfl_up(double v, int d) { return __shfl_up_sync(FULL, v, d); }
    static __device__ __forceinline__ double shfl_down(double v, int d) { return __shfl_down_sync(FULL, v, d); }
};

template <> struct VOps<double2> {
    static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
    static __device__ __forceinline__ double2 mul(double a, double2 v) { return make_double2(a * v.x, a * v.y); }
    static __device__ __forceinline__ double2 fma(double a, double2 v, double2 w)
    {
        return make_double2(__fma_rn(a, v.x, w.x), __fma_rn(a, v.y, w.y));
    }
    static __device__ __forceinline__ double2 add(double2 v, double2 w) { return make_double2(v.x + w.x, v.y + w.y); }
    static __device__ __forceinline__ double2 shfl_up(double2 v, int d)
    {
        return make_double2(__shfl_up_sync(FULL, v.x, d), __shfl_up_sync(FULL, v.y, d));
    }
    static __device__ __forceinline__ double2 shfl_down(double2 v, int d)
    {
        return make_double2(__shfl_down_sync(FULL, v.x, d), __shfl_down_sync(FULL, v.y, d));
    }
};

template <> struct VOps<float> {
    static __device__ __forceinline__ float zero() { return 0.0f; }
    static __device__ __forceinline__ float mul(float a, float v) { return a * v; }
    static __device__ __forceinline__ float fma(float a, float v, float w) { return __fmaf_rn(a, v, w); }
    static __device__ __forceinline__ float add(float v, float w) { return v + w; }
    static __device__ __forceinline__ float shfl_up(float v, int d) { return __shfl_up_sync(FULL, v, d); }
    static __device__ __forceinline__ float shfl_down(float v, int d) { return __shfl_down_sync(FULL, v, d); }
};

template <> struct VOps<float2> {
    static __device__ __forceinline__ float2 zero() { return make_float2(0.0f, 0.0f); }
    static __device__ __forceinline__ float2 mul(float a, float2 v) { return make_float2(a * v.x, a * v.y); }
    static __device__ __forceinline__ float2 fma(float a, float2 v, float2 w)
    {
        return make_float2(__fmaf_rn(a, v.x, w.x), __fmaf_rn(a, v.y, w.y));
    }
    static __device__ __forceinline__ float2 add(float2 v, float2 w) { return make_float2(v.x + w.x, v.y + w.y); }
    static __device__ __forceinline__ float2 shfl_up(float2 v, int d)
    {
        return make_float2(__shfl_up_sync(FULL, v.x, d), __shfl_up_sync(FULL, v.y, d));
    }
    static __device__ __forceinline__ float2 shfl_down(float2 v, int d)
    {
        return make_float2(__shfl_down_sync(FULL, v.x, d), __shfl_down_sync(FULL, v.y, d));
    }
};

template <> struct VOps<dd> {
    static __device__ __forceinline__ dd zero() { return dd(0.0, 0.0); }
    static __device__ __forceinline__ dd mul(dd a, dd v) { return a * v; }
    static __device__ __forceinline__ dd fma(dd a, dd v, dd w) { return dd_fma(a, v, w); }
    static __device__ __forceinline__ dd add(dd v, dd w) { return v + w; }
    static __device__ __forceinline__ dd shfl_up(dd v, int d)
    {
        return dd(__shfl_up_sync(FULL, v.hi, d), __shfl_up_sync(FULL, v.lo, d));
    }
    static __device__ __forceinline__ dd shfl_down(dd v, int d)
    {
        return dd(__shfl_down_sync(FULL, v.hi, d), __shfl_down_sync(FULL, v.lo, d));
    }
};

// Shuffles of the scan multiplier type (double, float or dd).
template <class S> __device__ __forceinline__ S shfl_up_s(S v, int d) { return __shfl_up_sync(FULL, v, d); }
template <class S> __device__ __forceinline__ S shfl_down_s(S v, int d) { return __shfl_down_sync(FULL, v, d); }
template <> __device__ __forceinline__ dd shfl_up_s<dd>(dd v, int d) { return VOps<dd>::shfl_up(v, d); }
template <> __device__ __forceinline__ dd shfl_down_s<dd>(dd v, int d) { return VOps<dd>::shfl_down(v, d); }

// FP64 <-> FP32 value conversions (round to nearest when narrowing).
__device__ __forceinline__ float to_f32(double v) { return __double2float_rn(v); }
__device__ __forceinline__ float2 to_f32(double2 v) { return make_float2(__double2float_rn(v.x), __double2float_rn(v.y)); }
__device__ __forceinline__ double to_f64(float v) { return (double)v; }
__device__ __forceinline__ double2 to_f64(float2 v) { return make_double2((double)v.x, (double)v.y); }
template <class V> struct Lower;
template <> struct Lower<double> { using type = float; };
template <> struct Lower<double2> { using type = float2; };
template <> struct Lower<float> { using type = float; };
template <> struct Lower<float2> { using type = float2; };

// Two-component vector of a scalar type (complex values: re, im).
template <class S> struct Vec2Of;
template <> struct Vec2Of<double> { using type = double2; };
template <> struct Vec2Of<float> { using type = float2; };

// Value conversions between storage and arithmetic types (FP32 <-> FP64,
// real or complex; round to nearest when narrowing).
__device__ __forceinline__ void cvt(double& d, double s) { d = s; }
__device__ __forceinline__ void cvt(double& d, float s) { d = (double)s; }
__device__ __forceinline__ void cvt(float& d, double s) { d = __double2float_rn(s); }
__device__ __forceinline__ void cvt(float& d, float s) { d = s; }
__device__ __forceinline__ void cvt(double2& d, double2 s) { d = s; }
__device__ __forceinline__ void cvt(double2& d, float2 s) { d = make_double2((double)s.x, (double)s.y); }
__device__ __forceinline__ void cvt(float2& d, double2 s) { d = make_float2(__double2float_rn(s.x), __double2float_rn(s.y)); }
__device__ __forceinline__ void cvt(float2& d, float2 s) { d = s; }
template <class D, class S>
__device__ __forceinline__ D conv(S s)
{
    D d;
    cvt(d, s);
    return d;
}

template <int R> struct Log2 { static constexpr int v = (R <= 1) ? 0 : 1 + Log2<R / 2>::v; };
template <> struct Log2<1> { static constexpr int v = 0; };

// ---- Shared-memory swizzle for a warp segment of 32*R rows.
// Lanes write the segment coalesced (row q = 32k + lane) and read it blocked
// (lane t reads rows R*t .. R*t+R-1).  XORing the low bits of the element
// index with the chunk index keeps both patterns free of bank conflicts:
// 8-byte elements are served 16 lanes per wavefront (16 bank pairs), 16-byte
// elements 8 lanes per wavefront (8 bank quads).
template <int R, bool CPLX>
__device__ __forceinline__ int swz(int e)
{
    if constexpr (R == 1) {
        return e;
    } else {
        constexpr int L2 = Log2<R>::v;
        constexpr int MASK = CPLX ? 7 : 15;
        return e ^ ((e >> L2) & MASK);
    }
}

// ---- cp.async (global -> shared, bypassing registers); bytes beyond
// src_size are zero-filled, which implements out-of-range and zeropad rows.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid)
{
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    int src = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool valid)
{
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    int src = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(src) : "memory");
}
// One element of 4 or 8 bytes (an FP32 or FP64 value).
template <class T>
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem, bool valid)
{
    if constexpr (sizeof(T) == 4) cp_async4(smem, gmem, valid);
    else cp_async8(smem, gmem, valid);
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid)
{
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    int src = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src) : "memory");
}
// 16 bytes of shared memory from the first `nbytes` (0, 4, 8, 12 or 16)
// bytes at gmem, the rest zero-filled; no byte beyond them is read.
__device__ __forceinline__ void cp_async16n(void* smem, const void* gmem, int nbytes)
{
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---- Named barrier over the `nthreads` threads of one system group.
__device__ __forceinline__ void group_bar(int id, int nthreads)
{
    asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}

// ---- Exact power-of-two renormalisation of a 2x2 matrix (keeps continuant
// products in range without rounding).
__device__ __forceinline__ void renorm2x2(double& a, double& b, double& c, double& d)
{
    double m = fmax(fmax(fabs(a), fabs(b)), fmax(fabs(c), fabs(d)));
    if (m > 0.0 && isfinite(m)) {
        int e = ilogb(m);
        a = scalbn(a, -e);
        b = scalbn(b, -e);
        c = scalbn(c, -e);
        d = scalbn(d, -e);
    }
}

}  // namespace pfb
