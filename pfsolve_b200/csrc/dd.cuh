// dd.cuh -- double-double ("quad emulation") arithmetic for the JW step.
//
// A value is an unevaluated sum hi + lo with |lo| <= ulp(hi)/2 (~106-bit
// significand), the representation PfSolve's quadDoubleDoublePrecision mode
// stores as pf_quad2 {x = hi, y = lo}
// (PfSolve/pfSolve_CodeGen/pfSolve_KernelsLevel0/pfSolve_KernelUtils.h:122-150).
// The operations are the published error-free transformations:
//   two_sum        Knuth, TAOCP vol. 2 (4.2.2, Theorem B)
//   quick_two_sum  Dekker 1971 (|a| >= |b|)
//   two_prod       product error through one fused multiply-add
// combined as in Hida, Li and Bailey, "Library for double-double and
// quad-double arithmetic" (2001): accurate addition, multiplication, and
// long division with two correction steps.  Division uses the hardware
// division of the leading terms (the `/` operator).
#pragma once
#include <cuda_runtime.h>

namespace pfb {

struct dd {
    double hi, lo;
    __host__ __device__ dd() : hi(0.0), lo(0.0) {}
    __host__ __device__ dd(double h) : hi(h), lo(0.0) {}
    __host__ __device__ dd(double h, double l) : hi(h), lo(l) {}
};

__device__ __forceinline__ dd two_sum(double a, double b)
{
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return dd(s, e);
}

__device__ __forceinline__ dd quick_two_sum(double a, double b)
{
    const double s = a + b;
    return dd(s, b - (s - a));
}

__device__ __forceinline__ dd two_prod(double a, double b)
{
    const double p = a * b;
    return dd(p, __fma_rn(a, b, -p));
}

__device__ __forceinline__ dd operator+(dd a, dd b)
{
    dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = quick_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return quick_two_sum(s.hi, s.lo);
}

__device__ __forceinline__ dd operator-(dd a) { return dd(-a.hi, -a.lo); }
__device__ __forceinline__ dd operator-(dd a, dd b) { return a + (-b); }

__device__ __forceinline__ dd operator*(dd a, dd b)
{
    dd p = two_prod(a.hi, b.hi);
    p.lo = __fma_rn(a.hi, b.lo, p.lo);
    p.lo = __fma_rn(a.lo, b.hi, p.lo);
    return quick_two_sum(p.hi, p.lo);
}

__device__ __forceinline__ dd operator*(double a, dd b) { return dd(a) * b; }

__device__ __forceinline__ dd operator/(dd a, dd b)
{
    const double q1 = a.hi / b.hi;
    dd r = a - b * dd(q1);
    const double q2 = r.hi / b.hi;
    r = r - b * dd(q2);
    const double q3 = r.hi / b.hi;
    const dd q = quick_two_sum(q1, q2);
    return q + dd(q3);
}

__device__ __forceinline__ bool dd_is_zero(dd a) { return a.hi == 0.0; }

// a*v + w: the product's two terms (two_prod and the cross terms) go into
// the accurate addition as they are, without the quick_two_sum that would
// renormalise them first -- the addition's two_sum steps are exact for any
// pair of doubles, and the result is renormalised at its end.  Three FP64
// operations fewer than a * v + w.
__device__ __forceinline__ dd dd_fma(dd a, dd v, dd w)
{
    dd p = two_prod(a.hi, v.hi);
    p.lo = __fma_rn(a.hi, v.lo, p.lo);
    p.lo = __fma_rn(a.lo, v.hi, p.lo);
    return p + w;
}

}  // namespace pfb
