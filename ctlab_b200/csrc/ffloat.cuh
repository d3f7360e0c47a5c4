// Float-float ("compensated FP32 pair") arithmetic used by the F32PAIR SAT
// variant.  A value is hi + lo with |lo| <= ulp(hi)/2.  Additions use
// Knuth's TwoSum and Dekker's Fast2Sum; products use the FMA-based exact
// product.  All additions go through __fadd_rn / __fsub_rn so the compiler
// cannot contract or reassociate them.
#pragma once

struct ff2 {
    float hi, lo;
};

__device__ __forceinline__ ff2 ff_two_sum(float a, float b)
{
    float s = __fadd_rn(a, b);
    float bb = __fsub_rn(s, a);
    float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return {s, e};
}

__device__ __forceinline__ ff2 ff_fast_two_sum(float a, float b)
{
    float s = __fadd_rn(a, b);
    float e = __fsub_rn(b, __fsub_rn(s, a));
    return {s, e};
}

__device__ __forceinline__ ff2 ff_add(ff2 a, ff2 b)
{
    ff2 s = ff_two_sum(a.hi, b.hi);
    ff2 t = ff_two_sum(a.lo, b.lo);
    s.lo = __fadd_rn(s.lo, t.hi);
    s = ff_fast_two_sum(s.hi, s.lo);
    s.lo = __fadd_rn(s.lo, t.lo);
    return ff_fast_two_sum(s.hi, s.lo);
}

__device__ __forceinline__ ff2 ff_neg(ff2 a) { return {-a.hi, -a.lo}; }

__device__ __forceinline__ ff2 ff_sub(ff2 a, ff2 b) { return ff_add(a, ff_neg(b)); }

// a * f for a float-float a and a float f (exact product of the high part).
__device__ __forceinline__ ff2 ff_mul_f(ff2 a, float f)
{
    float p = __fmul_rn(a.hi, f);
    float e = __fmaf_rn(a.hi, f, -p);
    e = __fmaf_rn(a.lo, f, e);
    return ff_fast_two_sum(p, e);
}

__device__ __forceinline__ float ff_to_float(ff2 a) { return __fadd_rn(a.hi, a.lo); }
