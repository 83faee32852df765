// Two cells per thread.  The second-generation single-level stage kernels
// (bgf_flow2.cuh) give each thread two vertically adjacent cells and evaluate
// both with one instruction stream: a value of the pair type V2<T> holds the two
// cells' values.  For FP32 in the fast build the pair is one 64-bit register and
// additions, subtractions, products and fused multiply-adds use the paired FP32
// instructions of sm_100 (add / sub / mul / fma .f32x2, PTX ISA 8.6): one issue
// slot for both cells.  Comparisons, min / max, selects, division and square root
// act per lane.  FP64 pairs are two scalars.
//
// Every operation is the IEEE operation of the scalar code it replaces.  The
// paired instructions are used in the fast build only, which may contract products
// into fused multiply-adds and flushes subnormals: measured on B200, kernels built
// from the paired forms did not reproduce the separately rounded scalar sequence
// bit for bit (an isolated test of each form did), so the exact build evaluates
// the two lanes with scalar IEEE operations (`__fadd_rn` / `__fmul_rn`, never
// contracted) and keeps the bit-exact contract of the one-cell kernels.
//
// Included inside namespace bgf::BGF_VARIANT (each arithmetic variant compiles its
// own copy with its own flags).
#pragma once

template <class T> struct V2 {
    T a, b;
};
struct M2 {
    bool a, b;
};

__device__ __forceinline__ M2 operator&&(M2 x, M2 y) { return M2{x.a && y.a, x.b && y.b}; }
__device__ __forceinline__ M2 operator||(M2 x, M2 y) { return M2{x.a || y.a, x.b || y.b}; }
__device__ __forceinline__ M2 operator!(M2 x) { return M2{!x.a, !x.b}; }

// ---------------------------------------------------------------- scalars
template <class T> __device__ __forceinline__ T add(T x, T y) { return x + y; }
template <class T> __device__ __forceinline__ T sub(T x, T y) { return x - y; }
template <class T> __device__ __forceinline__ T mul(T x, T y) { return x * y; }
template <class T> __device__ __forceinline__ T mad(T x, T y, T z) { return x * y + z; }
template <class T> __device__ __forceinline__ T dv(T x, T y) { return x / y; }
template <class T> __device__ __forceinline__ T vsqrt(T x) { return M<T>::sqrt_(x); }
template <class T> __device__ __forceinline__ T vmin(T x, T y) { return M<T>::fmin_(x, y); }
template <class T> __device__ __forceinline__ T vmax(T x, T y) { return M<T>::fmax_(x, y); }
template <class T> __device__ __forceinline__ T vabs(T x) { return M<T>::fabs_(x); }
template <class T> __device__ __forceinline__ bool lt(T x, T y) { return x < y; }
template <class T> __device__ __forceinline__ bool gt(T x, T y) { return x > y; }
template <class T> __device__ __forceinline__ bool ge(T x, T y) { return x >= y; }
template <class T> __device__ __forceinline__ bool le(T x, T y) { return x <= y; }
template <class T> __device__ __forceinline__ bool eq(T x, T y) { return x == y; }
template <class T> __device__ __forceinline__ T sel(bool m, T x, T y) { return m ? x : y; }

// ---------------------------------------------------------------- FP32 pairs
#if BGF_FAST
__device__ __forceinline__ unsigned long long pk(V2<float> v)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.a), "f"(v.b));
    return r;
}
__device__ __forceinline__ V2<float> upk(unsigned long long r)
{
    V2<float> v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.a), "=f"(v.b) : "l"(r));
    return v;
}
__device__ __forceinline__ V2<float> add(V2<float> x, V2<float> y)
{
    unsigned long long r;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(x)), "l"(pk(y)));
    return upk(r);
}
__device__ __forceinline__ V2<float> sub(V2<float> x, V2<float> y)
{
    unsigned long long r;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(x)), "l"(pk(y)));
    return upk(r);
}
__device__ __forceinline__ V2<float> mul(V2<float> x, V2<float> y)
{
    unsigned long long r;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(x)), "l"(pk(y)));
    return upk(r);
}
__device__ __forceinline__ V2<float> mad(V2<float> x, V2<float> y, V2<float> z)
{
    unsigned long long r;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk(x)), "l"(pk(y)), "l"(pk(z)));
    return upk(r);
}
// Quotients in the fast build: the numerator times the hardware reciprocal
// approximation of the denominator (rcp.approx.ftz.f32, at most 1 ulp off, one
// multi-function-unit instruction), so a pair of quotients costs two reciprocals and
// one paired product instead of two full-range divisions.  A zero denominator gives
// an infinite reciprocal, as the division gives an infinite or NaN quotient; every
// caller selects such a lane away (dry cells, faces with no wave speed).
__device__ __forceinline__ float rcpa(float y)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
    return r;
}
__device__ __forceinline__ float dv(float x, float y) { return x * rcpa(y); }
__device__ __forceinline__ V2<float> dv(V2<float> x, V2<float> y) { return mul(x, V2<float>{rcpa(y.a), rcpa(y.b)}); }
// Cube root for Manning's friction factor: h^(1/3) = 2^(log2(h) / 3) with the
// hardware base-2 logarithm and exponential approximations (relative error about
// 1e-7 |log2 h| on the depths of wet cells; h = 0 gives 0).
__device__ __forceinline__ float cbrta(float h)
{
    float l, r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(h));
    l *= 0.333333343f;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(l));
    return r;
}
#else
__device__ __forceinline__ V2<float> add(V2<float> x, V2<float> y) { return V2<float>{__fadd_rn(x.a, y.a), __fadd_rn(x.b, y.b)}; }
__device__ __forceinline__ V2<float> sub(V2<float> x, V2<float> y) { return V2<float>{__fsub_rn(x.a, y.a), __fsub_rn(x.b, y.b)}; }
__device__ __forceinline__ V2<float> mul(V2<float> x, V2<float> y) { return V2<float>{__fmul_rn(x.a, y.a), __fmul_rn(x.b, y.b)}; }
__device__ __forceinline__ V2<float> mad(V2<float> x, V2<float> y, V2<float> z) { return add(mul(x, y), z); }
#endif

// ---------------------------------------------------------------- FP64 pairs
__device__ __forceinline__ V2<double> add(V2<double> x, V2<double> y) { return V2<double>{x.a + y.a, x.b + y.b}; }
__device__ __forceinline__ V2<double> sub(V2<double> x, V2<double> y) { return V2<double>{x.a - y.a, x.b - y.b}; }
__device__ __forceinline__ V2<double> mul(V2<double> x, V2<double> y) { return V2<double>{x.a * y.a, x.b * y.b}; }
__device__ __forceinline__ V2<double> mad(V2<double> x, V2<double> y, V2<double> z)
{
    return V2<double>{x.a * y.a + z.a, x.b * y.b + z.b};
}

// ---------------------------------------------------------------- per-lane operations on pairs
template <class T> __device__ __forceinline__ V2<T> dv(V2<T> x, V2<T> y) { return V2<T>{x.a / y.a, x.b / y.b}; }
template <class T> __device__ __forceinline__ V2<T> vsqrt(V2<T> x) { return V2<T>{M<T>::sqrt_(x.a), M<T>::sqrt_(x.b)}; }
template <class T> __device__ __forceinline__ V2<T> vmin(V2<T> x, V2<T> y)
{
    return V2<T>{M<T>::fmin_(x.a, y.a), M<T>::fmin_(x.b, y.b)};
}
template <class T> __device__ __forceinline__ V2<T> vmax(V2<T> x, V2<T> y)
{
    return V2<T>{M<T>::fmax_(x.a, y.a), M<T>::fmax_(x.b, y.b)};
}
template <class T> __device__ __forceinline__ V2<T> vabs(V2<T> x) { return V2<T>{M<T>::fabs_(x.a), M<T>::fabs_(x.b)}; }
template <class T> __device__ __forceinline__ T vcopysign(T x, T y)
{
    if constexpr (sizeof(T) == 4) return copysignf(x, y);
    else return copysign(x, y);
}
template <class T> __device__ __forceinline__ V2<T> vcopysign(V2<T> x, V2<T> y)
{
    return V2<T>{vcopysign<T>(x.a, y.a), vcopysign<T>(x.b, y.b)};
}
template <class T> __device__ __forceinline__ M2 lt(V2<T> x, V2<T> y) { return M2{x.a < y.a, x.b < y.b}; }
template <class T> __device__ __forceinline__ M2 gt(V2<T> x, V2<T> y) { return M2{x.a > y.a, x.b > y.b}; }
template <class T> __device__ __forceinline__ M2 ge(V2<T> x, V2<T> y) { return M2{x.a >= y.a, x.b >= y.b}; }
template <class T> __device__ __forceinline__ M2 le(V2<T> x, V2<T> y) { return M2{x.a <= y.a, x.b <= y.b}; }
template <class T> __device__ __forceinline__ M2 eq(V2<T> x, V2<T> y) { return M2{x.a == y.a, x.b == y.b}; }
template <class T> __device__ __forceinline__ V2<T> sel(M2 m, V2<T> x, V2<T> y)
{
    return V2<T>{m.a ? x.a : y.a, m.b ? x.b : y.b};
}

// Scalar type of a value type (T for T, T for V2<T>) and its mask type.
template <class V> struct LaneOf {
    using T = V;
    using Mask = bool;
};
template <class S> struct LaneOf<V2<S>> {
    using T = S;
    using Mask = M2;
};
