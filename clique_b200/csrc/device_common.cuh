// Scalar helpers shared by the kernels: a value type V<T,C> that is T for
// real data and an aligned (re, im) pair for complex data, with the few
// operators the kernels need.  Storage arrays are T* with complex entries
// interleaved, so element e of a complex array lives at T offset 2e.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

namespace cliqgpu {

template <class T>
struct alignas(2 * sizeof(T)) cx {
    T r, i;
};

template <class T> __host__ __device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return {a.r + b.r, a.i + b.i}; }
template <class T> __host__ __device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return {a.r - b.r, a.i - b.i}; }
template <class T> __host__ __device__ __forceinline__ cx<T> operator*(cx<T> a, cx<T> b) {
    return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r};
}
template <class T> __host__ __device__ __forceinline__ cx<T> operator*(cx<T> a, T s) { return {a.r * s, a.i * s}; }
template <class T> __host__ __device__ __forceinline__ cx<T> operator/(cx<T> a, cx<T> b) {
    // Smith's algorithm for complex division
    if (fabs(b.r) >= fabs(b.i)) {
        T q = b.i / b.r, den = b.r + b.i * q;
        return {(a.r + a.i * q) / den, (a.i - a.r * q) / den};
    } else {
        T q = b.r / b.i, den = b.r * q + b.i;
        return {(a.r * q + a.i) / den, (a.i * q - a.r) / den};
    }
}
template <class T> __host__ __device__ __forceinline__ cx<T>& operator+=(cx<T>& a, cx<T> b) { a.r += b.r; a.i += b.i; return a; }
template <class T> __host__ __device__ __forceinline__ cx<T>& operator-=(cx<T>& a, cx<T> b) { a.r -= b.r; a.i -= b.i; return a; }

template <class T, bool C>
using V = typename std::conditional<C, cx<T>, T>::type;

// Whether an earlier bounded wait gave up (status[1] set): read once per
// CTA by thread 0 and shared, so that every thread of the CTA takes the same
// branch (a flag set by another CTA between two threads' reads would
// otherwise split the CTA at its barriers).
__device__ __forceinline__ bool cta_timed_out(const int32_t* status) {
    __shared__ int s_timed_out;
    if (threadIdx.x == 0) s_timed_out = *reinterpret_cast<const volatile int32_t*>(&status[1]) != 0;
    __syncthreads();
    return s_timed_out != 0;
}

template <class T> __device__ __forceinline__ T conjv(T a) { return a; }
template <class T> __device__ __forceinline__ cx<T> conjv(cx<T> a) { return {a.r, -a.i}; }
template <bool CJ, class X> __device__ __forceinline__ X opc(X a) { if constexpr (CJ) return conjv(a); else return a; }

template <class X> __device__ __forceinline__ X vzero() { return X{}; }
template <class X> __device__ __forceinline__ X vone();
template <> __device__ __forceinline__ float vone<float>() { return 1.f; }
template <> __device__ __forceinline__ double vone<double>() { return 1.0; }
template <> __device__ __forceinline__ cx<float> vone<cx<float>>() { return {1.f, 0.f}; }
template <> __device__ __forceinline__ cx<double> vone<cx<double>>() { return {1.0, 0.0}; }

template <class X> __device__ __forceinline__ bool is_zero(X a) { return a == X(0); }
template <class T> __device__ __forceinline__ bool is_zero(cx<T> a) { return a.r == T(0) && a.i == T(0); }

// fused multiply-accumulate acc += a*b
__device__ __forceinline__ void mac(float& acc, float a, float b) { acc = fmaf(a, b, acc); }
__device__ __forceinline__ void mac(double& acc, double a, double b) { acc = fma(a, b, acc); }
template <class T> __device__ __forceinline__ void mac(cx<T>& acc, cx<T> a, cx<T> b) {
    acc.r = fma(a.r, b.r, acc.r); acc.r = fma(-a.i, b.i, acc.r);
    acc.i = fma(a.r, b.i, acc.i); acc.i = fma(a.i, b.r, acc.i);
}

// element load / store from a T* arena
template <class T, bool C> __device__ __forceinline__ V<T, C> ldv(const T* p, int64_t e) {
    return reinterpret_cast<const V<T, C>*>(p)[e];
}
template <class T, bool C> __device__ __forceinline__ void stv(T* p, int64_t e, V<T, C> v) {
    reinterpret_cast<V<T, C>*>(p)[e] = v;
}
// L2-coherent load (bypasses L1) for data produced by other CTAs of the same launch
template <class T, bool C> __device__ __forceinline__ V<T, C> ldv_cg(const T* p, int64_t e) {
    if constexpr (C) {
        if constexpr (sizeof(T) == 8) {
            double2 v = __ldcg(reinterpret_cast<const double2*>(p) + e);
            return V<T, C>{(T)v.x, (T)v.y};
        } else {
            float2 v = __ldcg(reinterpret_cast<const float2*>(p) + e);
            return V<T, C>{(T)v.x, (T)v.y};
        }
    } else {
        return __ldcg(p + e);
    }
}

// conversions between precisions
template <class To, class From> __device__ __forceinline__ To cvt(From a) { return (To)a; }
template <class To, class From> __device__ __forceinline__ cx<To> cvtc(cx<From> a) { return {(To)a.r, (To)a.i}; }

template <class Dst, class Src> struct Conv { __device__ static Dst go(Src a) { return (Dst)a; } };
template <class A, class B> struct Conv<cx<A>, cx<B>> { __device__ static cx<A> go(cx<B> a) { return {(A)a.r, (A)a.i}; } };
template <class Dst, class Src> __device__ __forceinline__ Dst conv(Src a) { return Conv<Dst, Src>::go(a); }

// FP64 pivot storage: D is double (real) or cx<double> (complex)
template <bool C> using DV = typename std::conditional<C, cx<double>, double>::type;

}  // namespace cliqgpu
