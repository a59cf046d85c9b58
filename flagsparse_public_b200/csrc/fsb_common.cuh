// fsb_common.cuh -- element types, accumulator algebra, cache-hinted loads and
// warp-segment reductions shared by the sm_100a sparse kernels.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include "../../include/flagsparse_b200.h"

namespace fsb {

// Merge-path units of the SpMM kernels hold at most this many items (rows +
// nonzeros; a unit's nonzero count is kept in 32 bits).  Unit coordinates
// must come from fsb_merge_partition for the same matrix and items.
constexpr int32_t kMaxItemsPerUnit = 1 << 24;

// ---------------------------------------------------------------- types ----
struct __align__(4) c32_t { __half re, im; };
struct __align__(8) c64_t { float re, im; };
struct __align__(16) c128_t { double re, im; };

// f32 accumulator carrying a running error term (Dot2, Ogita-Rump-Oishi 2005):
// value = s + c.  Products enter through TwoProduct (FMA residual) and sums
// through TwoSum, so the result is as if accumulated in about twice f32
// precision and rounded once.
struct __align__(8) comp_t { float s, c; };

// ------------------------------------------------------ raw cache loads ----
template <int BYTES> struct raw_type;
template <> struct raw_type<2>  { using T = unsigned short; };
template <> struct raw_type<4>  { using T = unsigned int; };
template <> struct raw_type<8>  { using T = uint2; };
template <> struct raw_type<16> { using T = uint4; };

template <class T, int N> struct vec_t { T v[N]; };

// Streaming load (evict-first in L1 and L2): the sparse matrix is read once.
template <class T, int N>
__device__ __forceinline__ vec_t<T, N> ld_stream(const T* p) {
    using R = typename raw_type<sizeof(T) * N>::T;
    R r = __ldcs(reinterpret_cast<const R*>(p));
    vec_t<T, N> out;
    memcpy(&out, &r, sizeof(R));
    return out;
}
// Read-only cached load: x / B are gathered many times.
template <class T, int N>
__device__ __forceinline__ vec_t<T, N> ld_ro(const T* p) {
    using R = typename raw_type<sizeof(T) * N>::T;
    R r = __ldg(reinterpret_cast<const R*>(p));
    vec_t<T, N> out;
    memcpy(&out, &r, sizeof(R));
    return out;
}
// L2 policy that keeps lines resident (dense operands gathered many times
// while the sparse stream passes through once).
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// Read-only load with an L2 cache policy (2, 4, 8 or 16 bytes).
template <class T, int N>
__device__ __forceinline__ vec_t<T, N> ld_keep(const T* p, uint64_t pol) {
    constexpr int BY = (int)sizeof(T) * N;
    vec_t<T, N> out;
    if constexpr (BY == 2) {
        unsigned short r;
        asm("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(r) : "l"(p), "l"(pol));
        memcpy(&out, &r, 2);
    } else if constexpr (BY == 4) {
        unsigned int r;
        asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(r) : "l"(p), "l"(pol));
        memcpy(&out, &r, 4);
    } else if constexpr (BY == 8) {
        uint2 r;
        asm("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(r.x), "=r"(r.y) : "l"(p), "l"(pol));
        memcpy(&out, &r, 8);
    } else {
        static_assert(BY == 16, "ld_keep: 2, 4, 8 or 16 bytes");
        uint4 r;
        asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
            : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
            : "l"(p), "l"(pol));
        memcpy(&out, &r, 16);
    }
    return out;
}
template <class T>
__device__ __forceinline__ T ld_stream1(const T* p) { return ld_stream<T, 1>(p).v[0]; }
template <class T>
__device__ __forceinline__ T ld_ro1(const T* p) { return ld_ro<T, 1>(p).v[0]; }

template <class T, int N>
__device__ __forceinline__ void st_stream(T* p, const vec_t<T, N>& v) {
    using R = typename raw_type<sizeof(T) * N>::T;
    R r;
    memcpy(&r, &v, sizeof(R));
    __stcs(reinterpret_cast<R*>(p), r);
}
template <class T>
__device__ __forceinline__ void st_stream1(T* p, T v) {
    vec_t<T, 1> w; w.v[0] = v; st_stream<T, 1>(p, w);
}

// Indices: 64-bit arithmetic everywhere, whatever the stored width.
template <class I> __device__ __forceinline__ int64_t idx(I v) { return (int64_t)v; }

// bfloat16 is the upper half of a float32: widening is a 16-bit shift on the
// integer pipe (exact)
__device__ __forceinline__ float widen_bf16(__nv_bfloat16 v) {
    unsigned short u;
    memcpy(&u, &v, 2);
    return __uint_as_float((unsigned)u << 16);
}

// ------------------------------------------------------ accumulator ops ----
// Acc<V, A>: how a product of two V values enters an A accumulator.
template <class V, class A> struct Acc;

#define FSB_REAL_ACC(VT, AT, CONV)                                              \
    template <> struct Acc<VT, AT> {                                            \
        static __device__ __forceinline__ AT zero() { return (AT)0; }           \
        static __device__ __forceinline__ AT fma(VT a, VT b, AT acc) {          \
            return ::fma((AT)CONV(a), (AT)CONV(b), acc);                        \
        }                                                                       \
    };
#define FSB_ID(v) (v)
FSB_REAL_ACC(float, float, FSB_ID)
FSB_REAL_ACC(float, double, FSB_ID)
FSB_REAL_ACC(double, double, FSB_ID)
FSB_REAL_ACC(__half, float, __half2float)
FSB_REAL_ACC(__nv_bfloat16, float, widen_bf16)
#undef FSB_REAL_ACC

template <> struct Acc<c64_t, c64_t> {
    static __device__ __forceinline__ c64_t zero() { return c64_t{0.f, 0.f}; }
    static __device__ __forceinline__ c64_t fma(c64_t a, c64_t b, c64_t acc) {
        acc.re = fmaf(a.re, b.re, acc.re);
        acc.re = fmaf(-a.im, b.im, acc.re);
        acc.im = fmaf(a.re, b.im, acc.im);
        acc.im = fmaf(a.im, b.re, acc.im);
        return acc;
    }
};
// complex32: float16 pairs widened to float32 in registers (FlagSparse
// accumulates complex32 in float32, spmm_csr.py:576-598)
template <> struct Acc<c32_t, c64_t> {
    static __device__ __forceinline__ c64_t zero() { return c64_t{0.f, 0.f}; }
    static __device__ __forceinline__ c64_t fma(c32_t a, c32_t b, c64_t acc) {
        const float ar = __half2float(a.re), ai = __half2float(a.im);
        const float br = __half2float(b.re), bi = __half2float(b.im);
        acc.re = fmaf(ar, br, acc.re);
        acc.re = fmaf(-ai, bi, acc.re);
        acc.im = fmaf(ar, bi, acc.im);
        acc.im = fmaf(ai, br, acc.im);
        return acc;
    }
};
template <> struct Acc<c64_t, c128_t> {
    static __device__ __forceinline__ c128_t zero() { return c128_t{0.0, 0.0}; }
    static __device__ __forceinline__ c128_t fma(c64_t a, c64_t b, c128_t acc) {
        acc.re = ::fma((double)a.re, (double)b.re, acc.re);
        acc.re = ::fma(-(double)a.im, (double)b.im, acc.re);
        acc.im = ::fma((double)a.re, (double)b.im, acc.im);
        acc.im = ::fma((double)a.im, (double)b.re, acc.im);
        return acc;
    }
};
template <> struct Acc<c128_t, c128_t> {
    static __device__ __forceinline__ c128_t zero() { return c128_t{0.0, 0.0}; }
    static __device__ __forceinline__ c128_t fma(c128_t a, c128_t b, c128_t acc) {
        acc.re = ::fma(a.re, b.re, acc.re);
        acc.re = ::fma(-a.im, b.im, acc.re);
        acc.im = ::fma(a.re, b.im, acc.im);
        acc.im = ::fma(a.im, b.re, acc.im);
        return acc;
    }
};

__device__ __forceinline__ float to_f32(float v) { return v; }
__device__ __forceinline__ float to_f32(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_f32(__nv_bfloat16 v) { return widen_bf16(v); }

// TwoSum (Knuth): s + p = t + e exactly.
__device__ __forceinline__ comp_t comp_add_value(comp_t acc, float p, float p_err) {
    float t = acc.s + p;
    float z = t - acc.s;
    float e = (acc.s - (t - z)) + (p - z);
    acc.s = t;
    acc.c = acc.c + (e + p_err);
    return acc;
}
template <class V> struct Acc<V, comp_t> {
    static __device__ __forceinline__ comp_t zero() { return comp_t{0.f, 0.f}; }
    static __device__ __forceinline__ comp_t fma(V a, V b, comp_t acc) {
        float fa = to_f32(a), fb = to_f32(b);
        float p = fa * fb;
        float pe = fmaf(fa, fb, -p);  // TwoProduct residual
        return comp_add_value(acc, p, pe);
    }
};

// Sum of two accumulators (reductions, carries).
__device__ __forceinline__ float acc_add(float a, float b) { return a + b; }
__device__ __forceinline__ double acc_add(double a, double b) { return a + b; }
__device__ __forceinline__ c64_t acc_add(c64_t a, c64_t b) { return c64_t{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ c128_t acc_add(c128_t a, c128_t b) { return c128_t{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ comp_t acc_add(comp_t a, comp_t b) {
    comp_t r = comp_add_value(a, b.s, 0.f);
    r.c += b.c;
    return r;
}

// Shuffles of accumulators and values.
__device__ __forceinline__ float shfl_xor(unsigned m, float v, int o, int w) { return __shfl_xor_sync(m, v, o, w); }
__device__ __forceinline__ double shfl_xor(unsigned m, double v, int o, int w) { return __shfl_xor_sync(m, v, o, w); }
__device__ __forceinline__ c64_t shfl_xor(unsigned m, c64_t v, int o, int w) {
    return c64_t{__shfl_xor_sync(m, v.re, o, w), __shfl_xor_sync(m, v.im, o, w)};
}
__device__ __forceinline__ c128_t shfl_xor(unsigned m, c128_t v, int o, int w) {
    return c128_t{__shfl_xor_sync(m, v.re, o, w), __shfl_xor_sync(m, v.im, o, w)};
}
__device__ __forceinline__ comp_t shfl_xor(unsigned m, comp_t v, int o, int w) {
    return comp_t{__shfl_xor_sync(m, v.s, o, w), __shfl_xor_sync(m, v.c, o, w)};
}

__device__ __forceinline__ float shfl_up(unsigned m, float v, int o) { return __shfl_up_sync(m, v, o); }
__device__ __forceinline__ double shfl_up(unsigned m, double v, int o) { return __shfl_up_sync(m, v, o); }
__device__ __forceinline__ c64_t shfl_up(unsigned m, c64_t v, int o) {
    return c64_t{__shfl_up_sync(m, v.re, o), __shfl_up_sync(m, v.im, o)};
}
__device__ __forceinline__ c128_t shfl_up(unsigned m, c128_t v, int o) {
    return c128_t{__shfl_up_sync(m, v.re, o), __shfl_up_sync(m, v.im, o)};
}
__device__ __forceinline__ comp_t shfl_up(unsigned m, comp_t v, int o) {
    return comp_t{__shfl_up_sync(m, v.s, o), __shfl_up_sync(m, v.c, o)};
}

// Broadcast shuffles of stored values / indices (SpMM nonzero broadcast).
template <class T>
__device__ __forceinline__ T shfl_idx(unsigned m, T v, int src, int w) { return __shfl_sync(m, v, src, w); }
template <>
__device__ __forceinline__ c64_t shfl_idx(unsigned m, c64_t v, int src, int w) {
    return c64_t{__shfl_sync(m, v.re, src, w), __shfl_sync(m, v.im, src, w)};
}
template <>
__device__ __forceinline__ c32_t shfl_idx(unsigned m, c32_t v, int src, int w) {
    unsigned u;
    memcpy(&u, &v, 4);
    u = __shfl_sync(m, u, src, w);
    c32_t r;
    memcpy(&r, &u, 4);
    return r;
}
template <>
__device__ __forceinline__ c128_t shfl_idx(unsigned m, c128_t v, int src, int w) {
    return c128_t{__shfl_sync(m, v.re, src, w), __shfl_sync(m, v.im, src, w)};
}

// Reduce across a power-of-two segment of `width` lanes (xor butterfly over
// offsets first..width/2).  All lanes of the segment end with the total.
template <class A>
__device__ __forceinline__ A segment_reduce(unsigned mask, A v, int first, int width) {
    for (int o = first; o < width; o <<= 1) v = acc_add(v, shfl_xor(mask, v, o, width));
    return v;
}

// Atomic accumulation (COO atomic routes; relaxed, order not deterministic).
__device__ __forceinline__ void atomic_accumulate(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_accumulate(double* p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_accumulate(c64_t* p, c64_t v) {
    atomicAdd(&p->re, v.re);
    atomicAdd(&p->im, v.im);
}
__device__ __forceinline__ void atomic_accumulate(c128_t* p, c128_t v) {
    atomicAdd(&p->re, v.re);
    atomicAdd(&p->im, v.im);
}

// -------------------------------------------------- output conversion ----
template <class O, class A> struct Out;
template <> struct Out<float, float>   { static __device__ __forceinline__ float  cvt(float a)  { return a; } };
template <> struct Out<float, double>  { static __device__ __forceinline__ float  cvt(double a) { return (float)a; } };
template <> struct Out<double, double> { static __device__ __forceinline__ double cvt(double a) { return a; } };
template <> struct Out<__half, float>  { static __device__ __forceinline__ __half cvt(float a)  { return __float2half_rn(a); } };
template <> struct Out<__nv_bfloat16, float> {
    static __device__ __forceinline__ __nv_bfloat16 cvt(float a) { return __float2bfloat16_rn(a); }
};
template <> struct Out<c32_t, c64_t>   {
    static __device__ __forceinline__ c32_t cvt(c64_t a) { return c32_t{__float2half_rn(a.re), __float2half_rn(a.im)}; }
};
template <> struct Out<c64_t, c64_t>   { static __device__ __forceinline__ c64_t cvt(c64_t a) { return a; } };
template <> struct Out<c64_t, c128_t>  {
    static __device__ __forceinline__ c64_t cvt(c128_t a) { return c64_t{(float)a.re, (float)a.im}; }
};
template <> struct Out<c128_t, c128_t> { static __device__ __forceinline__ c128_t cvt(c128_t a) { return a; } };
template <> struct Out<float, comp_t>  { static __device__ __forceinline__ float cvt(comp_t a) { return a.s + a.c; } };
template <> struct Out<__half, comp_t> {
    static __device__ __forceinline__ __half cvt(comp_t a) { return __float2half_rn(a.s + a.c); }
};
template <> struct Out<__nv_bfloat16, comp_t> {
    static __device__ __forceinline__ __nv_bfloat16 cvt(comp_t a) { return __float2bfloat16_rn(a.s + a.c); }
};

// Zero of a stored value type (padding lanes of a broadcast).
template <class V> __device__ __forceinline__ V vzero() { return V(0); }
template <> __device__ __forceinline__ __half vzero<__half>() { return __float2half(0.f); }
template <> __device__ __forceinline__ __nv_bfloat16 vzero<__nv_bfloat16>() { return __float2bfloat16(0.f); }
template <> __device__ __forceinline__ c32_t vzero<c32_t>() { return c32_t{__float2half(0.f), __float2half(0.f)}; }
template <> __device__ __forceinline__ c64_t vzero<c64_t>() { return c64_t{0.f, 0.f}; }
template <> __device__ __forceinline__ c128_t vzero<c128_t>() { return c128_t{0.0, 0.0}; }

// Lanes of a 16-byte vector for value type V (used for A and B streams).
template <class V> struct VecWidth { static constexpr int value = 16 / (int)sizeof(V); };

// Mask of the `width`-lane segment of the warp that contains `lane`.
__device__ __forceinline__ unsigned segment_mask(int lane, int width) {
    if (width >= 32) return 0xffffffffu;
    unsigned base = (unsigned)(lane & ~(width - 1));
    return ((1u << width) - 1u) << base;
}

__host__ __device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace fsb

// ------------------------------------------------------------ host side ----
namespace fsb_host {
void set_error(const char* fmt, ...);
int check_launch(const char* what);
}  // namespace fsb_host
