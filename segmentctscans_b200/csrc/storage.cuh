// Storage formats of the solver state (Xi, V, Vbar).  Arithmetic is FP32 for
// the FP32 and 16-bit formats (FP64 for the FP64 state): a load widens
// exactly, a store rounds to nearest, ties to even.  So
// that every kernel form sees the same values, anything the reference keeps in
// memory (Xi, V, Vbar) is rounded to the storage format before it is used
// again, also when a kernel keeps it on chip.
//
// bfloat16 keeps 8 mantissa bits: rounded to nearest, the stored V of a
// converging solve stops moving once an update is below half a unit in the
// last place, and the solve settles away from the FP32 one.  The stored V of
// that format is therefore rounded stochastically, with random bits from a
// counter-based hash of (line, slice n, iteration, pair of components): the
// rounding is unbiased, reproducible, and identical in every kernel form.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>
#include <type_traits>

namespace potts {

// "lowbias32" mixer of Chris Wellons' hash-prospector (public domain).
__host__ __device__ __forceinline__ uint32_t sr_mix(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// 32 random bits for components 2*pair and 2*pair+1 (low and high half) of
// the V stored at (line, global slice n) by the primal step of iteration it
// (0-based).  Key multipliers: the golden-ratio and xxHash32 primes.
__host__ __device__ __forceinline__ uint32_t sr_hash(uint32_t line, uint32_t n, uint32_t it, uint32_t pair)
{
    return sr_mix((line * 0x9e3779b1u) ^ (n * 0x85ebca77u) ^ ((it * 4u + pair) * 0xc2b2ae3du));
}

// The 16 random bits of V component i from the hashes h[i / 2].
__device__ __forceinline__ uint32_t sr_bits(uint32_t h, int i) { return (i & 1) ? (h >> 16) : (h & 0xffffu); }

template <typename T>
struct Store;

template <>
struct Store<float> {
    using Real = float;  // arithmetic type of the kernels for this format
    static constexpr bool kExact = true;
    static constexpr bool kStochasticV = false;
    __device__ __forceinline__ static float st_v(float x, uint32_t) { return x; }
    __device__ __forceinline__ static float ld(float x) { return x; }
    __device__ __forceinline__ static float st(float x) { return x; }
    __device__ __forceinline__ static float round(float x) { return x; }
    __device__ __forceinline__ static float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
    __device__ __forceinline__ static void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
};

template <>
struct Store<__nv_bfloat16> {
    using Real = float;
    static constexpr bool kExact = false;
    static constexpr bool kStochasticV = true;
    // stored V: add 16 random bits below the kept half of the binary32
    // pattern, then cut (finite values only; V is always finite)
    __device__ __forceinline__ static __nv_bfloat16 st_v(float x, uint32_t bits)
    {
        uint32_t b = __float_as_uint(x);
        if ((b & 0x7fffffffu) < 0x7f800000u) b += bits;
        return __ushort_as_bfloat16((unsigned short)(b >> 16));
    }
    __device__ __forceinline__ static float ld(__nv_bfloat16 x) { return __bfloat162float(x); }
    __device__ __forceinline__ static __nv_bfloat16 st(float x) { return __float2bfloat16_rn(x); }
    __device__ __forceinline__ static float round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
    __device__ __forceinline__ static float2 ld2(const __nv_bfloat16 *p)
    {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p));
    }
    __device__ __forceinline__ static void st2(__nv_bfloat16 *p, float2 v)
    {
        *reinterpret_cast<__nv_bfloat162 *>(p) = __float22bfloat162_rn(v);
    }
    // two stored values as one 32-bit word (the first in the low half), widened / rounded
    __device__ __forceinline__ static float2 cvt2(uint32_t w)
    {
        return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
    }
    __device__ __forceinline__ static uint32_t pack2(float2 v)
    {
        const __nv_bfloat162 b = __float22bfloat162_rn(v);
        return (uint32_t)__bfloat16_as_ushort(b.x) | ((uint32_t)__bfloat16_as_ushort(b.y) << 16);
    }
};

template <>
struct Store<__half> {
    using Real = float;
    static constexpr bool kExact = false;
    static constexpr bool kStochasticV = false;
    __device__ __forceinline__ static __half st_v(float x, uint32_t) { return __float2half_rn(x); }
    __device__ __forceinline__ static float ld(__half x) { return __half2float(x); }
    __device__ __forceinline__ static __half st(float x) { return __float2half_rn(x); }
    __device__ __forceinline__ static float round(float x) { return __half2float(__float2half_rn(x)); }
    __device__ __forceinline__ static float2 ld2(const __half *p)
    {
        return __half22float2(*reinterpret_cast<const __half2 *>(p));
    }
    __device__ __forceinline__ static void st2(__half *p, float2 v)
    {
        *reinterpret_cast<__half2 *>(p) = __float22half2_rn(v);
    }
    __device__ __forceinline__ static float2 cvt2(uint32_t w)
    {
        return __half22float2(__halves2half2(__ushort_as_half((unsigned short)(w & 0xffffu)),
                                             __ushort_as_half((unsigned short)(w >> 16))));
    }
    __device__ __forceinline__ static uint32_t pack2(float2 v)
    {
        const __half2 h = __float22half2_rn(v);
        return (uint32_t)__half_as_ushort(__low2half(h)) | ((uint32_t)__half_as_ushort(__high2half(h)) << 16);
    }
};

// FP64 state with FP64 arithmetic: the split kernels only (the FP64 solve,
// large-volume counterpart of the CPU oracle).
template <>
struct Store<double> {
    using Real = double;
    static constexpr bool kExact = true;
    static constexpr bool kStochasticV = false;
    __device__ __forceinline__ static double st_v(double x, uint32_t) { return x; }
    __device__ __forceinline__ static double ld(double x) { return x; }
    __device__ __forceinline__ static double st(double x) { return x; }
    __device__ __forceinline__ static double round(double x) { return x; }
};

}  // namespace potts
