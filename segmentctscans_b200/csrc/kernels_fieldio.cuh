// Field I/O and the steps on either side of the Potts solve, on the cylinder layout:
//   archive payload      Field<T>::save / load (include/field.h:92-150): the in-mask voxels in
//                        column -> row -> n order, each one element-wide field of an MSB-first
//                        bit stream (include/io/outbitstream.h, include/io/inbitstream.h)
//   convert_to_fp        transpose/convert_to_fp.cpp:11-47 (clamp and scale to [0, 1])
//   intensity histogram  transpose/find_intensity_range.cpp:22-62 (65536 bins of uint16 voxels)
//   raw label box        potts-model/potts-model.cpp:184-241 (uint8 box of round(255 v), 255 outside)
//
// The archive's voxel order is the storage order of the lines (columns ascending, rows of a
// column consecutively), so archive voxel i = L * n_images + n is voxel n of line L, stored at
// L * nstride + n.  The payload starts `shift` (0..7) bits into a byte, after the header; the
// kernels see it as 32-bit words staged from that byte on, so that voxel i of a 32-bit archive
// is the word pair (i, i + 1) shifted left by `shift`, and unit i of a 16-bit archive sits in
// the 64-bit window of words (i / 2, i / 2 + 1) at bit 16 (i & 1) + shift.  Every kernel reads
// each voxel once and writes it once (HBM-bound byte work).
#pragma once

#include <cooperative_groups.h>

#include <cstdint>

#include "geometry.cuh"
#include "kernels_hist.cuh"

namespace potts {

constexpr int kIoThreads = 256;

template <int kBits>
struct IoElem;
template <>
struct IoElem<32> {
    using T = uint32_t;  // FP32 bit patterns
};
template <>
struct IoElem<16> {
    using T = uint16_t;
};

// Plain description of a field's lines: line L holds n in [0, ns) at L * nstride + n.
struct IoLines {
    int64_t n_lines;
    int ns;
    int nstride;
};

// Word w of the staged payload in stream order (the bytes were loaded little-endian).
__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0u, 0x0123u); }
__device__ __forceinline__ uint32_t stream_word(const uint32_t *__restrict__ w, int64_t i) { return bswap32(__ldg(w + i)); }

// The stream unit that starts `shift` bits into staged unit i (i counts kBits-wide units).
template <int kBits>
__device__ __forceinline__ typename IoElem<kBits>::T unpack_unit(const uint32_t *__restrict__ words, int64_t i,
                                                                  int shift)
{
    if constexpr (kBits == 32) {
        return __funnelshift_l(stream_word(words, i + 1), stream_word(words, i), (unsigned)shift);
    } else {
        const int64_t w = i >> 1;
        const uint64_t win = ((uint64_t)stream_word(words, w) << 32) | stream_word(words, w + 1);
        return (uint16_t)((win << (16 * (int)(i & 1) + shift)) >> 48);
    }
}

// Payload -> field (Field<T>::load, include/field.h:121-147): every in-mask voxel of every line;
// the padding n >= ns is not written.  kVec: each thread turns 16 staged bytes (one uint4 load plus
// the next word) into 16 output bytes (4 FP32 voxels or 8 uint16 voxels); needs lines whose voxel
// count and stride are multiples of 16 bytes' worth and a 16-byte aligned field.
template <int kBits, bool kVec>
__global__ void __launch_bounds__(kIoThreads) archive_unpack_kernel(IoLines g, const uint32_t *__restrict__ words,
                                                                     int shift,
                                                                     typename IoElem<kBits>::T *__restrict__ out)
{
    constexpr int kPer = 128 / kBits;  // voxels per 16 bytes
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const int64_t i0 = L * g.ns;
        typename IoElem<kBits>::T *dst = out + L * g.nstride;
        if constexpr (kVec) {
            const uint32_t *wl = words + i0 * kBits / 32;  // 16-byte aligned: i0 is a multiple of kPer
            for (int q = threadIdx.x; q < g.ns / kPer; q += kIoThreads) {
                const uint4 a = __ldg(reinterpret_cast<const uint4 *>(wl) + q);
                const uint32_t w0 = bswap32(a.x), w1 = bswap32(a.y), w2 = bswap32(a.z), w3 = bswap32(a.w);
                const uint32_t w4 = bswap32(__ldg(wl + 4 * q + 4));
                const unsigned sh = (unsigned)shift;
                uint4 r;
                if constexpr (kBits == 32) {
                    r = make_uint4(__funnelshift_l(w1, w0, sh), __funnelshift_l(w2, w1, sh), __funnelshift_l(w3, w2, sh),
                                   __funnelshift_l(w4, w3, sh));
                } else {
                    // 16-bit units: the shifted words hold units (2k, 2k+1) as (high, low) halves
                    const uint32_t s0 = __funnelshift_l(w1, w0, sh), s1 = __funnelshift_l(w2, w1, sh),
                                   s2 = __funnelshift_l(w3, w2, sh), s3 = __funnelshift_l(w4, w3, sh);
                    r = make_uint4(__byte_perm(s0, 0u, 0x1032u), __byte_perm(s1, 0u, 0x1032u),
                                   __byte_perm(s2, 0u, 0x1032u), __byte_perm(s3, 0u, 0x1032u));
                }
                reinterpret_cast<uint4 *>(dst)[q] = r;
            }
        } else {
#pragma unroll 4
            for (int n = threadIdx.x; n < g.ns; n += kIoThreads) dst[n] = unpack_unit<kBits>(words, i0 + n, shift);
        }
    }
}

// Byte order of a stream unit in memory (most significant byte first).
__device__ __forceinline__ uint32_t to_stream_order(uint32_t v) { return __byte_perm(v, 0u, 0x0123u); }
__device__ __forceinline__ uint16_t to_stream_order(uint16_t v) { return (uint16_t)((v << 8) | (v >> 8)); }

// Field -> payload (Field<T>::save, include/field.h:92-119): unit i of the staged output holds the
// low `shift` bits of voxel i - 1 and the high kBits - shift bits of voxel i (voxel -1 is 0: those
// bits belong to the header, which the host merges into byte 0).  With shift > 0 one more unit
// carries the low bits of the last voxel.
// kVec (FP32 only): 4 voxels per thread, one 16-byte load and one 16-byte store (lines of a
// multiple of 4 voxels, 16-byte aligned field).
template <int kBits, bool kVec>
__global__ void __launch_bounds__(kIoThreads) archive_pack_kernel(IoLines g,
                                                                   const typename IoElem<kBits>::T *__restrict__ in,
                                                                   int shift,
                                                                   typename IoElem<kBits>::T *__restrict__ out)
{
    using T = typename IoElem<kBits>::T;
    static_assert(!kVec || kBits == 32, "vector packing of FP32 archives");
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const int64_t i0 = L * g.ns;
        const T *src = in + L * g.nstride;
        // the voxel before the line's first one: the last voxel of the previous line
        const T before = L > 0 ? in[(L - 1) * g.nstride + g.ns - 1] : (T)0;
        if constexpr (kVec) {
            const unsigned sh = (unsigned)shift;
            for (int q = threadIdx.x; q < g.ns / 4; q += kIoThreads) {
                const uint4 v = __ldg(reinterpret_cast<const uint4 *>(src) + q);
                const uint32_t p = q > 0 ? __ldg(src + 4 * q - 1) : (uint32_t)before;
                // unit k = low `shift` bits of voxel k-1, then the high bits of voxel k
                const uint4 u = make_uint4(__funnelshift_r(v.x, p, sh), __funnelshift_r(v.y, v.x, sh),
                                           __funnelshift_r(v.z, v.y, sh), __funnelshift_r(v.w, v.z, sh));
                reinterpret_cast<uint4 *>(out + i0)[q] =
                    make_uint4(bswap32(u.x), bswap32(u.y), bswap32(u.z), bswap32(u.w));
            }
        } else {
#pragma unroll 4
            for (int n = threadIdx.x; n < g.ns; n += kIoThreads) {
                const uint32_t v = src[n];
                const uint32_t p = n > 0 ? (uint32_t)src[n - 1] : (uint32_t)before;
                const uint32_t u = shift ? ((v >> shift) | (p << (kBits - shift))) : v;
                out[i0 + n] = to_stream_order((T)u);
            }
        }
    }
    if (shift && blockIdx.x == 0 && threadIdx.x == 0 && g.n_lines > 0) {
        const uint32_t last = in[(g.n_lines - 1) * g.nstride + g.ns - 1];
        out[g.n_lines * g.ns] = to_stream_order((T)(last << (kBits - shift)));
    }
}

// convert_to_fp_kernel (transpose/convert_to_fp.cpp:11-47): 0 at or below lo, 1 at or above hi,
// else (v - lo) / (hi - lo) in single precision.
__device__ __forceinline__ float to_unit(float v, float lo, float hi, float range)
{
    if (v <= lo) return 0.0f;
    if (v >= hi) return 1.0f;
    return __fdiv_rn(__fsub_rn(v, lo), range);
}

// One block per line.  At 768^2 x 1024 (uint16 in, FP32 out: 2 B read, 4 B written per voxel)
// this measured faster than one warp per line, than a flat range of 8-voxel items, and than a
// table of the 65536 uint16 results in place of the division: the write-heavy stream, not the
// arithmetic, is the limit.  kVec: 4 voxels per thread (lines of a multiple of 4
// voxels, 16-byte aligned fields).
template <typename T, bool kVec>
__global__ void __launch_bounds__(kIoThreads) convert_to_fp_kernel(IoLines g, const T *__restrict__ in, float lo,
                                                                    float hi, float *__restrict__ out)
{
    const float range = __fsub_rn(hi, lo);
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const T *src = in + L * g.nstride;
        float *dst = out + L * g.nstride;
        if constexpr (kVec) {
            for (int q = threadIdx.x; q < g.ns / 4; q += kIoThreads) {
                float4 v;
                if constexpr (sizeof(T) == 2) {
                    const uint2 p = __ldg(reinterpret_cast<const uint2 *>(src) + q);
                    v = make_float4((float)(p.x & 0xffffu), (float)(p.x >> 16), (float)(p.y & 0xffffu),
                                    (float)(p.y >> 16));
                } else {
                    v = __ldg(reinterpret_cast<const float4 *>(src) + q);
                }
                reinterpret_cast<float4 *>(dst)[q] = make_float4(to_unit(v.x, lo, hi, range), to_unit(v.y, lo, hi, range),
                                                                 to_unit(v.z, lo, hi, range), to_unit(v.w, lo, hi, range));
            }
        } else {
#pragma unroll 4
            for (int n = threadIdx.x; n < g.ns; n += kIoThreads) dst[n] = to_unit((float)__ldg(src + n), lo, hi, range);
        }
    }
}

// histogram_kernel + histogram_reduce_kernel (transpose/find_intensity_range.cpp:22-62): the
// 65536-bin histogram of a uint16 field.  A two-block cluster reads the same lines; block rank k
// counts the values whose top bit is k into its own 32768 shared-memory counters (128 KB), so every
// value is counted once, with a shared-memory atomic, and the second read of a line is served by L2.
// One block of 1024 threads per multiprocessor, one warp per line; each block flushes its non-zero
// bins to the 64-bit global counts.  kVec: 8 values per lane and step (16-byte loads).
constexpr int kU16Cluster = 2;
constexpr int kU16Slice = 32768;
constexpr int kU16Threads = 1024;

template <bool kVec>
__global__ void __cluster_dims__(kU16Cluster, 1, 1) __launch_bounds__(kU16Threads, 1)
    u16_hist_cluster_kernel(IoLines g, const uint16_t *__restrict__ f, unsigned long long *__restrict__ ghist)
{
    namespace cg = cooperative_groups;
    extern __shared__ uint32_t sh_u16[];
    for (int i = threadIdx.x; i < kU16Slice; i += blockDim.x) sh_u16[i] = 0u;
    __syncthreads();
    const uint32_t half = cg::this_cluster().block_rank();
    constexpr int kWarps = kU16Threads / 32;
    const int lane = threadIdx.x & 31;
    const int64_t pairs = gridDim.x / kU16Cluster;
    auto count = [&](uint32_t v) {
        if ((v >> 15) == half) atomicAdd(sh_u16 + (v & 0x7fffu), 1u);
    };
    for (int64_t L = (blockIdx.x / kU16Cluster) * kWarps + (threadIdx.x >> 5); L < g.n_lines; L += pairs * kWarps) {
        const uint16_t *line = f + L * g.nstride;
        if constexpr (kVec) {
#pragma unroll 4
            for (int q = lane; q < g.ns / 8; q += 32) {
                const uint4 p = __ldg(reinterpret_cast<const uint4 *>(line) + q);
                count(p.x & 0xffffu);
                count(p.x >> 16);
                count(p.y & 0xffffu);
                count(p.y >> 16);
                count(p.z & 0xffffu);
                count(p.z >> 16);
                count(p.w & 0xffffu);
                count(p.w >> 16);
            }
        } else {
            for (int n = lane; n < g.ns; n += 32) count(__ldg(line + n));
        }
    }
    __syncthreads();
    const int base = (int)half * kU16Slice;
    for (int i = threadIdx.x; i < kU16Slice; i += blockDim.x)
        if (sh_u16[i]) atomicAdd(ghist + base + i, (unsigned long long)sh_u16[i]);
}

// The raw label box of potts-model.cpp:184-241: box line b = c * row_size + r (column c + col_begin,
// row r + row_begin) holds n_images bytes, min(255, max(0, round(255 v))) inside the mask and
// 255 outside.
struct BoxGeom {
    const uint32_t *start_row;  // [cols]
    const uint32_t *base;       // [cols + 1]
    uint32_t col_begin, row_begin;
    int row_size;
    int64_t box_lines;  // col_size * row_size
    int ns, nstride;
};

__device__ __forceinline__ uint8_t label_byte(float v)
{
    const float s = roundf(__fmul_rn(255.0f, v));  // std::round(255 * v): halves away from zero
    return (uint8_t)(s >= 255.0f ? 255 : (s <= 0.0f ? 0 : (int)s));
}

// One warp per box line.  kVec: 4 voxels per lane and step (a float4 in, 4 bytes out): slices a
// multiple of 4, aligned buffers.  Box lines are fewer than 2^32 (rows and columns are below 2^16).
template <bool kVec>
__global__ void __launch_bounds__(kIoThreads) raw_box_kernel(BoxGeom g, const float *__restrict__ f,
                                                              uint8_t *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (kIoThreads / 32);
    for (int64_t b = (int64_t)blockIdx.x * (kIoThreads / 32) + (threadIdx.x >> 5); b < g.box_lines; b += warps) {
        const uint32_t bl = (uint32_t)b;
        const uint32_t col = g.col_begin + bl / (uint32_t)g.row_size;
        const int64_t row = (int64_t)g.row_begin + bl % (uint32_t)g.row_size;
        const int64_t sr = __ldg(g.start_row + col);
        const uint32_t b0 = __ldg(g.base + col), b1 = __ldg(g.base + col + 1);
        const int64_t cnt = (int64_t)(b1 - b0) / g.nstride;
        uint8_t *dst = out + b * g.ns;
        const bool inside = cnt > 0 && row >= sr && row < sr + cnt;
        const float *src = inside ? f + (int64_t)b0 + (row - sr) * g.nstride : f;
        if constexpr (kVec) {
#pragma unroll 8
            for (int q = lane; q < g.ns / 4; q += 32) {
                uint32_t r = 0xffffffffu;
                if (inside) {
                    const float4 v = __ldg(reinterpret_cast<const float4 *>(src) + q);
                    r = (uint32_t)label_byte(v.x) | ((uint32_t)label_byte(v.y) << 8) |
                        ((uint32_t)label_byte(v.z) << 16) | ((uint32_t)label_byte(v.w) << 24);
                }
                reinterpret_cast<uint32_t *>(dst)[q] = r;
            }
        } else if (inside) {
#pragma unroll 4
            for (int n = lane; n < g.ns; n += 32) dst[n] = label_byte(__ldg(src + n));
        } else {
            for (int n = lane; n < g.ns; n += 32) dst[n] = 255;
        }
    }
}

}  // namespace potts
