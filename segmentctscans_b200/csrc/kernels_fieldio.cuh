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
__device__ __forceinline__ uint32_t stream_word(const uint32_t *__restrict__ w, int64_t i)
{
    return __byte_perm(__ldcs(w + i), 0u, 0x0123u);
}

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
// the padding n >= ns is not written.
template <int kBits>
__global__ void __launch_bounds__(kIoThreads) archive_unpack_kernel(IoLines g, const uint32_t *__restrict__ words,
                                                                     int shift,
                                                                     typename IoElem<kBits>::T *__restrict__ out)
{
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const int64_t i0 = L * g.ns;
        typename IoElem<kBits>::T *dst = out + L * g.nstride;
#pragma unroll 4
        for (int n = threadIdx.x; n < g.ns; n += kIoThreads) dst[n] = unpack_unit<kBits>(words, i0 + n, shift);
    }
}

// Byte order of a stream unit in memory (most significant byte first).
__device__ __forceinline__ uint32_t to_stream_order(uint32_t v) { return __byte_perm(v, 0u, 0x0123u); }
__device__ __forceinline__ uint16_t to_stream_order(uint16_t v) { return (uint16_t)((v << 8) | (v >> 8)); }

// Field -> payload (Field<T>::save, include/field.h:92-119): unit i of the staged output holds the
// low `shift` bits of voxel i - 1 and the high kBits - shift bits of voxel i (voxel -1 is 0: those
// bits belong to the header, which the host merges into byte 0).  With shift > 0 one more unit
// carries the low bits of the last voxel.
template <int kBits>
__global__ void __launch_bounds__(kIoThreads) archive_pack_kernel(IoLines g,
                                                                   const typename IoElem<kBits>::T *__restrict__ in,
                                                                   int shift,
                                                                   typename IoElem<kBits>::T *__restrict__ out)
{
    using T = typename IoElem<kBits>::T;
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const int64_t i0 = L * g.ns;
        const T *src = in + L * g.nstride;
        // the voxel before the line's first one: the last voxel of the previous line
        const T before = L > 0 ? in[(L - 1) * g.nstride + g.ns - 1] : (T)0;
#pragma unroll 4
        for (int n = threadIdx.x; n < g.ns; n += kIoThreads) {
            const uint32_t v = src[n];
            const uint32_t p = n > 0 ? (uint32_t)src[n - 1] : (uint32_t)before;
            const uint32_t u = shift ? ((v >> shift) | (p << (kBits - shift))) : v;
            out[i0 + n] = to_stream_order((T)u);
        }
    }
    if (shift && blockIdx.x == 0 && threadIdx.x == 0 && g.n_lines > 0) {
        const uint32_t last = in[(g.n_lines - 1) * g.nstride + g.ns - 1];
        out[g.n_lines * g.ns] = to_stream_order((T)(last << (kBits - shift)));
    }
}

// convert_to_fp_kernel (transpose/convert_to_fp.cpp:11-47): 0 at or below lo, 1 at or above hi,
// else (v - lo) / (hi - lo) in single precision.
template <typename T>
__global__ void __launch_bounds__(kIoThreads) convert_to_fp_kernel(IoLines g, const T *__restrict__ in, float lo,
                                                                    float hi, float *__restrict__ out)
{
    const float range = __fsub_rn(hi, lo);
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const T *src = in + L * g.nstride;
        float *dst = out + L * g.nstride;
#pragma unroll 4
        for (int n = threadIdx.x; n < g.ns; n += kIoThreads) {
            const float v = (float)__ldcs(src + n);
            float r;
            if (v <= lo)
                r = 0.0f;
            else if (v >= hi)
                r = 1.0f;
            else
                r = __fdiv_rn(__fsub_rn(v, lo), range);
            __stcs(dst + n, r);
        }
    }
}

// histogram_kernel + histogram_reduce_kernel (transpose/find_intensity_range.cpp:22-62): the
// 65536-bin histogram of a uint16 field.  The counters live in the distributed shared memory of
// a two-block cluster (block rank k owns bins [32768 k, 32768 (k + 1)), 128 KB each); lanes of a
// warp holding the same value add once; each cluster flushes its non-zero bins to the 64-bit
// global counts.
constexpr int kU16Cluster = 2;
constexpr int kU16Slice = 32768;

__global__ void __cluster_dims__(kU16Cluster, 1, 1) __launch_bounds__(kIoThreads, 1)
    u16_hist_cluster_kernel(IoLines g, const uint16_t *__restrict__ f, unsigned long long *__restrict__ ghist)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ uint32_t sh_u16[];
    for (int i = threadIdx.x; i < kU16Slice; i += blockDim.x) sh_u16[i] = 0u;
    cluster.sync();
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const uint16_t *line = f + L * g.nstride;
        for (int n0 = 0; n0 < g.ns; n0 += blockDim.x) {  // whole warps, for the lane combining
            const int n = n0 + threadIdx.x;
            const int id = n < g.ns ? (int)__ldcs(line + n) : -1;
            warp_count(id, [&](int b, uint32_t c) {
                uint32_t *dst = cluster.map_shared_rank(sh_u16, (unsigned)(b / kU16Slice));
                atomicAdd(dst + (b % kU16Slice), c);
            });
        }
    }
    cluster.sync();
    const int base = (int)cluster.block_rank() * kU16Slice;
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

__global__ void __launch_bounds__(kIoThreads) raw_box_kernel(BoxGeom g, const float *__restrict__ f,
                                                              uint8_t *__restrict__ out)
{
    for (int64_t b = blockIdx.x; b < g.box_lines; b += gridDim.x) {
        const uint32_t col = g.col_begin + (uint32_t)(b / g.row_size);
        const int64_t row = (int64_t)g.row_begin + (b % g.row_size);
        const int64_t sr = g.start_row[col];
        const int64_t cnt = (int64_t)(g.base[col + 1] - g.base[col]) / g.nstride;
        uint8_t *dst = out + b * g.ns;
        if (cnt > 0 && row >= sr && row < sr + cnt) {
            const float *src = f + (int64_t)g.base[col] + (row - sr) * g.nstride;
#pragma unroll 4
            for (int n = threadIdx.x; n < g.ns; n += kIoThreads) dst[n] = label_byte(__ldcs(src + n));
        } else {
            for (int n = threadIdx.x; n < g.ns; n += kIoThreads) dst[n] = 255;
        }
    }
}

}  // namespace potts
