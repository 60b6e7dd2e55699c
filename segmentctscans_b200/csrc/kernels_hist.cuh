// Label-finding inputs: the GPU steps that run before the Potts solve on the
// same cylinder layout.
//   min_max          min_max/min_max.cpp:18-54 (in-mask min and max)
//   grad_min_max     uv-hist/uv-hist-kernel.cpp:29-68 (min and max of the strictly positive values)
//   grad_magn        grad-magn/grad_magn.cpp:17-58 (central-difference gradient magnitude)
//   calc_hist        calc_hist/calc_hist.cpp:23-80 (1-D histogram, optional jitter)
//   uv_hist          uv-hist/uv-hist-kernel.cpp:100-197 (2-D histogram of (u, grad magnitude))
// Fields are laid out like the mapping: line L (a stored (row, col) pair) holds
// slices n in [0, n_images) at L * nstride + n.  Every kernel reads each field
// value once (HBM-bound); the reductions end in per-block partial results or
// privatised histograms, so no two runs differ.
#pragma once

#include <cooperative_groups.h>

#include <cstdint>

#include "geometry.cuh"

namespace potts {

constexpr int kHistThreads = 256;

// ---------------------------------------------------------------------------
// min / max
// ---------------------------------------------------------------------------
// Per block: min and max over the in-mask values (only those > 0 when kPositive), one warp per
// line (lines blockIdx.x * 8 + warp, then every gridDim.x * 8); FLT_MAX / -FLT_MAX when the block
// saw none.  kVec: 16-byte loads (lines of a multiple of 4 values and stride, aligned field).
template <bool kPositive, bool kVec>
__global__ void __launch_bounds__(kHistThreads) minmax_partial_kernel(Geometry g, const float *__restrict__ f,
                                                                      float2 *__restrict__ partial)
{
    float lo = 3.402823466e38f, hi = -3.402823466e38f;
    auto see = [&](float x) {
        if (!kPositive || x > 0.0f) {
            lo = fminf(lo, x);
            hi = fmaxf(hi, x);
        }
    };
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (kHistThreads / 32);
    for (int64_t L = (int64_t)blockIdx.x * (kHistThreads / 32) + (threadIdx.x >> 5); L < g.n_lines; L += warps) {
        const float *line = f + L * g.nstride_w;
        if constexpr (kVec) {
#pragma unroll 4
            for (int q = lane; q < g.ns / 4; q += 32) {
                const float4 v = __ldg(reinterpret_cast<const float4 *>(line) + q);
                see(v.x);
                see(v.y);
                see(v.z);
                see(v.w);
            }
        } else {
            for (int n = lane; n < g.ns; n += 32) see(__ldg(line + n));
        }
    }
    __shared__ float slo[kHistThreads / 32], shi[kHistThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        slo[w] = lo;
        shi[w] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < kHistThreads / 32; ++i) {
            lo = fminf(lo, slo[i]);
            hi = fmaxf(hi, shi[i]);
        }
        partial[blockIdx.x] = make_float2(lo, hi);
    }
}

// One block folds the per-block results into out[0] = min, out[1] = max.
__global__ void __launch_bounds__(kHistThreads) minmax_final_kernel(const float2 *__restrict__ partial, int n,
                                                                    float *__restrict__ out)
{
    float lo = 3.402823466e38f, hi = -3.402823466e38f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float2 p = partial[i];
        lo = fminf(lo, p.x);
        hi = fmaxf(hi, p.y);
    }
    __shared__ float slo[kHistThreads / 32], shi[kHistThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        slo[w] = lo;
        shi[w] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < kHistThreads / 32; ++i) {
            lo = fminf(lo, slo[i]);
            hi = fmaxf(hi, shi[i]);
        }
        out[0] = lo;
        out[1] = hi;
    }
}

// ---------------------------------------------------------------------------
// Gradient magnitude (grad_magn.cpp:27-55): v = 0.5 sqrt(q_n^2 + q_r^2 + q_c^2) with central
// differences q = u(x + e) - u(x - e), each accumulated from 0 as the reference does; -1 where
// any of the six neighbours is outside the mask.  The sum of squares is contracted as the
// reference's clang build contracts it (one rounded square, then two multiply-adds), like the
// other stencils of the library.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kHistThreads) grad_magn_kernel(Geometry g, const float *__restrict__ u,
                                                                 float *__restrict__ v)
{
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const LineInfo li = load_line(g, L);
        const bool inner = (li.flags & kHasNextRow) && (li.flags & kHasPrevRow) && li.next_col >= 0 &&
                           li.prev_col >= 0;
        const int64_t o0 = L * g.nstride_w;
        for (int n = threadIdx.x; n < g.ns; n += blockDim.x) {
            const int64_t o = o0 + n;
            float r = -1.0f;
            if (inner && n > 0 && n + 1 < g.ns) {
                float q1 = 0.0f, q2 = 0.0f, q3 = 0.0f;
                q1 += u[o + 1];
                q2 += u[o + g.nstride_w];
                q3 += u[(int64_t)li.next_col * g.nstride_w + n];
                q1 -= u[o - 1];
                q2 -= u[o - g.nstride_w];
                q3 -= u[(int64_t)li.prev_col * g.nstride_w + n];
                float s = q1 * q1;
                s = fmaf(q2, q2, s);
                s = fmaf(q3, q3, s);
                r = 0.5f * __fsqrt_rn(s);
            }
            v[o] = r;
        }
    }
}

// ---------------------------------------------------------------------------
// Histogram bins (calc_hist.cpp:62-66, uv-hist-kernel.cpp:139-149): t = (x - start) / (end -
// start), bin = round(nb t - 0.5) (the multiply-add contracted as the reference's clang build
// does), clamped to [0, nb - 1]; a NaN quotient (start == end) gives bin 0, as the GPU's
// float-to-int conversion does in the reference.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int hist_bin(float x, float start, float end, int nb)
{
    const float t = __fdiv_rn(x - start, end - start);
    const float r = roundf(fmaf((float)nb, t, -0.5f));
    if (!(r >= 0.0f)) return 0;
    if (r >= (float)(nb - 1)) return nb - 1;
    return (int)r;
}

// Jitter of voxel `idx` (in-mask index L * n_images + n) for calc_hist's smoothing: uniform in
// [-delta/2, delta/2) from SplitMix64 (Steele, Lea and Flood, 2014; public domain) of
// (seed, idx).  The reference draws from a randomly seeded Philox stream, so its jittered
// histograms differ from run to run; this one is reproducible for a given seed.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ float hist_jitter(uint64_t seed, uint64_t idx, float delta)
{
    const float u01 = (float)(uint32_t)(splitmix64(seed ^ (idx * 0xd1342543de82ef95ull)) >> 40) * 0x1p-24f;
    return __fadd_rn(-0.5f * delta, __fmul_rn(delta, u01));
}

// Adds 1 to counter `id` (>= 0) for every lane whose id it is, one atomic per distinct id of the
// warp (lanes of a line often share a bin).  add(ptr_of(id), count) does the atomic.
template <typename Add>
__device__ __forceinline__ void warp_count(int id, Add add)
{
    const unsigned active = __ballot_sync(0xffffffffu, id >= 0);
    if (id < 0) return;
    const unsigned same = __match_any_sync(active, id);
    if ((threadIdx.x & 31) == __ffs(same) - 1) add(id, (uint32_t)__popc(same));
}

// 1-D histogram (calc_hist.cpp:23-80) into a shared-memory copy per block, flushed with one
// global atomic per non-zero bin.  nb * 4 bytes of dynamic shared memory.
template <bool kJitter>
__global__ void __launch_bounds__(kHistThreads) hist1d_kernel(Geometry g, const float *__restrict__ f, float rs,
                                                              float re, int nb, float delta, uint64_t seed,
                                                              uint32_t *__restrict__ ghist)
{
    extern __shared__ uint32_t sh_hist[];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) sh_hist[i] = 0u;
    __syncthreads();
    const float hd = delta * 0.5f;  // delta / 2, exact
    const float lo = rs - hd;
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const float *line = f + L * g.nstride_w;
        // whole warps walk the line so that the warp-level combining sees full warps
        for (int n0 = 0; n0 < g.ns; n0 += blockDim.x) {
            const int n = n0 + threadIdx.x;
            int id = -1;
            if (n < g.ns) {
                float x = __ldg(line + n);
                if (kJitter) x = __fadd_rn(x, hist_jitter(seed, (uint64_t)L * g.ns + n, delta));
                if (lo <= x && __fadd_rn(x, hd) <= re) id = hist_bin(x, rs, re, nb);
            }
            warp_count(id, [&](int b, uint32_t c) { atomicAdd(sh_hist + b, c); });
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        if (sh_hist[i]) atomicAdd(ghist + i, sh_hist[i]);
}

// The same with global atomics only (bin counts too large for shared memory).
template <bool kJitter>
__global__ void __launch_bounds__(kHistThreads) hist1d_global_kernel(Geometry g, const float *__restrict__ f,
                                                                     float rs, float re, int nb, float delta,
                                                                     uint64_t seed, uint32_t *__restrict__ ghist)
{
    const float hd = delta * 0.5f;
    const float lo = rs - hd;
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const float *line = f + L * g.nstride_w;
        for (int n0 = 0; n0 < g.ns; n0 += blockDim.x) {
            const int n = n0 + threadIdx.x;
            int id = -1;
            if (n < g.ns) {
                float x = __ldg(line + n);
                if (kJitter) x = __fadd_rn(x, hist_jitter(seed, (uint64_t)L * g.ns + n, delta));
                if (lo <= x && __fadd_rn(x, hd) <= re) id = hist_bin(x, rs, re, nb);
            }
            warp_count(id, [&](int b, uint32_t c) { atomicAdd(ghist + b, c); });
        }
    }
}

// Bin of the pair (x = u, y = grad magnitude) in the 2-D histogram (uv-hist-kernel.cpp:133-150):
// ybin * stride + xbin, or -1 outside [u_start, u_end] x [v_start, v_end].
struct UvRange {
    float us, ue, vs, ve;
    int nb, stride;
};
__device__ __forceinline__ int uv_bin(float x, float y, const UvRange &r)
{
    if (!(r.us <= x && x <= r.ue && r.vs <= y && y <= r.ve)) return -1;
    return hist_bin(y, r.vs, r.ve, r.nb) * r.stride + hist_bin(x, r.us, r.ue, r.nb);
}

// 2-D histogram held in the distributed shared memory of a cluster of kUvCluster blocks:
// block rank k of the cluster owns bins [k kUvSlice, (k+1) kUvSlice), and every block of the
// cluster adds into whichever block owns a bin.  Each cluster flushes its non-zero bins to the
// global histogram once.  1 MB of 32-bit counters: 512 x 512 bins fit.
constexpr int kUvCluster = 8;
constexpr int kUvSlice = 32768;   // counters per block (128 KB)
constexpr int kUvThreads = 1024;  // one block per multiprocessor: as many warps as it holds

__global__ void __cluster_dims__(kUvCluster, 1, 1) __launch_bounds__(kUvThreads, 1)
    uv_hist_cluster_kernel(Geometry g, const float *__restrict__ u, const float *__restrict__ v, UvRange r,
                           int total_bins, uint32_t *__restrict__ ghist)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ uint32_t sh_uv[];
    for (int i = threadIdx.x; i < kUvSlice; i += blockDim.x) sh_uv[i] = 0u;
    cluster.sync();
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const int64_t o0 = L * g.nstride_w;
        for (int n0 = 0; n0 < g.ns; n0 += blockDim.x) {
            const int n = n0 + threadIdx.x;
            int id = -1;
            if (n < g.ns) id = uv_bin(__ldg(u + o0 + n), __ldg(v + o0 + n), r);
            warp_count(id, [&](int b, uint32_t c) {
                uint32_t *dst = cluster.map_shared_rank(sh_uv, (unsigned)(b / kUvSlice));
                atomicAdd(dst + (b % kUvSlice), c);
            });
        }
    }
    cluster.sync();
    const int base = (int)cluster.block_rank() * kUvSlice;
    for (int i = threadIdx.x; i < kUvSlice && base + i < total_bins; i += blockDim.x)
        if (sh_uv[i]) atomicAdd(ghist + base + i, sh_uv[i]);
}

// The same with global atomics only (histograms larger than a cluster's shared memory).
__global__ void __launch_bounds__(kHistThreads) uv_hist_global_kernel(Geometry g, const float *__restrict__ u,
                                                                      const float *__restrict__ v, UvRange r,
                                                                      uint32_t *__restrict__ ghist)
{
    for (int64_t L = blockIdx.x; L < g.n_lines; L += gridDim.x) {
        const int64_t o0 = L * g.nstride_w;
        for (int n0 = 0; n0 < g.ns; n0 += blockDim.x) {
            const int n = n0 + threadIdx.x;
            int id = -1;
            if (n < g.ns) id = uv_bin(__ldg(u + o0 + n), __ldg(v + o0 + n), r);
            warp_count(id, [&](int b, uint32_t c) { atomicAdd(ghist + b, c); });
        }
    }
}

}  // namespace potts
