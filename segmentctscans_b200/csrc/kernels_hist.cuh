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

#include <cstdint>

#include "geometry.cuh"
#include "tma.cuh"

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

// Block-wide fold of (min, max, min, max) into thread 0's a.
__device__ __forceinline__ void fold_minmax4(float4 &a)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a.x = fminf(a.x, __shfl_xor_sync(0xffffffffu, a.x, o));
        a.y = fmaxf(a.y, __shfl_xor_sync(0xffffffffu, a.y, o));
        a.z = fminf(a.z, __shfl_xor_sync(0xffffffffu, a.z, o));
        a.w = fmaxf(a.w, __shfl_xor_sync(0xffffffffu, a.w, o));
    }
    __shared__ float4 sw[kHistThreads / 32];
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 1; i < kHistThreads / 32; ++i) {
            a.x = fminf(a.x, sw[i].x);
            a.y = fmaxf(a.y, sw[i].y);
            a.z = fminf(a.z, sw[i].z);
            a.w = fmaxf(a.w, sw[i].w);
        }
}

// The ranges of the 2-D histogram in one pass over both fields (uv-hist-kernel.cpp:70-98): per
// block (min u, max u, min v, max v) over every u and the strictly positive v; kVec: 16-byte
// loads of both.  minmax_pair_final_kernel folds the blocks into out[0..3].
template <bool kVec>
__global__ void __launch_bounds__(kHistThreads) minmax_pair_partial_kernel(Geometry g, const float *__restrict__ u,
                                                                           const float *__restrict__ v,
                                                                           float4 *__restrict__ partial)
{
    float4 a = make_float4(3.402823466e38f, -3.402823466e38f, 3.402823466e38f, -3.402823466e38f);
    auto see = [&](float x, float y) {
        a.x = fminf(a.x, x);
        a.y = fmaxf(a.y, x);
        if (y > 0.0f) {
            a.z = fminf(a.z, y);
            a.w = fmaxf(a.w, y);
        }
    };
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (kHistThreads / 32);
    for (int64_t L = (int64_t)blockIdx.x * (kHistThreads / 32) + (threadIdx.x >> 5); L < g.n_lines; L += warps) {
        const float *lu = u + L * g.nstride_w, *lv = v + L * g.nstride_w;
        if constexpr (kVec) {
#pragma unroll 2
            for (int q = lane; q < g.ns / 4; q += 32) {
                const float4 x = __ldg(reinterpret_cast<const float4 *>(lu) + q);
                const float4 y = __ldg(reinterpret_cast<const float4 *>(lv) + q);
                see(x.x, y.x);
                see(x.y, y.y);
                see(x.z, y.z);
                see(x.w, y.w);
            }
        } else {
            for (int n = lane; n < g.ns; n += 32) see(__ldg(lu + n), __ldg(lv + n));
        }
    }
    fold_minmax4(a);
    if (threadIdx.x == 0) partial[blockIdx.x] = a;
}

__global__ void __launch_bounds__(kHistThreads) minmax_pair_final_kernel(const float4 *__restrict__ partial, int n,
                                                                         float *__restrict__ out)
{
    float4 a = make_float4(3.402823466e38f, -3.402823466e38f, 3.402823466e38f, -3.402823466e38f);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 p = partial[i];
        a.x = fminf(a.x, p.x);
        a.y = fmaxf(a.y, p.y);
        a.z = fminf(a.z, p.z);
        a.w = fmaxf(a.w, p.w);
    }
    fold_minmax4(a);
    if (threadIdx.x == 0) {
        out[0] = a.x;
        out[1] = a.y;
        out[2] = a.z;
        out[3] = a.w;
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

// Gradient magnitude as a column march (fields of 16-byte lines, 16-byte line stride): a block owns
// GmTile::TR rows x GmTile::TN slices of a work item's columns [ca, cb) (the work items of the
// Potts kernel: x = first row, y = first slice, z/w = column range) and walks along the columns
// with a ring of SLOTS column planes of u in shared memory (rows r0-1 .. r0+TR, slices n0-4 ..
// n0+TN+3: one TMA box, issued SLOTS-3 planes ahead of the plane after the one being computed).
// Every u value then comes from DRAM once per tile and its six neighbours from shared memory, with
// several planes in flight per block.  Thread t takes the slices n0+4(t%32) .. +3 of rows t/32
// and t/32+8.  The operations per voxel are grad_magn_kernel's, so the bits are the same.  Box
// rows outside a plane's column belong to other columns (or are zero fill) and are never used:
// the column table decides every neighbour.  Every wait is bounded; a block whose wait gives up
// sets *err, drains its loads in flight (bounded) and stops.
struct GmTile {
    static constexpr int TR = 16, TN = 128, XR = TR + 2, XS = TN + 8, SLOTS = 5;
    static constexpr int PLANE = XR * XS;                // floats of one box
    static constexpr int SLOT = (PLANE + 31) / 32 * 32;  // 128-byte aligned slots
    static constexpr uint32_t BOX_BYTES = 4u * PLANE;
    static constexpr int OFF_BAR = 4 * SLOTS * SLOT;
    static constexpr int SMEM_BYTES = OFF_BAR + SLOTS * 8 + 8 + 128;  // + abort flag, alignment slack
};
constexpr int kGmThreads = 256;

__global__ void __launch_bounds__(kGmThreads, 4)
    grad_magn_tiled_kernel(Geometry g, const int4 *__restrict__ cols, int col_begin, int col_end,
                           const int4 *__restrict__ work, const __grid_constant__ CUtensorMap u_map,
                           float *__restrict__ v, int *err)
{
    using T = GmTile;
    static_assert(kGmThreads == 256 && T::TR == 16 && T::TN == 128, "thread assignments are for 16 x 128 tiles");
    extern __shared__ __align__(128) uint8_t gm_raw[];
    uint8_t *const base = gm_raw + ((128u - (smem_addr(gm_raw) & 127u)) & 127u);
    float *const smf = reinterpret_cast<float *>(base);
    uint64_t *const bar = reinterpret_cast<uint64_t *>(base + T::OFF_BAR);
    volatile int *const abort = reinterpret_cast<volatile int *>(base + T::OFF_BAR + T::SLOTS * 8);
    const int t = threadIdx.x;
    const int4 wk = work[blockIdx.x];
    const int r0 = wk.x, n0 = wk.y, ca = wk.z, cb = wk.w;
    auto col_at = [&](int c) { return (c >= col_begin && c < col_end) ? __ldg(cols + c) : make_int4(0, 0, 0, 0); };
    if (t == 0) {
        for (int k = 0; k < T::SLOTS; ++k) mbar_init(bar + k, 1);
        *abort = 0;
        mbar_fence_init();
        tma_prefetch_desc(&u_map);
    }
    __syncthreads();
    // plane c (ca - 1 <= c <= cb) sits in slot (c - ca + 1) mod SLOTS
    auto slot_of = [&](int c) { return (c - ca + 1) % T::SLOTS; };
    uint32_t phase = 0, pending = 0;  // per slot: parity of the next wait, load in flight (thread 0's view)
    auto issue = [&](int c) {         // thread 0 only
        const int s = slot_of(c);
        const int4 ci = col_at(c);
        mbar_arrive_expect_tx(bar + s, T::BOX_BYTES);
        tma_load_2d(smf + s * T::SLOT, &u_map, bar + s, n0 - 4, ci.x - ci.y + r0 - 1);
        pending |= 1u << s;
    };
    auto wait_plane = [&](int c) {  // every thread
        const int s = slot_of(c);
        const bool ok = mbar_wait_warp(bar + s, (phase >> s) & 1u, abort);
        if (ok) {
            phase ^= 1u << s;
            pending &= ~(1u << s);
        }
        return ok;
    };
    if (t == 0)
        for (int c = ca - 1; c <= cb && c < ca - 1 + (T::SLOTS - 1); ++c) issue(c);
    wait_plane(ca - 1);
    wait_plane(ca);
    const int qd = t & 31, h = t >> 5;
    const int nq = n0 + 4 * qd;  // first slice of the thread's quad
    const bool qin = nq < g.ns;  // g.ns % 4 == 0: the whole quad is in the line
#pragma unroll 1
    for (int c = ca; c < cb; ++c) {
        wait_plane(c + 1);
        // past this barrier every thread is done with plane c-2: its slot takes plane c+SLOTS-2
        __syncthreads();
        if (*abort) break;
        if (t == 0 && c + T::SLOTS - 2 <= cb) issue(c + T::SLOTS - 2);
        const int4 ci = col_at(c), cp = col_at(c - 1), cn = col_at(c + 1);
        const float *X = smf + slot_of(c) * T::SLOT;
        const float *Xp = smf + slot_of(c - 1) * T::SLOT, *Xn = smf + slot_of(c + 1) * T::SLOT;
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int rr = h + 8 * m, row = r0 + rr;
            const int b = (rr + 1) * T::XS + 4 * qd + 4;  // slice nq of this row in a box
            const float4 a = *reinterpret_cast<const float4 *>(X + b);
            // slices nq-1 and nq+4 (every lane takes part in the shuffles)
            float before = __shfl_up_sync(0xffffffffu, a.w, 1), after = __shfl_down_sync(0xffffffffu, a.x, 1);
            if (qd == 0) before = X[b - 1];
            if (qd == 31) after = X[b + 4];
            if (!(row >= ci.y && row < ci.z && qin)) continue;
            float r[4] = {-1.0f, -1.0f, -1.0f, -1.0f};
            if (row > ci.y && row + 1 < ci.z && row >= cp.y && row < cp.z && row >= cn.y && row < cn.z) {
                const float4 rn = *reinterpret_cast<const float4 *>(X + b + T::XS);
                const float4 rp = *reinterpret_cast<const float4 *>(X + b - T::XS);
                const float4 cnv = *reinterpret_cast<const float4 *>(Xn + b);
                const float4 cpv = *reinterpret_cast<const float4 *>(Xp + b);
                const float xs[6] = {before, a.x, a.y, a.z, a.w, after};
                const float rnv[4] = {rn.x, rn.y, rn.z, rn.w}, rpv[4] = {rp.x, rp.y, rp.z, rp.w};
                const float cnl[4] = {cnv.x, cnv.y, cnv.z, cnv.w}, cpl[4] = {cpv.x, cpv.y, cpv.z, cpv.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int n = nq + j;
                    if (n > 0 && n + 1 < g.ns) {
                        float q1 = 0.0f, q2 = 0.0f, q3 = 0.0f;
                        q1 += xs[j + 2];
                        q2 += rnv[j];
                        q3 += cnl[j];
                        q1 -= xs[j];
                        q2 -= rpv[j];
                        q3 -= cpl[j];
                        float s = q1 * q1;
                        s = fmaf(q2, q2, s);
                        s = fmaf(q3, q3, s);
                        r[j] = 0.5f * __fsqrt_rn(s);
                    }
                }
            }
            const int64_t line = (int64_t)ci.x + (row - ci.y);
            *reinterpret_cast<float4 *>(v + line * g.nstride_w + nq) = make_float4(r[0], r[1], r[2], r[3]);
        }
    }
    if (t == 0 && *abort) {
        // loads still in flight must land before the block's shared memory goes away
        for (int k = 0; k < T::SLOTS; ++k)
            if ((pending >> k) & 1u) mbar_wait_bounded(bar + k, (phase >> k) & 1u, kDrainTries);
        atomicExch(err, 1);
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

// hist_bin without its division where that cannot change the bin.  rinv = __frcp_rn(end - start),
// the correctly rounded reciprocal.  For |t| <= 1 the product RN((x - start) rinv) differs from
// the quotient t = RN((x - start) / (end - start)) by at most 1.5 ulp(1) (relative errors of
// 2^-24 in rinv, in the product and in t), so y' = fma(nb, product, -0.5) differs from
// hist_bin's fma(nb, t, -0.5) by less than nb 4.2e-7.  The bin is round(y) (halves away from
// zero, then clamped), which can only differ between y and y' when y' lies within that distance
// of a half-integer: then, and for a non-finite y', the division decides.  The bins are the same
// as hist_bin's for every input (one division in about 2 nb 1e-6 of the cases).  Away from a
// half-integer, round(y) is the nearer of floor(y) and floor(y) + 1, which the fraction
// f = y - floor(y) (exact for every finite y) picks: f > 1/2 rounds up.
__device__ __forceinline__ int hist_bin_r(float x, float start, float end, float rinv, int nb)
{
    const float y = fmaf((float)nb, __fmul_rn(__fsub_rn(x, start), rinv), -0.5f);
    const float fl = floorf(y);
    const float f = __fsub_rn(y, fl);
    if (fabsf(__fsub_rn(f, 0.5f)) > fmaf((float)nb, 1e-6f, 1e-6f)) {  // false for a NaN or infinite y
        const float r = f > 0.5f ? __fadd_rn(fl, 1.0f) : fl;  // f > 1/2 only where |y| < 2^23: exact
        return (int)fminf(fmaxf(r, 0.0f), (float)(nb - 1));     // r is finite here
    }
    // near a half-integer: the bin is floor(y) or floor(y) + 1, clamped, which are the same at
    // both ends (x at start or end, e.g. a field saturated there)
    if (f == f && (__fadd_rn(fl, 1.0f) <= 0.0f || fl >= (float)(nb - 1))) return fl >= 0.0f ? nb - 1 : 0;
    return hist_bin(x, start, end, nb);
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

// Adds 1 to counter `id` for every lane whose id it is (kNoBin, and -1 converted: the lane adds
// nothing).  The lanes that share lane 0's id add together with one atomic from lane 0; every
// other lane adds its own 1 (one shuffle and one ballot).  Used where a warp's lanes often share a
// counter or a shared counter is costly: the coarse cell count of the 2-D histogram (64 x 64
// cells) and the 1-D histogram in global memory.  The shared-memory histogram kernels add one
// atomic per lane instead (see hist1d_kernel).  add(id, count) does the atomic; every lane that
// adds reaches the same call, so the warp issues it once.
constexpr uint32_t kNoBin = 0xffffffffu;
template <typename Add>
__device__ __forceinline__ void warp_count(uint32_t id, Add add)
{
    const uint32_t first = __shfl_sync(0xffffffffu, id, 0);
    const unsigned same = __ballot_sync(0xffffffffu, id == first);
    const bool other = id != first;
    if (id != kNoBin && (other || (threadIdx.x & 31) == 0)) add(id, other ? 1u : (uint32_t)__popc(same));
}

// Eight values of one line for one lane of a warp that walks the line in steps of 256 values
// (slices base .. base+255): with kVec two 16-byte loads (quads base/4 + lane and + 32; lines of
// a multiple of 4 values and stride, 16-byte aligned field), else eight coalesced 4-byte loads
// (slices base + lane + 32 j).  Bit j of the result: value j exists.  Several loads in flight
// per lane keep enough bytes moving to cover the memory latency.
template <bool kVec>
__device__ __forceinline__ unsigned load8(const float *__restrict__ line, int ns, int base, int lane, float (&x)[8])
{
    unsigned valid = 0u;
    if constexpr (kVec) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int q = (base >> 2) + lane + 32 * h;
            if (4 * q < ns) {
                const float4 t = __ldg(reinterpret_cast<const float4 *>(line) + q);
                x[4 * h] = t.x, x[4 * h + 1] = t.y, x[4 * h + 2] = t.z, x[4 * h + 3] = t.w;
                valid |= 0xfu << (4 * h);
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int n = base + lane + 32 * j;
            if (n < ns) {
                x[j] = __ldg(line + n);
                valid |= 1u << j;
            }
        }
    }
    return valid;
}

// The slice of value j of load8.
template <bool kVec>
__device__ __forceinline__ int slice8(int base, int lane, int j)
{
    if constexpr (kVec)
        return 4 * ((base >> 2) + lane + 32 * (j >> 2)) + (j & 3);
    else
        return base + lane + 32 * j;
}

// 1-D histogram (calc_hist.cpp:23-80) into shared-memory copies, flushed with one global atomic
// per non-zero bin.  `copies` = 1 (one copy per block) or kHistThreads / 32 (one per warp: when a
// few bins hold most voxels, warps then never contend for the same counter); copies * nb * 4
// bytes of dynamic shared memory.
template <bool kJitter, bool kVec>
__global__ void __launch_bounds__(kHistThreads) hist1d_kernel(Geometry g, const float *__restrict__ f, float rs,
                                                              float re, int nb, int copies, float delta,
                                                              uint64_t seed, uint32_t *__restrict__ ghist)
{
    extern __shared__ uint32_t sh_all[];
    for (int i = threadIdx.x; i < nb * copies; i += blockDim.x) sh_all[i] = 0u;
    __syncthreads();
    uint32_t *sh_hist = sh_all + (copies > 1 ? (int)(threadIdx.x >> 5) * nb : 0);
    const float hd = delta * 0.5f;  // delta / 2, exact
    const float lo = rs - hd;
    const float rinv = __frcp_rn(__fsub_rn(re, rs));
    const int lane = threadIdx.x & 31;
    constexpr int kWarps = kHistThreads / 32;
    // one warp per line
    for (int64_t L = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5); L < g.n_lines; L += (int64_t)gridDim.x * kWarps) {
        const float *line = f + L * g.nstride_w;
        for (int base = 0; base < g.ns; base += 256) {
            float x[8];
            const unsigned valid = load8<kVec>(line, g.ns, base, lane, x);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                uint32_t id = kNoBin;
                if ((valid >> j) & 1u) {
                    float xv = x[j];
                    if (kJitter)
                        xv = __fadd_rn(xv, hist_jitter(seed, (uint64_t)L * g.ns + slice8<kVec>(base, lane, j), delta));
                    // x + 0 compares as x: without jitter the upper test needs no addition
                    if (lo <= xv && (kJitter ? __fadd_rn(xv, hd) : xv) <= re)
                        id = (uint32_t)hist_bin_r(xv, rs, re, rinv, nb);
                }
                // each lane adds its own 1 to its warp's copy (or the block's): grouping the lanes
                // of one bin measured slower even where half the field sits in one bin
                if (id != kNoBin) atomicAdd(sh_hist + id, 1u);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        uint32_t t = 0;
        for (int c = 0; c < copies; ++c) t += sh_all[c * nb + i];
        if (t) atomicAdd(ghist + i, t);
    }
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
            warp_count(id, [&](uint32_t b, uint32_t c) { atomicAdd(ghist + b, c); });
        }
    }
}

// Ranges and layout of the 2-D histogram (uv-hist-kernel.cpp:133-150): the pair (x = u, y = grad
// magnitude) counts at ybin * stride + xbin when it lies in [u_start, u_end] x [v_start, v_end].
struct UvRange {
    float us, ue, vs, ve;
    int nb, stride;
};

// Both bins of the pair, or false outside the ranges.  ru / rv: __frcp_rn(ue - us) and
// __frcp_rn(ve - vs) (hist_bin_r).
__device__ __forceinline__ bool uv_bins(float x, float y, const UvRange &r, float ru, float rv, int &xb, int &yb)
{
    if (!(r.us <= x && x <= r.ue && r.vs <= y && y <= r.ve)) return false;
    xb = hist_bin_r(x, r.us, r.ue, ru, r.nb);
    yb = hist_bin_r(y, r.vs, r.ve, rv, r.nb);
    return true;
}

// The 2-D histogram with its densest bins in every block's own shared memory.  The bins are
// grouped into coarse cells of 2^cs x 2^cs bins (cdim cells per axis, at most kUvCoarseMax);
// uv_coarse_kernel counts the cells over a sample of the lines, the host gives the densest
// cells (up to kUvHotBins bins) a slot, and uv_hist_hot_kernel counts a voxel in its block's
// slot counters when its cell has one, else with a global atomic.  Counts are exact either
// way; the choice of cells only changes speed.
constexpr int kUvCoarseMax = 64;    // coarse cells per axis
constexpr int kUvHotBins = 32768;   // bins counted in a block's shared memory (128 KB)
constexpr int kUvThreads = 1024;    // one block per multiprocessor: as many warps as it holds

template <bool kVec>
__global__ void __launch_bounds__(kHistThreads) uv_coarse_kernel(Geometry g, const float *__restrict__ u,
                                                                 const float *__restrict__ v, UvRange r, int cs,
                                                                 int cdim, int step, uint32_t *__restrict__ gcoarse)
{
    __shared__ uint32_t sh[kUvCoarseMax * kUvCoarseMax];
    const int cells = cdim * cdim;
    for (int i = threadIdx.x; i < cells; i += blockDim.x) sh[i] = 0u;
    __syncthreads();
    const float ru = __frcp_rn(__fsub_rn(r.ue, r.us)), rv = __frcp_rn(__fsub_rn(r.ve, r.vs));
    const int lane = threadIdx.x & 31;
    constexpr int kWarps = kHistThreads / 32;
    for (int64_t k = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5); k * step < g.n_lines;
         k += (int64_t)gridDim.x * kWarps) {
        const int64_t o0 = k * step * g.nstride_w;
        for (int base = 0; base < g.ns; base += 256) {
            float x[8], y[8];
            const unsigned valid = load8<kVec>(u + o0, g.ns, base, lane, x) & load8<kVec>(v + o0, g.ns, base, lane, y);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                uint32_t id = kNoBin;
                int xb, yb;
                if (((valid >> j) & 1u) && uv_bins(x[j], y[j], r, ru, rv, xb, yb))
                    id = (uint32_t)((yb >> cs) * cdim + (xb >> cs));
                warp_count(id, [&](uint32_t b, uint32_t c) { atomicAdd(sh + b, c); });
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < cells; i += blockDim.x)
        if (sh[i]) atomicAdd(gcoarse + i, sh[i]);
}

// Dynamic shared memory: n_slots << 2cs counters, then the cell -> slot table (cdim^2 int16).
template <bool kVec>
__global__ void __launch_bounds__(kUvThreads, 1)
    uv_hist_hot_kernel(Geometry g, const float *__restrict__ u, const float *__restrict__ v, UvRange r, int cs,
                       int cdim, const int16_t *__restrict__ table, const int16_t *__restrict__ slot_cell,
                       int n_slots, uint32_t *__restrict__ ghist)
{
    extern __shared__ uint32_t sh_hot[];
    const int n_hot = n_slots << (2 * cs);
    int16_t *stab = reinterpret_cast<int16_t *>(sh_hot + n_hot);
    for (int i = threadIdx.x; i < n_hot; i += blockDim.x) sh_hot[i] = 0u;
    for (int i = threadIdx.x; i < cdim * cdim; i += blockDim.x) stab[i] = table[i];
    __syncthreads();
    const int mask = (1 << cs) - 1;
    const float ru = __frcp_rn(__fsub_rn(r.ue, r.us)), rv = __frcp_rn(__fsub_rn(r.ve, r.vs));
    const int lane = threadIdx.x & 31;
    constexpr int kWarps = kUvThreads / 32;
    // one warp per line
    for (int64_t L = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5); L < g.n_lines; L += (int64_t)gridDim.x * kWarps) {
        const int64_t o0 = L * g.nstride_w;
        for (int base = 0; base < g.ns; base += 256) {
            float x[8], y[8];
            const unsigned valid = load8<kVec>(u + o0, g.ns, base, lane, x) & load8<kVec>(v + o0, g.ns, base, lane, y);
            // each lane adds its own 1: the 2-D bins of a warp are mostly distinct, and lanes that
            // do share a counter only serialise in the atomic unit (a warp of one bin is at worst
            // one voxel per clock per multiprocessor), which costs less than grouping them
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                int xb, yb;
                if (((valid >> j) & 1u) && uv_bins(x[j], y[j], r, ru, rv, xb, yb)) {
                    const int slot = stab[(yb >> cs) * cdim + (xb >> cs)];
                    if (slot >= 0)
                        atomicAdd(sh_hot + ((slot << (2 * cs)) | ((yb & mask) << cs) | (xb & mask)), 1u);
                    else
                        atomicAdd(ghist + (size_t)yb * r.stride + xb, 1u);
                }
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_hot; i += blockDim.x) {
        const uint32_t c = sh_hot[i];
        if (!c) continue;
        const int cell = slot_cell[i >> (2 * cs)];
        const int yb = ((cell / cdim) << cs) | ((i >> cs) & mask);
        const int xb = ((cell % cdim) << cs) | (i & mask);
        atomicAdd(ghist + (size_t)yb * r.stride + xb, c);
    }
}

}  // namespace potts
