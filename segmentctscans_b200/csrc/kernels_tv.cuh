// TV-L2 (ROF) denoising by Chambolle's projection algorithm on the cylinder
// (totalvarmin/chambolle.cpp:33-218): the next row of the reference's scope
// table after the Potts solve, on the same layout and neighbour tables.
// State: xi (3 planes) and v (1 plane) laid out like g (the mapping's stride).
// Arithmetic as in the reference's clang build: a multiply and an add are
// fused for the sum of squares, 1 + tau |G|, xi + tau G and g - lambda d; the
// rest are IEEE single operations in source order (the library is compiled
// with -fmad=false).
#pragma once

#include <cstdint>

#include "geometry.cuh"
#include "kernels_plain.cuh"

namespace potts {

// div_kernel (:33-87): d = -xi_n(x-e_n) + xi_n(x) - xi_r(x-e_r) + xi_r(x) - xi_c(x-e_c) + xi_c(x),
// each term only where that neighbour exists, in this order.
__device__ __forceinline__ float tv_div_at(const Geometry &g, const float *__restrict__ xi, int64_t o, int n,
                                           const LineInfo &li)
{
    const float *x0 = xi, *x1 = xi + g.plane_w, *x2 = xi + 2 * g.plane_w;
    float d = 0.0f;
    if (n > 0) d -= x0[o - 1];
    if (n + 1 < g.ns) d += x0[o];
    if (li.flags & kHasPrevRow) d -= x1[o - g.nstride_w];
    if (li.flags & kHasNextRow) d += x1[o];
    if (li.prev_col >= 0) d -= x2[(int64_t)li.prev_col * g.nstride_w + n];
    if (li.next_col >= 0) d += x2[o];
    return d;
}

__global__ void __launch_bounds__(kPlainThreads) tv_div_kernel(Geometry g, const float *__restrict__ xi,
                                                               float *__restrict__ v)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    if (!p.valid) return;
    const LineInfo li = load_line(g, p.line);
    const int64_t o = p.line * g.nstride_w + p.n;
    v[o] = tv_div_at(g, xi, o, p.n, li);
}

// grad_kernel (:89-166): G = grad+ v - (grad+ g) / lambda, xi <- (xi + tau G) / (1 + tau |G|),
// max |dxi|^2 into *dq.
__global__ void __launch_bounds__(kPlainThreads) tv_grad_kernel(Geometry g, const float *__restrict__ gin,
                                                                float *__restrict__ xi, const float *__restrict__ v,
                                                                float lam, float tau, float *dq)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    float d = 0.0f;
    if (p.valid) {
        const LineInfo li = load_line(g, p.line);
        const int64_t o = p.line * g.nstride_w + p.n;
        float g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
        if (p.n + 1 < g.ns) g1 = (v[o + 1] - v[o]) - __fdiv_rn(gin[o + 1] - gin[o], lam);
        if (li.flags & kHasNextRow) {
            const int64_t q = o + g.nstride_w;
            g2 = (v[q] - v[o]) - __fdiv_rn(gin[q] - gin[o], lam);
        }
        if (li.next_col >= 0) {
            const int64_t q = (int64_t)li.next_col * g.nstride_w + p.n;
            g3 = (v[q] - v[o]) - __fdiv_rn(gin[q] - gin[o], lam);
        }
        float s = g1 * g1;
        s = fmaf(g2, g2, s);
        s = fmaf(g3, g3, s);
        const float denom = fmaf(tau, __fsqrt_rn(s), 1.0f);
        float *x0 = xi + o, *x1 = xi + g.plane_w + o, *x2 = xi + 2 * g.plane_w + o;
        const float q1 = __fdiv_rn(fmaf(tau, g1, *x0), denom);
        const float q2 = __fdiv_rn(fmaf(tau, g2, *x1), denom);
        const float q3 = __fdiv_rn(fmaf(tau, g3, *x2), denom);
        const float e1 = *x0 - q1, e2 = *x1 - q2, e3 = *x2 - q3;
        d = e1 * e1;
        d = fmaf(e2, e2, d);
        d = fmaf(e3, e3, d);
        *x0 = q1;
        *x1 = q2;
        *x2 = q3;
    }
    if (dq) block_max_to(d, dq);
}

// One fused iteration: the div and grad kernels in one launch.  Each thread
// rebuilds v = div xi at its voxel and at the three forward neighbours from
// xi_in (neighbour reads are L1/L2 hits), so v is never stored, and writes
// xi_out (ping-pong: other threads still read xi_in).  Same operations in the
// same order as tv_div_kernel + tv_grad_kernel, so the same bits; DRAM traffic
// xi in (3) + g (1) + xi out (3) = 28 B per voxel instead of 48 B.
__global__ void __launch_bounds__(kPlainThreads) tv_fused_kernel(Geometry g, const float *__restrict__ gin,
                                                                 const float *__restrict__ xi_in,
                                                                 float *__restrict__ xi_out, float lam, float tau,
                                                                 float *dq)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    float d = 0.0f;
    if (p.valid) {
        const LineInfo li = load_line(g, p.line);
        const int64_t o = p.line * g.nstride_w + p.n;
        const float v0 = tv_div_at(g, xi_in, o, p.n, li);
        float g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
        if (p.n + 1 < g.ns) {
            const float vn = tv_div_at(g, xi_in, o + 1, p.n + 1, li);
            g1 = (vn - v0) - __fdiv_rn(gin[o + 1] - gin[o], lam);
        }
        if (li.flags & kHasNextRow) {
            const int64_t q = o + g.nstride_w;
            const float vr = tv_div_at(g, xi_in, q, p.n, load_line(g, p.line + 1));
            g2 = (vr - v0) - __fdiv_rn(gin[q] - gin[o], lam);
        }
        if (li.next_col >= 0) {
            const int64_t q = (int64_t)li.next_col * g.nstride_w + p.n;
            const float vc = tv_div_at(g, xi_in, q, p.n, load_line(g, li.next_col));
            g3 = (vc - v0) - __fdiv_rn(gin[q] - gin[o], lam);
        }
        float s = g1 * g1;
        s = fmaf(g2, g2, s);
        s = fmaf(g3, g3, s);
        const float denom = fmaf(tau, __fsqrt_rn(s), 1.0f);
        const float x0 = xi_in[o], x1 = xi_in[g.plane_w + o], x2 = xi_in[2 * g.plane_w + o];
        const float q1 = __fdiv_rn(fmaf(tau, g1, x0), denom);
        const float q2 = __fdiv_rn(fmaf(tau, g2, x1), denom);
        const float q3 = __fdiv_rn(fmaf(tau, g3, x2), denom);
        const float e1 = x0 - q1, e2 = x1 - q2, e3 = x2 - q3;
        d = e1 * e1;
        d = fmaf(e2, e2, d);
        d = fmaf(e3, e3, d);
        xi_out[o] = q1;
        xi_out[g.plane_w + o] = q2;
        xi_out[2 * g.plane_w + o] = q3;
    }
    if (dq) block_max_to(d, dq);
}

// update_kernel (:168-218): g <- g - lambda div xi.
__global__ void __launch_bounds__(kPlainThreads) tv_update_kernel(Geometry g, float *__restrict__ gio,
                                                                  const float *__restrict__ xi, float lam)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    if (!p.valid) return;
    const LineInfo li = load_line(g, p.line);
    const int64_t o = p.line * g.nstride_w + p.n;
    gio[o] = fmaf(-lam, tv_div_at(g, xi, o, p.n, li), gio[o]);
}

}  // namespace potts

namespace potts {

// Tiled fused iteration.  A block owns a tile of TR rows x TN slices and marches
// over the columns [ca, cb) of its work item (x = first row, y = first slice,
// z/w = column range, the work items of the Potts kernel).  Shared memory holds
// a ring of three column planes of xi (rows r0-1 .. r0+TR, slices n0-1 ..
// n0+TN) and of g (rows r0 .. r0+TR, slices n0 .. n0+TN), filled by cp.async
// two planes ahead of the plane being updated, and two planes of v = div xi
// (the g box), so that each xi, g value is read from DRAM once per plane and v
// is computed once per voxel.  The operations per voxel are those of
// tv_div_at and tv_grad_kernel, in the same order.  Rows of the boxes are
// padded so that slice n0 starts a 16-byte word: xi rows hold slice n at
// n - n0 + 4 (stride TN + 8), g and v rows at n - n0 (stride TN + 4); the
// slices n0 .. n0+TN-1 of a row come in 16-byte copies, the halo slices
// singly.
template <int TR, int TN>
struct TvTile {
    static_assert(TN % 4 == 0, "16-byte row chunks");
    static constexpr int XR = TR + 2, XS = TN + 8;  // xi box: rows r0-1 .., row stride
    static constexpr int VR = TR + 1, GS = TN + 4;  // v and g boxes: rows r0 .., row stride
    static constexpr int XC = XR * XS;              // one xi component
    static constexpr int XI_PLANE = 3 * XC;
    static constexpr int V_PLANE = VR * GS;
    static constexpr int SMEM_FLOATS = 3 * XI_PLANE + 3 * V_PLANE + 2 * V_PLANE;
};

// column table entry: x = first line, y/z = row range of the column (the Potts kernel's table)
__device__ __forceinline__ bool tv_row_in(int4 ci, int row) { return row >= ci.y && row < ci.z; }

// asynchronous copies global -> shared: 4 bytes (zero when !valid), and 16 bytes of which the
// first `bytes` are read and the rest zero-filled
__device__ __forceinline__ void tv_cp_async4(float *dst, const float *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void tv_cp_async16(float *dst, const float *src, int bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tv_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most one group (the newest) of this thread's copies is in flight
__device__ __forceinline__ void tv_cp_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Issue the copies of one column plane (table entry ci) into the xi box sx and the g box sg.
// Global rows start on 16-byte words: the line stride is a multiple of 32 floats, the planes
// are multiples of it and the base pointers are 16-byte aligned (checked by the host).
template <int TR, int TN>
__device__ __forceinline__ void tv_issue_plane(const Geometry &g, int4 ci, int r0, int n0,
                                               const float *__restrict__ xi_in, const float *__restrict__ gin,
                                               float *sx, float *sg)
{
    using T = TvTile<TR, TN>;
    constexpr int CH = TN / 4;      // 16-byte chunks per row
    constexpr int XO = CH + 2;      // xi row: chunks, then slice n0-1, then slice n0+TN
    constexpr int GO = CH + 1;      // g row: chunks, then slice n0+TN
    for (int i = threadIdx.x; i < 3 * T::XR * XO; i += blockDim.x) {
        const int line = i / XO, k = i % XO;  // line = comp * XR + rr
        const int comp = line / T::XR, rr = line % T::XR;
        const int row = r0 - 1 + rr;
        const bool rin = tv_row_in(ci, row);
        const int64_t gl = comp * g.plane_w + (int64_t)(ci.x + row - ci.y) * g.nstride_w;
        float *dst = sx + comp * T::XC + rr * T::XS;
        if (k < CH) {
            const int n = n0 + 4 * k;
            const int bytes = rin ? 4 * max(0, min(4, g.ns - n)) : 0;
            tv_cp_async16(dst + 4 + 4 * k, bytes ? xi_in + gl + n : xi_in, bytes);
        } else {
            const int n = k == CH ? n0 - 1 : n0 + TN;
            const bool in = rin && n >= 0 && n < g.ns;
            tv_cp_async4(dst + (k == CH ? 3 : TN + 4), in ? xi_in + gl + n : xi_in, in);
        }
    }
    for (int i = threadIdx.x; i < T::VR * GO; i += blockDim.x) {
        const int rr = i / GO, k = i % GO;
        const int row = r0 + rr;
        const bool rin = tv_row_in(ci, row);
        const int64_t gl = (int64_t)(ci.x + row - ci.y) * g.nstride_w;
        float *dst = sg + rr * T::GS;
        if (k < CH) {
            const int n = n0 + 4 * k;
            const int bytes = rin ? 4 * max(0, min(4, g.ns - n)) : 0;
            tv_cp_async16(dst + 4 * k, bytes ? gin + gl + n : gin, bytes);
        } else {
            const int n = n0 + TN;
            const bool in = rin && n < g.ns;
            tv_cp_async4(dst + TN, in ? gin + gl + n : gin, in);
        }
    }
}

// v = div xi at (plane with table entry ci, its xi box sx; the previous plane's xi box sxp and
// entry cp) for the v box (rows r0 .. r0+TR, slices n0 .. n0+TN).
template <int TR, int TN>
__device__ __forceinline__ void tv_plane_div(const Geometry &g, int4 ci, int4 cp, int4 cn, int r0, int n0,
                                             const float *sx, const float *sxp, float *sv)
{
    using T = TvTile<TR, TN>;
    constexpr int VN = TN + 1;
    const float *s0 = sx, *s1 = sx + T::XC, *s2p = sxp + 2 * T::XC, *s2 = sx + 2 * T::XC;
    for (int i = threadIdx.x; i < T::VR * VN; i += blockDim.x) {
        const int rr = i / VN, nn = i % VN;
        const int row = r0 + rr, n = n0 + nn;
        float d = 0.0f;
        if (tv_row_in(ci, row) && n < g.ns) {
            const int b = (rr + 1) * T::XS + (nn + 4);  // (row, n) in the xi box
            if (n > 0) d -= s0[b - 1];
            if (n + 1 < g.ns) d += s0[b];
            if (row > ci.y) d -= s1[b - T::XS];
            if (row + 1 < ci.z) d += s1[b];
            if (tv_row_in(cp, row)) d -= s2p[b];
            if (tv_row_in(cn, row)) d += s2[b];
        }
        sv[rr * T::GS + nn] = d;
    }
}

}  // namespace potts

namespace potts {

constexpr int kTvThreads = 256;

template <int TR, int TN>
__global__ void __launch_bounds__(kTvThreads)
    tv_tiled_kernel(Geometry g, const int4 *__restrict__ cols, int col_begin, int col_end,
                    const int4 *__restrict__ work, const float *__restrict__ gin, const float *__restrict__ xi_in,
                    float *__restrict__ xi_out, float lam, float tau, float *dq)
{
    using T = TvTile<TR, TN>;
    extern __shared__ __align__(16) float tv_smem[];
    // ring slots (0..2 for xi and g, 0..1 for v), selected arithmetically to stay in registers
    auto sx = [&](int sl) { return tv_smem + sl * T::XI_PLANE; };
    auto sg = [&](int sl) { return tv_smem + 3 * T::XI_PLANE + sl * T::V_PLANE; };
    auto sv = [&](int sl) { return tv_smem + 3 * T::XI_PLANE + (3 + sl) * T::V_PLANE; };
    const int4 wk = work[blockIdx.x];
    const int r0 = wk.x, n0 = wk.y, ca = wk.z, cb = wk.w;
    auto col_at = [&](int c) { return (c >= col_begin && c < col_end) ? cols[c] : make_int4(0, 0, 0, 0); };

    // planes ca-1, ca, ca+1 into slots 0, 1, 2 (plane c sits in slot (c - ca + 1) mod 3)
    for (int k = 0; k < 3; ++k) {
        if (ca - 1 + k <= cb) tv_issue_plane<TR, TN>(g, col_at(ca - 1 + k), r0, n0, xi_in, gin, sx(k), sg(k));
        tv_cp_commit();
    }
    tv_cp_wait_one();  // planes ca-1 and ca have landed (this thread's copies)
    __syncthreads();   // ... and every thread's
    tv_plane_div<TR, TN>(g, col_at(ca), col_at(ca - 1), col_at(ca + 1), r0, n0, sx(1), sx(0), sv(0));
    __syncthreads();
    float dmax = 0.0f;
    int sp = 0, sc = 1, sn = 2;  // slots of planes c-1, c, c+1
    int vc = 0;                  // v slot of plane c
    for (int c = ca; c < cb; ++c) {
        // plane c+2 into the slot of plane c-1, free since the last barrier
        if (c + 2 <= cb) tv_issue_plane<TR, TN>(g, col_at(c + 2), r0, n0, xi_in, gin, sx(sp), sg(sp));
        tv_cp_commit();
        tv_cp_wait_one();  // plane c+1 has landed
        __syncthreads();
        const int4 ci = col_at(c), cn = col_at(c + 1);
        tv_plane_div<TR, TN>(g, cn, ci, col_at(c + 2), r0, n0, sx(sn), sx(sc), sv(vc ^ 1));
        __syncthreads();
        const float *v0p = sv(vc), *v1p = sv(vc ^ 1), *g0p = sg(sc), *g1p = sg(sn);
        const float *x0 = sx(sc), *x1 = x0 + T::XC, *x2 = x0 + 2 * T::XC;
        for (int i = threadIdx.x; i < TR * TN; i += blockDim.x) {
            const int rr = i / TN, nn = i % TN;
            const int row = r0 + rr, n = n0 + nn;
            if (!tv_row_in(ci, row) || n >= g.ns) continue;
            const int a = rr * T::GS + nn;                  // (row, n) in the v and g boxes
            const int b = (rr + 1) * T::XS + (nn + 4);      // (row, n) in the xi box
            const float v0 = v0p[a], gg = g0p[a];
            float g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
            if (n + 1 < g.ns) g1 = (v0p[a + 1] - v0) - __fdiv_rn(g0p[a + 1] - gg, lam);
            if (row + 1 < ci.z) g2 = (v0p[a + T::GS] - v0) - __fdiv_rn(g0p[a + T::GS] - gg, lam);
            if (tv_row_in(cn, row)) g3 = (v1p[a] - v0) - __fdiv_rn(g1p[a] - gg, lam);
            float s = g1 * g1;
            s = fmaf(g2, g2, s);
            s = fmaf(g3, g3, s);
            const float denom = fmaf(tau, __fsqrt_rn(s), 1.0f);
            const float q1 = __fdiv_rn(fmaf(tau, g1, x0[b]), denom);
            const float q2 = __fdiv_rn(fmaf(tau, g2, x1[b]), denom);
            const float q3 = __fdiv_rn(fmaf(tau, g3, x2[b]), denom);
            const float e1 = x0[b] - q1, e2 = x1[b] - q2, e3 = x2[b] - q3;
            float d = e1 * e1;
            d = fmaf(e2, e2, d);
            d = fmaf(e3, e3, d);
            dmax = fmaxf(dmax, d);
            const int64_t o = (int64_t)(ci.x + row - ci.y) * g.nstride_w + n;
            xi_out[o] = q1;
            xi_out[g.plane_w + o] = q2;
            xi_out[2 * g.plane_w + o] = q3;
        }
        __syncthreads();
        const int t = sp;
        sp = sc;
        sc = sn;
        sn = t;
        vc ^= 1;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");  // nothing may be in flight at exit
    if (dq) block_max_to(dmax, dq);
}

}  // namespace potts
