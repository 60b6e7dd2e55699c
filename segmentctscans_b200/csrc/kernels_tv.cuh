// TV-L2 (ROF) denoising by Chambolle's projection algorithm on the cylinder
// (totalvarmin/chambolle.cpp:33-218): the next row of the reference's scope
// table after the Potts solve, on the same layout and neighbour tables.
// State: xi (3 planes) and v (1 plane) laid out like g (the mapping's stride).
// Arithmetic as in the reference's clang build: a multiply and an add are
// fused for the sum of squares, 1 + tau |G|, xi + tau G and g - lambda d; the
// rest are IEEE single operations in source order (the library is compiled
// with -fmad=false).
#pragma once

#include <cuda.h>

#include <cstdint>

#include "geometry.cuh"
#include "kernels_plain.cuh"
#include "tma.cuh"

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

// The lambda-scaled forward differences of g that grad_kernel (:89-166) computes in every
// iteration, computed once per solve with the same operations: D_n = (g(x+e_n) - g(x)) /
// lambda, D_r and D_c likewise (zero where the neighbour does not exist), three planes laid
// out like g.  g does not change during the iterations, so an iteration that reads D gets
// the same bits as one that recomputes it.
__global__ void __launch_bounds__(kPlainThreads) tv_gdiff_kernel(Geometry g, const float *__restrict__ gin,
                                                                 float *__restrict__ D, float lam)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    if (!p.valid) return;
    const LineInfo li = load_line(g, p.line);
    const int64_t o = p.line * g.nstride_w + p.n;
    float d1 = 0.0f, d2 = 0.0f, d3 = 0.0f;
    if (p.n + 1 < g.ns) d1 = __fdiv_rn(gin[o + 1] - gin[o], lam);
    if (li.flags & kHasNextRow) d2 = __fdiv_rn(gin[o + g.nstride_w] - gin[o], lam);
    if (li.next_col >= 0) d3 = __fdiv_rn(gin[(int64_t)li.next_col * g.nstride_w + p.n] - gin[o], lam);
    D[o] = d1;
    D[g.plane_w + o] = d2;
    D[2 * g.plane_w + o] = d3;
}

}  // namespace potts

namespace potts {

// Tiled fused iteration.  A block owns a tile of TR rows x TN slices and marches
// over the columns [ca, cb) of its work item (x = first row, y = first slice,
// z/w = column range, the work items of the Potts kernel).  Shared memory holds
// a ring of three column planes of xi (rows r0-1 .. r0+TR, slices n0-4 ..
// n0+TN+3, the three components), each one TMA box loaded two planes ahead of
// the plane being updated, and two planes of v = div xi (rows r0 .. r0+TR,
// slices n0 .. n0+TN), so that each xi value is read from DRAM once per plane
// and v is computed once per voxel.  The lambda-scaled differences of g come
// from tv_gdiff_kernel's planes.  The operations per voxel are those of
// tv_div_at and tv_grad_kernel, in the same order.  The xi box starts at slice
// n0-4 so that its first word is 16-byte aligned: slice n sits at n - n0 + 4 of
// a row (stride TN + 8); v rows hold slice n at n - n0 (stride TN + 4).  Box
// rows outside the plane's column come from other columns or are zero-filled;
// they are never read.
template <int TR, int TN>
struct TvTile {
    static_assert(TN % 4 == 0, "16-byte aligned box start");
    static constexpr int XR = TR + 2, XS = TN + 8;  // xi box: rows r0-1 .., row stride
    static constexpr int VR = TR + 1, GS = TN + 4;  // v box: rows r0 .., row stride
    static constexpr int XC = XR * XS;              // one xi component
    static constexpr int XI_PLANE = 3 * XC;
    static constexpr int XI_SLOT = (XI_PLANE + 31) / 32 * 32;  // 128-byte aligned slots
    static constexpr int V_PLANE = VR * GS;
    static constexpr uint32_t BOX_BYTES = 4u * XI_PLANE;
    static constexpr int OFF_BAR = 4 * (3 * XI_SLOT + 2 * V_PLANE);  // bytes: 3 mbarriers, abort flag
    static constexpr int SMEM_BYTES = OFF_BAR + 3 * 8 + 8 + 128;     // + alignment slack
};

// column table entry: x = first line, y/z = row range of the column (the Potts kernel's table)
__device__ __forceinline__ bool tv_row_in(int4 ci, int row) { return row >= ci.y && row < ci.z; }

}  // namespace potts

namespace potts {

constexpr int kTvThreads = 256;

// Thread assignments (8 x 128 tiles, 256 threads; fixed for the whole column march, so
// that index arithmetic is done once per block):
//  - update: thread t owns slice nn = t % 128 and rows 4h .. 4h+3 (h = t / 128), walking
//    down the rows with the v value of the row below kept in a register;
//  - divergence: the same slice, v rows 5h .. 5h+4 (of nine), xi_1 of the row above kept in
//    a register; thread t < 9 also computes v at slice n0+128 of row t;
//  - thread 0 issues the TMA loads.
// Every wait on a load is bounded; a block whose wait gives up sets *err, drains its loads in
// flight (bounded) and stops.
template <int TR, int TN>
__global__ void __launch_bounds__(kTvThreads, 3)
    tv_tiled_kernel(Geometry g, const int4 *__restrict__ cols, int col_begin, int col_end,
                    const int4 *__restrict__ work, const __grid_constant__ CUtensorMap xi_map,
                    const __grid_constant__ CUtensorMap d_map, const float *__restrict__ D, float *__restrict__ xi_out,
                    float tau, float *dq, int *err)
{
    static_assert(TR == 8 && TN == 128 && kTvThreads == 256, "thread assignments are for 8 x 128 tiles");
    using T = TvTile<TR, TN>;
    extern __shared__ __align__(128) uint8_t tv_raw[];
    // align to 128 bytes by pointer arithmetic on the shared array itself
    uint8_t *const base = tv_raw + ((128u - (smem_addr(tv_raw) & 127u)) & 127u);
    float *const smf = reinterpret_cast<float *>(base);
    uint64_t *const bar = reinterpret_cast<uint64_t *>(base + T::OFF_BAR);
    volatile int *const abort = reinterpret_cast<volatile int *>(base + T::OFF_BAR + 3 * 8);
    auto sx = [&](int sl) { return smf + sl * T::XI_SLOT; };
    auto sv = [&](int sl) { return smf + 3 * T::XI_SLOT + sl * T::V_PLANE; };
    const int t = threadIdx.x;
    const int4 wk = work[blockIdx.x];
    const int r0 = wk.x, n0 = wk.y, ca = wk.z, cb = wk.w;
    const int64_t nsw = g.nstride_w;
    auto col_at = [&](int c) { return (c >= col_begin && c < col_end) ? cols[c] : make_int4(0, 0, 0, 0); };

    if (t == 0) {
        for (int k = 0; k < 3; ++k) mbar_init(bar + k, 1);
        *abort = 0;
        mbar_fence_init();
        tma_prefetch_desc(&xi_map);
        tma_prefetch_desc(&d_map);
    }
    __syncthreads();
    uint32_t phase = 0, pending = 0;  // per slot: parity of the next wait, load in flight (thread 0's view)
    // plane c's xi box (rows r0-1 .., slices n0-4 ..) into ring slot `slot`, and its box of the
    // differences of g (rows r0 .., slices n0 ..) into L2; thread 0 only
    auto issue = [&](int c, int slot) {
        const int4 ci = col_at(c);
        mbar_arrive_expect_tx(bar + slot, T::BOX_BYTES);
        tma_load_3d(sx(slot), &xi_map, bar + slot, n0 - 4, ci.x - ci.y + r0 - 1, 0);
        pending |= 1u << slot;
        if (c >= ca) tma_prefetch_l2_3d(&d_map, n0, ci.x - ci.y + r0, 0);
    };
    auto wait_slot = [&](int slot) {  // warp-uniform
        const bool ok = mbar_wait_warp(bar + slot, (phase >> slot) & 1u, abort);
        if (ok) {
            phase ^= 1u << slot;
            pending &= ~(1u << slot);
        }
        return ok;
    };

    const int nn = t & (TN - 1), h = t >> 7;
    const int n = n0 + nn;
    const bool nin = n < g.ns, nbk = n > 0, nfw = n + 1 < g.ns;
    // v = div xi of the plane with entry ci (xi box X), previous plane cp (xi box Xp), next cn
    auto divergence = [&](int4 ci, int4 cp, int4 cn, const float *X, const float *Xp, float *V) {
        const float *s0 = X, *s1 = X + T::XC, *s2 = X + 2 * T::XC, *s2p = Xp + 2 * T::XC;
        float up = s1[(5 * h) * T::XS + nn + 4];  // xi_1 of the row above the first
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            const int rr = 5 * h + m;
            if (rr >= T::VR) break;
            const int row = r0 + rr, b = (rr + 1) * T::XS + nn + 4;
            const float a0m = s0[b - 1], a0 = s0[b], a1 = s1[b], a2p = s2p[b], a2 = s2[b];
            float d = 0.0f;
            if (tv_row_in(ci, row) && nin) {
                if (nbk) d -= a0m;
                if (nfw) d += a0;
                if (row > ci.y) d -= up;
                if (row + 1 < ci.z) d += a1;
                if (tv_row_in(cp, row)) d -= a2p;
                if (tv_row_in(cn, row)) d += a2;
            }
            V[rr * T::GS + nn] = d;
            up = a1;
        }
        if (t < T::VR) {  // slice n0+TN of row t
            const int rr = t, row = r0 + rr, ne = n0 + TN, b = (rr + 1) * T::XS + TN + 4;
            float d = 0.0f;
            if (tv_row_in(ci, row) && ne < g.ns) {
                d -= s0[b - 1];
                if (ne + 1 < g.ns) d += s0[b];
                if (row > ci.y) d -= s1[b - T::XS];
                if (row + 1 < ci.z) d += s1[b];
                if (tv_row_in(cp, row)) d -= s2p[b];
                if (tv_row_in(cn, row)) d += s2[b];
            }
            V[rr * T::GS + TN] = d;
        }
    };

    // planes ca-1, ca, ca+1 into slots 0, 1, 2 (plane c sits in slot (c - ca + 1) mod 3)
    if (t == 0)
        for (int k = 0; k < 3; ++k)
            if (ca - 1 + k <= cb) issue(ca - 1 + k, k);
    wait_slot(0);
    wait_slot(1);
    __syncthreads();
    if (!*abort) divergence(col_at(ca), col_at(ca - 1), col_at(ca + 1), sx(1), sx(0), sv(0));
    __syncthreads();
    float dmax = 0.0f;
    int sp = 0, sc = 1, sn = 2;  // slots of planes c-1, c, c+1
    int vc = 0;                  // v slot of plane c
    const int64_t rowoff = (int64_t)(r0 + 4 * h) * nsw + n;
#pragma unroll 1
    for (int c = ca; c < cb; ++c) {
        const int4 ci = col_at(c), cn = col_at(c + 1);
        const int64_t o0 = (int64_t)(ci.x - ci.y) * nsw + rowoff;
        // this plane's differences of g, in flight during the wait and the divergence
        float dg[4][3];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const bool in = tv_row_in(ci, r0 + 4 * h + m) && nin;
            const int64_t o = o0 + m * nsw;
#pragma unroll
            for (int k = 0; k < 3; ++k) dg[m][k] = in ? __ldg(D + k * g.plane_w + o) : 0.0f;
        }
        wait_slot(sn);  // plane c+1
        // past this barrier every thread is done with iteration c-1: the slot of plane c-1 and
        // the v slot of plane c-1 are free
        __syncthreads();
        if (*abort) break;
        if (t == 0 && c + 2 <= cb) issue(c + 2, sp);
        divergence(cn, ci, col_at(c + 2), sx(sn), sx(sc), sv(vc ^ 1));
        __syncthreads();
        const float *Vc = sv(vc), *Vn = sv(vc ^ 1);
        const float *x0 = sx(sc), *x1 = x0 + T::XC, *x2 = x0 + 2 * T::XC;
        float v0 = Vc[(4 * h) * T::GS + nn];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int rr = 4 * h + m, row = r0 + rr;
            const int a = rr * T::GS + nn, b = (rr + 1) * T::XS + nn + 4;
            const float vr = Vc[a + 1], vd = Vc[a + T::GS];
            if (tv_row_in(ci, row) && nin) {
                float g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
                if (nfw) g1 = (vr - v0) - dg[m][0];
                if (row + 1 < ci.z) g2 = (vd - v0) - dg[m][1];
                if (tv_row_in(cn, row)) g3 = (Vn[a] - v0) - dg[m][2];
                float s = g1 * g1;
                s = fmaf(g2, g2, s);
                s = fmaf(g3, g3, s);
                const float denom = fmaf(tau, __fsqrt_rn(s), 1.0f);
                const float xa = x0[b], xb = x1[b], xc = x2[b];
                const float q1 = __fdiv_rn(fmaf(tau, g1, xa), denom);
                const float q2 = __fdiv_rn(fmaf(tau, g2, xb), denom);
                const float q3 = __fdiv_rn(fmaf(tau, g3, xc), denom);
                const float e1 = xa - q1, e2 = xb - q2, e3 = xc - q3;
                float d = e1 * e1;
                d = fmaf(e2, e2, d);
                d = fmaf(e3, e3, d);
                dmax = fmaxf(dmax, d);
                const int64_t o = o0 + m * nsw;
                xi_out[o] = q1;
                xi_out[g.plane_w + o] = q2;
                xi_out[2 * g.plane_w + o] = q3;
            }
            v0 = vd;
        }
        const int tmp = sp;
        sp = sc;
        sc = sn;
        sn = tmp;
        vc ^= 1;
    }
    if (t == 0 && *abort) {
        // loads still in flight must land before the block's shared memory goes away
        for (int k = 0; k < 3; ++k)
            if ((pending >> k) & 1u) mbar_wait_bounded(bar + k, (phase >> k) & 1u, kDrainTries);
        atomicExch(err, 1);
    }
    if (dq) block_max_to(dmax, dq);
}

}  // namespace potts
