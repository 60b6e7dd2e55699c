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

}  // namespace potts

namespace potts {

constexpr int kTvThreads = 256;

// Thread assignments (8 x 128 tiles, 256 threads; fixed for the whole column march, so
// that index arithmetic is done once per block):
//  - update: thread t owns slice nn = t % 128 and rows 4h .. 4h+3 (h = t / 128), walking
//    down the rows with the v and g values of the row below kept in registers;
//  - divergence: the same slice, v rows 5h .. 5h+4 (of nine), xi_1 of the row above kept in
//    registers; thread t < 9 also computes v at slice n0+128 of row t;
//  - copies: 16-byte chunk t % 32 of the xi box lines t/32 + 8j (j < 4; 30 lines =
//    3 components x 10 rows) and of the g box lines t/32 + 8j (j < 2; 9 rows); thread t < 60
//    copies the halo slice of xi line t/2 (n0-1 for even t, n0+128 for odd t), threads
//    64 .. 72 the slice n0+128 of g row t-64.
template <int TR, int TN>
__global__ void __launch_bounds__(kTvThreads, 3)
    tv_tiled_kernel(Geometry g, const int4 *__restrict__ cols, int col_begin, int col_end,
                    const int4 *__restrict__ work, const float *__restrict__ gin, const float *__restrict__ xi_in,
                    float *__restrict__ xi_out, float lam, float tau, float *dq)
{
    static_assert(TR == 8 && TN == 128 && kTvThreads == 256, "thread assignments are for 8 x 128 tiles");
    using T = TvTile<TR, TN>;
    extern __shared__ __align__(16) float tv_smem[];
    auto sx = [&](int sl) { return tv_smem + sl * T::XI_PLANE; };
    auto sg = [&](int sl) { return tv_smem + 3 * T::XI_PLANE + sl * T::V_PLANE; };
    auto sv = [&](int sl) { return tv_smem + 3 * T::XI_PLANE + (3 + sl) * T::V_PLANE; };
    const int t = threadIdx.x;
    const int4 wk = work[blockIdx.x];
    const int r0 = wk.x, n0 = wk.y, ca = wk.z, cb = wk.w;
    const int64_t nsw = g.nstride_w;
    auto col_at = [&](int c) { return (c >= col_begin && c < col_end) ? cols[c] : make_int4(0, 0, 0, 0); };

    // ---- copy assignments
    const int ck = t & 31, cl = t >> 5;
    const int cbytes = 4 * max(0, min(4, g.ns - (n0 + 4 * ck)));
    int64_t xoff[4];
    int xdst[4], xrow[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int line = cl + 8 * j, comp = line / 10, rr = line % 10;
        xrow[j] = line < 30 ? r0 - 1 + rr : INT32_MIN;  // INT32_MIN: no line, never in a column
        xoff[j] = comp * g.plane_w + (int64_t)(r0 - 1 + rr) * nsw + n0 + 4 * ck;
        xdst[j] = comp * T::XC + rr * T::XS + 4 + 4 * ck;
    }
    const int grow1 = cl == 0 ? r0 + 8 : INT32_MIN;  // the ninth g row, copied by warp 0
    // halo slices: kind 1 = xi, 2 = g
    int s_kind = 0, s_row = INT32_MIN, s_dst = 0;
    int64_t s_off = 0;
    if (t < 60) {
        const int line = t >> 1, comp = line / 10, rr = line % 10, n = (t & 1) ? n0 + TN : n0 - 1;
        s_kind = 1;
        s_row = (n >= 0 && n < g.ns) ? r0 - 1 + rr : INT32_MIN;
        s_off = comp * g.plane_w + (int64_t)(r0 - 1 + rr) * nsw + n;
        s_dst = comp * T::XC + rr * T::XS + ((t & 1) ? TN + 4 : 3);
    } else if (t >= 64 && t < 64 + T::VR) {
        const int rr = t - 64, n = n0 + TN;
        s_kind = 2;
        s_row = n < g.ns ? r0 + rr : INT32_MIN;
        s_off = (int64_t)(r0 + rr) * nsw + n;
        s_dst = rr * T::GS + TN;
    }
    auto issue = [&](int c, int slot) {
        const int4 ci = col_at(c);
        const int64_t shift = (int64_t)(ci.x - ci.y) * nsw;  // line of row r: ci.x + r - ci.y
        float *X = sx(slot), *G = sg(slot);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (xrow[j] == INT32_MIN) continue;
            const int b = tv_row_in(ci, xrow[j]) ? cbytes : 0;
            tv_cp_async16(X + xdst[j], b ? xi_in + xoff[j] + shift : xi_in, b);
        }
        {
            const int b = tv_row_in(ci, r0 + cl) ? cbytes : 0;
            tv_cp_async16(G + cl * T::GS + 4 * ck, b ? gin + (int64_t)(r0 + cl) * nsw + n0 + 4 * ck + shift : gin, b);
        }
        if (grow1 != INT32_MIN) {
            const int b = tv_row_in(ci, grow1) ? cbytes : 0;
            tv_cp_async16(G + 8 * T::GS + 4 * ck, b ? gin + (int64_t)grow1 * nsw + n0 + 4 * ck + shift : gin, b);
        }
        if (s_kind) {
            const bool in = tv_row_in(ci, s_row);
            const float *src = s_kind == 1 ? xi_in : gin;
            tv_cp_async4((s_kind == 1 ? X : G) + s_dst, in ? src + s_off + shift : src, in);
        }
    };

    // ---- divergence and update assignments
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
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
        if (ca - 1 + k <= cb) issue(ca - 1 + k, k);
        tv_cp_commit();
    }
    tv_cp_wait_one();  // planes ca-1 and ca have landed (this thread's copies)
    __syncthreads();   // ... and every thread's
    divergence(col_at(ca), col_at(ca - 1), col_at(ca + 1), sx(1), sx(0), sv(0));
    __syncthreads();
    float dmax = 0.0f;
    int sp = 0, sc = 1, sn = 2;  // slots of planes c-1, c, c+1
    int vc = 0;                  // v slot of plane c
    const int64_t rowoff = (int64_t)(r0 + 4 * h) * nsw + n;
#pragma unroll 1
    for (int c = ca; c < cb; ++c) {
        // plane c+2 into the slot of plane c-1, free since the last barrier
        if (c + 2 <= cb) issue(c + 2, sp);
        tv_cp_commit();
        tv_cp_wait_one();  // plane c+1 has landed
        __syncthreads();
        const int4 ci = col_at(c), cn = col_at(c + 1);
        divergence(cn, ci, col_at(c + 2), sx(sn), sx(sc), sv(vc ^ 1));
        __syncthreads();
        const float *Vc = sv(vc), *Vn = sv(vc ^ 1), *Gc = sg(sc), *Gn = sg(sn);
        const float *x0 = sx(sc), *x1 = x0 + T::XC, *x2 = x0 + 2 * T::XC;
        const int64_t o0 = (int64_t)(ci.x - ci.y) * nsw + rowoff;
        float v0 = Vc[(4 * h) * T::GS + nn], gg = Gc[(4 * h) * T::GS + nn];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int rr = 4 * h + m, row = r0 + rr;
            const int a = rr * T::GS + nn, b = (rr + 1) * T::XS + nn + 4;
            const float vr = Vc[a + 1], gr = Gc[a + 1], vd = Vc[a + T::GS], gd = Gc[a + T::GS];
            if (tv_row_in(ci, row) && nin) {
                float g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
                if (nfw) g1 = (vr - v0) - __fdiv_rn(gr - gg, lam);
                if (row + 1 < ci.z) g2 = (vd - v0) - __fdiv_rn(gd - gg, lam);
                if (tv_row_in(cn, row)) g3 = (Vn[a] - v0) - __fdiv_rn(Gn[a] - gg, lam);
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
            gg = gd;
        }
        __syncthreads();
        const int tmp = sp;
        sp = sc;
        sc = sn;
        sn = tmp;
        vc ^= 1;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");  // nothing may be in flight at exit
    if (dq) block_max_to(dmax, dq);
}

}  // namespace potts
