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
