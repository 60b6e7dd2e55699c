// Fused iteration: one launch turns (Xi^m, V^{m-1}) into (Xi^{m+1}, V^m).
//
// The reference runs the dual step (grad_kernel) and then the primal step
// (div_kernel) as two launches and keeps Vbar in memory.  Here the primal step
// of iteration m and the dual step of iteration m+1 run in one launch:
//   V^m    = Pi_S(V^{m-1} + tau1 (div- Xi^m - G))          at x and x + e_a
//   Vbar^m = 2 V^m - V^{m-1}                                (never stored)
//   Xi^{m+1} = Pi_K(Xi^m + tau2 grad+ Vbar^m)               at x
// The forward neighbours' V^m are recomputed from Xi^m and V^{m-1}, which are
// read from buffers nobody writes during the launch (Xi and V are ping-pong
// buffers), so every CTA sees the previous iteration's values.  Per voxel and
// iteration the state traffic is Xi and V read once and written once plus u
// read once: 2*4*(K-1) + 1 floats, 68 bytes for K = 3.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "geometry.cuh"
#include "kernels_plain.cuh"
#include "voxel.cuh"

namespace potts {

// Primal step at (line, n) from Xi^m and V^{m-1}: Vbar^m and V^m.
template <int K>
__device__ __forceinline__ float primal_at(const Geometry &g, int64_t line, const LineInfo &li, int n,
                                           const float *__restrict__ X, const float *__restrict__ V,
                                           const float *__restrict__ u, const PhaseParams<K> &pp,
                                           float (&vnew)[K - 1], float (&vbar)[K - 1])
{
    const int64_t o = line * g.nstride_w + n;
    const bool hn = n + 1 < g.ns, pn = n > 0;
    const bool hr = li.flags & kHasNextRow, pr = li.flags & kHasPrevRow;
    const bool hc = li.next_col >= 0, pc = li.prev_col >= 0;
    const int64_t opc = pc ? (int64_t)li.prev_col * g.nstride_w + n : o;
    float x[3 * (K - 1)], xn[K - 1], xr[K - 1], xc[K - 1], v[K - 1];
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        const float *b0 = X + (3 * i) * g.plane_w;
        const float *b1 = X + (3 * i + 1) * g.plane_w;
        const float *b2 = X + (3 * i + 2) * g.plane_w;
        x[3 * i] = b0[o];
        x[3 * i + 1] = b1[o];
        x[3 * i + 2] = b2[o];
        xn[i] = pn ? b0[o - 1] : 0.0f;
        xr[i] = pr ? b1[o - g.nstride_w] : 0.0f;
        xc[i] = pc ? b2[opc] : 0.0f;
        v[i] = V[i * g.plane_w + o];
    }
    const float uu = u[line * g.nstride_in + g.slab_start + n];
    return primal_voxel<K>(vnew, vbar, v, x, xn, xr, xc, pn, hn, pr, hr, pc, hc, uu, pp.c, pp.lam, pp.tau1);
}

// Direct form: one thread per voxel, forward neighbours' primal steps
// recomputed per thread.
template <int K>
__global__ void __launch_bounds__(kPlainThreads)
    fused_direct_kernel(Geometry g, const float *__restrict__ Xin, const float *__restrict__ Vin,
                        float *__restrict__ Xout, float *__restrict__ Vout, const float *__restrict__ u,
                        PhaseParams<K> pp, float tau2, DykstraThresholds thr, float *dq)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    float d = 0.0f;
    if (p.valid) {
        const LineInfo li = load_line(g, p.line);
        float vnew[K - 1], vb[K - 1], vbn[K - 1], vbr[K - 1], vbc[K - 1], tmp[K - 1];
        d = primal_at<K>(g, p.line, li, p.n, Xin, Vin, u, pp, vnew, vb);
        const bool hn = p.n + 1 < g.ns;
        const bool hr = li.flags & kHasNextRow;
        const bool hc = li.next_col >= 0;
#pragma unroll
        for (int i = 0; i < K - 1; ++i) vbn[i] = vbr[i] = vbc[i] = 0.0f;
        if (hn) primal_at<K>(g, p.line, li, p.n + 1, Xin, Vin, u, pp, tmp, vbn);
        if (hr) {
            const LineInfo lr = load_line(g, p.line + 1);
            primal_at<K>(g, p.line + 1, lr, p.n, Xin, Vin, u, pp, tmp, vbr);
        }
        if (hc) {
            const LineInfo lc = load_line(g, li.next_col);
            primal_at<K>(g, li.next_col, lc, p.n, Xin, Vin, u, pp, tmp, vbc);
        }
        const int64_t o = p.line * g.nstride_w + p.n;
        float x[3 * (K - 1)], xo[3 * (K - 1)];
#pragma unroll
        for (int j = 0; j < 3 * (K - 1); ++j) x[j] = Xin[j * g.plane_w + o];
        dual_voxel<K>(xo, x, vb, vbn, vbr, vbc, hn, hr, hc, tau2, thr);
#pragma unroll
        for (int j = 0; j < 3 * (K - 1); ++j) Xout[j * g.plane_w + o] = xo[j];
#pragma unroll
        for (int i = 0; i < K - 1; ++i) Vout[i * g.plane_w + o] = vnew[i];
    }
    if (dq) block_max_to(d, dq);
}

template <int K>
cudaError_t launch_fused(const Geometry &g, const float *Xin, const float *Vin, float *Xout, float *Vout, const float *u,
                 const PhaseParams<K> &pp, float tau2, DykstraThresholds thr, float *dq, cudaStream_t s)
{
    const int chunks = (g.ns + kPlainThreads - 1) / kPlainThreads;
    const unsigned nb = (unsigned)(g.n_lines * chunks);
    fused_direct_kernel<K><<<nb, kPlainThreads, 0, s>>>(g, Xin, Vin, Xout, Vout, u, pp, tau2, thr, dq);
    return cudaGetLastError();
}

}  // namespace potts
