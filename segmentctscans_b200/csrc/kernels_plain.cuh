// Split ("plain") kernels: the reference's kernel structure, one launch for
// the dual step and one for the primal step per iteration, one thread per
// voxel.  They are the parity baseline of the library, and the fused form uses
// them for its first dual step and its last primal step.
#pragma once

#include <cstdint>

#include <type_traits>

#include "geometry.cuh"
#include "storage.cuh"
#include "voxel.cuh"
#include "voxel_f64.cuh"
#include "voxel_fast.cuh"

namespace potts {

constexpr int kPlainThreads = 256;

// Thread -> (line, n) for the split kernels: blocks walk the lines, each
// block covers kPlainThreads consecutive n of one line.
struct PlainIndex {
    int64_t line;
    int n;
    bool valid;
};

__device__ __forceinline__ PlainIndex plain_index(const Geometry &g, int n_begin, int n_end)
{
    const int chunks = (n_end - n_begin + kPlainThreads - 1) / kPlainThreads;
    PlainIndex p;
    p.line = g.line_begin + (int64_t)blockIdx.x / chunks;
    p.n = n_begin + (int)(blockIdx.x % chunks) * kPlainThreads + (int)threadIdx.x;
    p.valid = p.line < g.n_lines && p.n < n_end;
    return p;
}

// init_v_kernel: V = Vbar = one-hot of the nearest label (Vbar optional).
template <int K, typename ST>
__global__ void __launch_bounds__(kPlainThreads) init_kernel(Geometry g, const float *__restrict__ u, ST *V, ST *Vb,
                                                              PhaseParams<K> pp)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    if (!p.valid) return;
    const int64_t o = p.line * g.nstride_w + p.n;
    const float x = u[p.line * g.nstride_in + g.slab_start + p.n];
    int cl;
    if constexpr (std::is_same_v<ST, double>)
        cl = nearest_label_f64<K>((double)x, pp.c);
    else
        cl = nearest_label<K>(x, pp.c);
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        const typename Store<ST>::Real one = (i == cl) ? 1.0f : 0.0f;
        V[i * g.plane_w + o] = Store<ST>::st(one);
        if (Vb) Vb[i * g.plane_w + o] = Store<ST>::st(one);
    }
}

// grad_kernel: Xi <- Pi_K(Xi + tau2 * grad+ Vbar), in place.  FAST: the fast
// FP32 arithmetic (voxel_fast.cuh; missing neighbours read as zeros).
template <int K, typename ST, bool FAST = false>
__global__ void __launch_bounds__(kPlainThreads) dual_kernel(Geometry g, ST *__restrict__ xi,
                                                              const ST *__restrict__ vb, float tau2,
                                                              DykstraThresholds thr)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    if (!p.valid) return;
    const LineInfo li = load_line(g, p.line);
    const int64_t o = p.line * g.nstride_w + p.n;
    const bool hn = p.n + 1 < g.ns;
    const bool hr = li.flags & kHasNextRow;
    const bool hc = li.next_col >= 0;
    const int64_t oc = hc ? (int64_t)li.next_col * g.nstride_w + p.n : o;
    using R = typename Store<ST>::Real;
    R vx[K - 1], vn[K - 1], vr[K - 1], vc[K - 1], x[3 * (K - 1)], xo[3 * (K - 1)];
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        const ST *b = vb + i * g.plane_w;
        vx[i] = Store<ST>::ld(b[o]);
        vn[i] = hn ? Store<ST>::ld(b[o + 1]) : R(0);
        vr[i] = hr ? Store<ST>::ld(b[o + g.nstride_w]) : R(0);
        vc[i] = hc ? Store<ST>::ld(b[oc]) : R(0);
    }
#pragma unroll
    for (int j = 0; j < 3 * (K - 1); ++j) x[j] = Store<ST>::ld(xi[j * g.plane_w + o]);
    if constexpr (std::is_same_v<R, double>) {
        dual_voxel_f64<K>(xo, x, vx, vn, vr, vc, hn, hr, hc, (double)tau2);
    } else if constexpr (FAST) {
        float q[K][3];
        fast::dual_q<K, float>(q, x, vx, vn, vr, vc, hn ? tau2 : 0.0f, hr ? tau2 : 0.0f, hc ? tau2 : 0.0f);
        if (fast::max_pair_dist2<K, float>(q) > 1.0f) fast::dual_project<K>(q);
        dual_store<K>(xo, q);
    } else {
        dual_voxel<K>(xo, x, vx, vn, vr, vc, hn, hr, hc, tau2, thr);
    }
#pragma unroll
    for (int j = 0; j < 3 * (K - 1); ++j) xi[j * g.plane_w + o] = Store<ST>::st(xo[j]);
}

// Block-wide max of a non-negative float, then one atomic per block into *dst.
__device__ __forceinline__ void block_max_to(float v, float *dst)
{
    __shared__ float red[32];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, s));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? red[lane] : 0.0f;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, s));
        // non-negative floats order like their bit patterns
        if (lane == 0 && v > 0.0f) atomicMax(reinterpret_cast<int *>(dst), __float_as_int(v));
    }
}

// div_kernel: V <- Pi_S(V + tau1 (div- Xi - G)), Vbar <- 2 V_new - V (optional),
// max |dV|^2 into *dq (optional).  it: 0-based iteration (keys the stochastic
// rounding of a bfloat16 V).
template <int K, typename ST, bool FAST = false>
__global__ void __launch_bounds__(kPlainThreads) primal_kernel(Geometry g, const ST *__restrict__ xi,
                                                                ST *__restrict__ V, ST *__restrict__ Vb,
                                                                const float *__restrict__ u, PhaseParams<K> pp,
                                                                float *dq, int it)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    float d = 0.0f;
    if (p.valid) {
        const LineInfo li = load_line(g, p.line);
        const int64_t o = p.line * g.nstride_w + p.n;
        const bool hn = p.n + 1 < g.ns, pn = p.n > 0;
        const bool hr = li.flags & kHasNextRow, pr = li.flags & kHasPrevRow;
        const bool hc = li.next_col >= 0, pc = li.prev_col >= 0;
        const int64_t opc = pc ? (int64_t)li.prev_col * g.nstride_w + p.n : o;
        using R = typename Store<ST>::Real;
        R x[3 * (K - 1)], xn[K - 1], xr[K - 1], xc[K - 1], v[K - 1], vnew[K - 1], vbar[K - 1];
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            const ST *b0 = xi + (3 * i) * g.plane_w;
            const ST *b1 = xi + (3 * i + 1) * g.plane_w;
            const ST *b2 = xi + (3 * i + 2) * g.plane_w;
            x[3 * i] = Store<ST>::ld(b0[o]);
            x[3 * i + 1] = Store<ST>::ld(b1[o]);
            x[3 * i + 2] = Store<ST>::ld(b2[o]);
            xn[i] = pn ? Store<ST>::ld(b0[o - 1]) : R(0);
            xr[i] = pr ? Store<ST>::ld(b1[o - g.nstride_w]) : R(0);
            xc[i] = pc ? Store<ST>::ld(b2[opc]) : R(0);
            v[i] = Store<ST>::ld(V[i * g.plane_w + o]);
        }
        const float uu = u[p.line * g.nstride_in + g.slab_start + p.n];
        if constexpr (std::is_same_v<R, double>)
            d = (float)primal_voxel_f64<K>(vnew, vbar, v, x, xn, xr, xc, pn, hn, pr, hr, pc, hc, (double)uu, pp.c,
                                           (double)pp.lam, (double)pp.tau1);
        else if constexpr (FAST)
            d = fast::primal<K, float>(vnew, vbar, v, x, xn, xr, xc, pc ? -1.0f : -0.0f, uu, pp.c, pp.lam, pp.tau1);
        else
            d = primal_voxel<K>(vnew, vbar, v, x, xn, xr, xc, pn, hn, pr, hr, pc, hc, uu, pp.c, pp.lam, pp.tau1);
        uint32_t h[(K - 1 + 1) / 2];
        if constexpr (Store<ST>::kStochasticV) {
#pragma unroll
            for (int k = 0; k < (K - 1 + 1) / 2; ++k)
                h[k] = sr_hash((uint32_t)(g.line_base + p.line), (uint32_t)(g.slab_start + p.n), (uint32_t)it,
                               (uint32_t)k);
        }
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            if constexpr (Store<ST>::kStochasticV)
                V[i * g.plane_w + o] = Store<ST>::st_v(vnew[i], sr_bits(h[i >> 1], i));
            else
                V[i * g.plane_w + o] = Store<ST>::st(vnew[i]);
            if (Vb) Vb[i * g.plane_w + o] = Store<ST>::st(vbar[i]);
        }
    }
    if (dq) block_max_to(d, dq);
}

// update_kernel: argmax over n in [res_begin, res_end) of the slab, written
// with the input mapping; optionally copies V and Xi out.
// V and Xi are written as OT (FP32, or FP64 from the FP64 state); OT is
// given, never deduced from the (possibly null) output pointers.
template <typename T>
struct Given {
    using type = T;
};
template <int K, typename ST, typename OT = float>
__global__ void __launch_bounds__(kPlainThreads) update_kernel(Geometry g, const ST *__restrict__ V,
                                                                const ST *__restrict__ xi, PhaseParams<K> pp,
                                                                int res_begin, int res_end, float *res,
                                                                uint8_t *labels, typename Given<OT>::type *V_out,
                                                                typename Given<OT>::type *Xi_out, int64_t plane_out)
{
    const PlainIndex p = plain_index(g, res_begin, res_end);
    if (!p.valid) return;
    const int64_t o = p.line * g.nstride_w + p.n;
    const int64_t oo = p.line * g.nstride_in + g.slab_start + p.n;
    typename Store<ST>::Real v[K - 1];
#pragma unroll
    for (int i = 0; i < K - 1; ++i) v[i] = Store<ST>::ld(V[i * g.plane_w + o]);
    int lab;
    if constexpr (std::is_same_v<ST, double>)
        lab = argmax_label_f64<K>(v);
    else
        lab = argmax_label<K>(v);
    if (res) res[oo] = pp.c[lab];
    if (labels) labels[oo] = (uint8_t)lab;
    if (V_out) {
#pragma unroll
        for (int i = 0; i < K - 1; ++i) V_out[i * plane_out + oo] = (OT)v[i];
    }
    if (Xi_out) {
#pragma unroll
        for (int j = 0; j < 3 * (K - 1); ++j) Xi_out[j * plane_out + oo] = (OT)Store<ST>::ld(xi[j * g.plane_w + o]);
    }
}

// ---------------------------------------------------------------------------
// FP64 energies of (V, Xi) over the slab: per voxel
//   e_i = lam (u - c_i)^2 - div Xi_i,  L += sum_i V_i e_i,  D += min_i e_i.
// One pair of partial sums per block; energy_finish adds them in block order.
// ---------------------------------------------------------------------------
template <int K, typename ST>
__global__ void __launch_bounds__(kPlainThreads) energy_kernel(Geometry g, const ST *__restrict__ xi,
                                                                const ST *__restrict__ V,
                                                                const float *__restrict__ u, PhaseParams<K> pp,
                                                                double2 *partial)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    double lag = 0.0, dual = 0.0;
    if (p.valid) {
        const LineInfo li = load_line(g, p.line);
        const int64_t o = p.line * g.nstride_w + p.n;
        const bool hn = p.n + 1 < g.ns, pn = p.n > 0;
        const bool hr = li.flags & kHasNextRow, pr = li.flags & kHasPrevRow;
        const bool hc = li.next_col >= 0, pc = li.prev_col >= 0;
        const int64_t opc = pc ? (int64_t)li.prev_col * g.nstride_w + p.n : o;
        const double uu = (double)u[p.line * g.nstride_in + g.slab_start + p.n];
        double xk0 = 0, xk1 = 0, xk2 = 0, xkn = 0, xkr = 0, xkc = 0, vk = 1, mn = 1.0e308;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            double x0, x1, x2, wn, wr, wc, vi;
            if (i < K - 1) {
                x0 = Store<ST>::ld(xi[(3 * i) * g.plane_w + o]);
                x1 = Store<ST>::ld(xi[(3 * i + 1) * g.plane_w + o]);
                x2 = Store<ST>::ld(xi[(3 * i + 2) * g.plane_w + o]);
                xk0 -= x0;
                xk1 -= x1;
                xk2 -= x2;
                wn = pn ? (double)Store<ST>::ld(xi[(3 * i) * g.plane_w + o - 1]) : 0.0;
                wr = pr ? (double)Store<ST>::ld(xi[(3 * i + 1) * g.plane_w + o - g.nstride_w]) : 0.0;
                wc = pc ? (double)Store<ST>::ld(xi[(3 * i + 2) * g.plane_w + opc]) : 0.0;
                xkn -= wn;
                xkr -= wr;
                xkc -= wc;
                vi = Store<ST>::ld(V[i * g.plane_w + o]);
                vk -= vi;
            } else {
                x0 = xk0;
                x1 = xk1;
                x2 = xk2;
                wn = xkn;
                wr = xkr;
                wc = xkc;
                vi = vk;
            }
            double div = 0.0;
            if (pn) div -= wn;
            if (hn) div += x0;
            if (pr) div -= wr;
            if (hr) div += x1;
            if (pc) div -= wc;
            if (hc) div += x2;
            const double dl = uu - (double)pp.c[i];
            const double e = (double)pp.lam * dl * dl - div;
            lag += vi * e;
            mn = e < mn ? e : mn;
        }
        dual = mn;
    }
    __shared__ double2 red[kPlainThreads / 32];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        lag += __shfl_xor_sync(0xffffffffu, lag, s);
        dual += __shfl_xor_sync(0xffffffffu, dual, s);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = make_double2(lag, dual);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = red[0];
        for (int w = 1; w < kPlainThreads / 32; ++w) {
            t.x += red[w].x;
            t.y += red[w].y;
        }
        partial[blockIdx.x] = t;
    }
}

// Adds the block partials in a fixed order (one block of 1024 threads: each
// thread a contiguous range, then a fixed tree), so the result is
// deterministic; writes (lagrangian, dual, gap) to out[0..2].
// (internal linkage: the header is included by several translation units)
static __global__ void __launch_bounds__(1024) energy_finish(const double2 *__restrict__ partial, int64_t count,
                                                      double *out)
{
    __shared__ double2 red[1024];
    const int64_t per = (count + 1023) / 1024;
    const int64_t b = threadIdx.x * per, e = b + per < count ? b + per : count;
    double2 t = make_double2(0.0, 0.0);
    for (int64_t i = b; i < e; ++i) {
        t.x += partial[i].x;
        t.y += partial[i].y;
    }
    red[threadIdx.x] = t;
    __syncthreads();
    for (int s = 512; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            red[threadIdx.x].x += red[threadIdx.x + s].x;
            red[threadIdx.x].y += red[threadIdx.x + s].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = red[0].x;
        out[1] = red[0].y;
        out[2] = red[0].x - red[0].y;
    }
}

}  // namespace potts
