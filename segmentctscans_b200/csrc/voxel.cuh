// Per-voxel arithmetic of the Potts primal-dual iteration, shared by every
// kernel of the library (split and fused forms), so that all forms produce the
// same bits.
//
// The translation unit is compiled with -fmad=false: no multiply-add is fused
// unless written as fmaf() here, every + - * / sqrt is an IEEE single
// operation in round-to-nearest, and the order of operations is the order in
// the source.  The places where fmaf() appears are the places where the
// reference's clang build contracts a multiply and an add.
#pragma once

#include <cstdint>

namespace potts {

constexpr int kMaxPhases = 6;

// Thresholds that let the Dykstra loop decide `sqrt(s) > 1` and
// `(double)sqrt(m) < 1e-6` without computing the square root.  Both
// predicates are monotone in s (resp. m) because IEEE sqrt is, so each is a
// comparison with one float, found by bisection on the host.
struct DykstraThresholds {
    float len_gt_one;  // sqrt(s) > 1      <=>  s > len_gt_one
    float exit_below;  // sqrt(m) < 1e-6   <=>  m < exit_below
};

__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }

// ---------------------------------------------------------------------------
// Dual step at one voxel (potts-model/potts-min-partition.cpp:96-247):
//   q = Xi + tau2 * grad+(Vbar), then Dykstra projection onto
//   K = {|q_i - q_j| <= 1 for all i < j} with at most 20 sweeps.
// It is split in three parts so that the tiled kernel can gather the voxels
// that need the full projection loop before running it:
//   dual_build_q      q from Xi and Vbar at x and its forward neighbours
//   dual_first_sweep_is_identity
//                     true when the first sweep changes nothing (no pair is
//                     longer than 1: every correction is zero, max|delta| = 0
//                     and the loop exits after one sweep)
//   dual_project      the full loop (from zero corrections); returns sweeps
// xi[3*i + axis] holds the stored K-1 labels; vb* are Vbar at x and at the
// forward neighbours along n, row, col; h* say whether that neighbour exists.
// ---------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void dual_build_q(float (&q)[K][3], const float (&xi)[3 * (K - 1)],
                                             const float (&vb)[K - 1], const float (&vbn)[K - 1],
                                             const float (&vbr)[K - 1], const float (&vbc)[K - 1], bool hn, bool hr,
                                             bool hc, float tau2)
{
    float vk = 1.0f, vkn = 1.0f, vkr = 1.0f, vkc = 1.0f;
    float xk0 = 0.0f, xk1 = 0.0f, xk2 = 0.0f;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        float vi, wn, wr, wc, x0, x1, x2;
        if (i < K - 1) {
            vi = vb[i];
            vk = vk - vi;
            wn = vbn[i];
            vkn = vkn - wn;
            wr = vbr[i];
            vkr = vkr - wr;
            wc = vbc[i];
            vkc = vkc - wc;
            x0 = xi[3 * i];
            x1 = xi[3 * i + 1];
            x2 = xi[3 * i + 2];
            xk0 = xk0 - x0;
            xk1 = xk1 - x1;
            xk2 = xk2 - x2;
        } else {
            vi = vk;
            wn = vkn;
            wr = vkr;
            wc = vkc;
            x0 = xk0;
            x1 = xk1;
            x2 = xk2;
        }
        const float g0 = hn ? (wn - vi) : 0.0f;
        const float g1 = hr ? (wr - vi) : 0.0f;
        const float g2 = hc ? (wc - vi) : 0.0f;
        q[i][0] = fmaf(g0, tau2, x0);
        q[i][1] = fmaf(g1, tau2, x1);
        q[i][2] = fmaf(g2, tau2, x2);
    }
}

template <int K>
__device__ __forceinline__ bool dual_first_sweep_is_identity(const float (&q)[K][3], DykstraThresholds thr)
{
    bool any_long = false;
#pragma unroll
    for (int i1 = 0; i1 < K - 1; ++i1) {
#pragma unroll
        for (int i2 = i1 + 1; i2 < K; ++i2) {
            const float a0 = q[i2][0] - q[i1][0];
            const float a1 = q[i2][1] - q[i1][1];
            const float a2 = q[i2][2] - q[i1][2];
            float s = a0 * a0;
            s = fmaf(a1, a1, s);
            s = fmaf(a2, a2, s);
            any_long |= (s > thr.len_gt_one);
        }
    }
    return !any_long;
}

template <int K>
__device__ __forceinline__ int dual_project(float (&q)[K][3], DykstraThresholds thr)
{
    constexpr int kPairs = K * (K - 1) / 2;
    float P[kPairs][3];
#pragma unroll
    for (int p = 0; p < kPairs; ++p) P[p][0] = P[p][1] = P[p][2] = 0.0f;
    int sweeps;
    for (sweeps = 1; sweeps <= 20; ++sweeps) {
        float max_dd = 0.0f;
        int p = 0;
#pragma unroll
        for (int i1 = 0; i1 < K - 1; ++i1) {
#pragma unroll
            for (int i2 = i1 + 1; i2 < K; ++i2, ++p) {
                const float h0 = (q[i2][0] - q[i1][0]) + P[p][0];
                const float h1 = (q[i2][1] - q[i1][1]) + P[p][1];
                const float h2 = (q[i2][2] - q[i1][2]) + P[p][2];
                float s = h0 * h0;
                s = fmaf(h1, h1, s);
                s = fmaf(h2, h2, s);
                float n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
                if (s > thr.len_gt_one) {
                    const float l = __fsqrt_rn(s);
                    const float lm1 = l - 1.0f;
                    n0 = __fdiv_rn(lm1 * h0, l);
                    n1 = __fdiv_rn(lm1 * h1, l);
                    n2 = __fdiv_rn(lm1 * h2, l);
                }
                const float d0 = 0.5f * (n0 - P[p][0]);
                const float d1 = 0.5f * (n1 - P[p][1]);
                const float d2 = 0.5f * (n2 - P[p][2]);
                float dd = d0 * d0;
                dd = fmaf(d1, d1, dd);
                dd = fmaf(d2, d2, dd);
                max_dd = fmax_ref(dd, max_dd);
                q[i1][0] = q[i1][0] + d0;
                q[i1][1] = q[i1][1] + d1;
                q[i1][2] = q[i1][2] + d2;
                q[i2][0] = q[i2][0] - d0;
                q[i2][1] = q[i2][1] - d1;
                q[i2][2] = q[i2][2] - d2;
                P[p][0] = n0;
                P[p][1] = n1;
                P[p][2] = n2;
            }
        }
        if (max_dd < thr.exit_below) break;
    }
    return sweeps > 20 ? 20 : sweeps;
}

template <int K>
__device__ __forceinline__ void dual_store(float (&xo)[3 * (K - 1)], const float (&q)[K][3])
{
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        xo[3 * i] = q[i][0];
        xo[3 * i + 1] = q[i][1];
        xo[3 * i + 2] = q[i][2];
    }
}

// The whole dual step at one voxel; returns the number of sweeps.
template <int K>
__device__ __forceinline__ int dual_voxel(float (&xo)[3 * (K - 1)], const float (&xi)[3 * (K - 1)],
                                          const float (&vb)[K - 1], const float (&vbn)[K - 1],
                                          const float (&vbr)[K - 1], const float (&vbc)[K - 1], bool hn, bool hr,
                                          bool hc, float tau2, DykstraThresholds thr)
{
    float q[K][3];
    dual_build_q<K>(q, xi, vb, vbn, vbr, vbc, hn, hr, hc, tau2);
    int sweeps = 1;
    if (!dual_first_sweep_is_identity<K>(q, thr)) sweeps = dual_project<K>(q, thr);
    dual_store<K>(xo, q);
    return sweeps;
}

// Compare-exchange putting the larger value first.
__device__ __forceinline__ void cx_desc(float &a, float &b)
{
    const float x = a, y = b;
    a = fmaxf(x, y);
    b = fminf(x, y);
}

// Descending sort of K values.  Any correct sort gives the same sorted values,
// so these small networks need not match the reference's.
template <int K>
__device__ __forceinline__ void sort_desc(float (&u)[K])
{
    if constexpr (K == 2) {
        cx_desc(u[0], u[1]);
    } else if constexpr (K == 3) {
        cx_desc(u[0], u[1]);
        cx_desc(u[1], u[2]);
        cx_desc(u[0], u[1]);
    } else if constexpr (K == 4) {
        cx_desc(u[0], u[1]);
        cx_desc(u[2], u[3]);
        cx_desc(u[0], u[2]);
        cx_desc(u[1], u[3]);
        cx_desc(u[1], u[2]);
    } else {
        // odd-even transposition sort: K rounds
#pragma unroll
        for (int r = 0; r < K; ++r) {
#pragma unroll
            for (int i = (r & 1); i + 1 < K; i += 2) cx_desc(u[i], u[i + 1]);
        }
    }
}

// x / j for a small positive integer j, correctly rounded.  Division by a
// power of two equals multiplication by its reciprocal exactly.
__device__ __forceinline__ float div_small(float x, int j)
{
    switch (j) {
    case 1: return x;
    case 2: return x * 0.5f;
    case 4: return x * 0.25f;
    default: return __fdiv_rn(x, (float)j);
    }
}

// Projection onto the simplex (potts-model/potts-min-partition.cpp:292-347).
template <int K>
__device__ __forceinline__ void project_simplex(float (&q)[K])
{
    float u[K];
#pragma unroll
    for (int i = 0; i < K; ++i) u[i] = q[i];
    sort_desc<K>(u);
    float sum = 0.0f, rho_sum = 0.0f;
    int rho = 0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        sum = sum + u[i];
        const float theta = div_small(sum - 1.0f, i + 1);
        if (u[i] > theta) {
            rho = i + 1;
            rho_sum = sum;
        }
    }
    const float theta = div_small(rho_sum - 1.0f, rho);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const float t = q[i] - theta;
        q[i] = (t < 0.0f) ? 0.0f : t;
    }
}

// ---------------------------------------------------------------------------
// Primal step at one voxel (potts-model/potts-min-partition.cpp:381-480):
//   q = Pi_S(V + tau1 * (div- Xi - lam (u - c)^2)),  Vbar = 2q - V.
// xi are the stored components at x; xin/xir/xic the n/row/col components of
// the backward neighbours; p*/h* say whether the backward/forward neighbour
// exists.  Returns |q - V|^2 over all K labels.
// ---------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ float primal_voxel(float (&vnew)[K - 1], float (&vbar)[K - 1], const float (&v)[K - 1],
                                              const float (&xi)[3 * (K - 1)], const float (&xin)[K - 1],
                                              const float (&xir)[K - 1], const float (&xic)[K - 1], bool pn,
                                              bool hn, bool pr, bool hr, bool pc, bool hc, float u,
                                              const float (&c)[K], float lam, float tau1)
{
    float q[K], vv[K];
    float vk = 1.0f;
    float xk0 = 0.0f, xk1 = 0.0f, xk2 = 0.0f, xkn = 0.0f, xkr = 0.0f, xkc = 0.0f;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        float x0, x1, x2, wn, wr, wc, vi;
        if (i < K - 1) {
            x0 = xi[3 * i];
            x1 = xi[3 * i + 1];
            x2 = xi[3 * i + 2];
            xk0 = xk0 - x0;
            xk1 = xk1 - x1;
            xk2 = xk2 - x2;
            wn = xin[i];
            xkn = xkn - wn;
            wr = xir[i];
            xkr = xkr - wr;
            wc = xic[i];
            xkc = xkc - wc;
            vi = v[i];
            vk = vk - vi;
        } else {
            x0 = xk0;
            x1 = xk1;
            x2 = xk2;
            wn = xkn;
            wr = xkr;
            wc = xkc;
            vi = vk;
        }
        float div = 0.0f;
        if (pn) div = div - wn;
        if (hn) div = div + x0;
        if (pr) div = div - wr;
        if (hr) div = div + x1;
        if (pc) div = div - wc;
        if (hc) div = div + x2;
        vv[i] = vi;
        const float dl = u - c[i];
        const float d2 = dl * dl;
        const float w = fmaf(-lam, d2, div);
        q[i] = fmaf(tau1, w, vi);
    }
    project_simplex<K>(q);
    float dq = 0.0f;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const float e = q[i] - vv[i];
        dq = (i == 0) ? e * e : fmaf(e, e, dq);
    }
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        vnew[i] = q[i];
        vbar[i] = 2.0f * q[i] - vv[i];
    }
    return dq;
}

// init_v_kernel (potts-model/potts-min-partition.cpp:56-94): index of the
// label nearest to u (strict <, the first of equals wins).
template <int K>
__device__ __forceinline__ int nearest_label(float u, const float (&c)[K])
{
    float best = 3.402823466e+38f;
    int cluster = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const float d = fabsf(c[k] - u);
        if (d < best) {
            best = d;
            cluster = k;
        }
    }
    return cluster;
}

// update_kernel (potts-model/potts-min-partition.cpp:491-538): argmax with
// strict >, starting from 0, so the first of equal maxima wins.
template <int K>
__device__ __forceinline__ int argmax_label(const float (&v)[K - 1])
{
    float best = 0.0f, vk = 1.0f;
    int lab = 0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        float vi;
        if (i < K - 1) {
            vi = v[i];
            vk = vk - vi;
        } else {
            vi = vk;
        }
        if (vi > best) {
            best = vi;
            lab = i;
        }
    }
    return lab;
}

}  // namespace potts
