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
    const float fhn = hn ? 1.0f : 0.0f, fhr = hr ? 1.0f : 0.0f, fhc = hc ? 1.0f : 0.0f;
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
        // the difference to a missing neighbour is multiplied by 0 (its value
        // must be finite), which equals the reference's skipped term
        const float g0 = fhn * (wn - vi);
        const float g1 = fhr * (wr - vi);
        const float g2 = fhc * (wc - vi);
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

// One sweep of Dykstra's loop over the pairs (i1 < i2) with corrections P;
// true when the loop exits after it (every step shorter than 1e-6).
template <int K>
__device__ __forceinline__ bool dykstra_sweep(float (&q)[K][3], float (&P)[K * (K - 1) / 2][3],
                                              DykstraThresholds thr)
{
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
    return max_dd < thr.exit_below;
}

template <int K>
__device__ __forceinline__ int dual_project(float (&q)[K][3], DykstraThresholds thr)
{
    constexpr int kPairs = K * (K - 1) / 2;
    float P[kPairs][3];
#pragma unroll
    for (int p = 0; p < kPairs; ++p) P[p][0] = P[p][1] = P[p][2] = 0.0f;
    int sweeps;
    for (sweeps = 1; sweeps <= 20; ++sweeps)
        if (dykstra_sweep<K>(q, P, thr)) break;
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

// u > RN(x / j) for j in 1..6, without a division in the common case.
// t = fma(j, u, -x) carries the exact sign of j*u - x.  When |t| exceeds
// max(|u| 2^-19, 2^-120), |u - x/j| is larger than the spacing of floats
// around u, so RN(x/j) lies strictly on the same side of u as x/j and the sign
// of t decides; otherwise the quotient is computed and compared.
__device__ __forceinline__ bool gt_div_small(float u, float x, int j)
{
    if (j == 1 || j == 2 || j == 4) return u > div_small(x, j);
    const float t = fmaf((float)j, u, -x);
    const float margin = fmaxf(fabsf(u) * 0x1p-19f, 0x1p-120f);
    if (fabsf(t) > margin) return t > 0.0f;
    return u > __fdiv_rn(x, (float)j);
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
        if (gt_div_small(u[i], sum - 1.0f, i + 1)) {  // u[i] > (sum - 1) / (i + 1)
            rho = i + 1;
            rho_sum = sum;
        }
    }
    const float theta = div_small(rho_sum - 1.0f, rho);
#pragma unroll
    for (int i = 0; i < K; ++i) q[i] = fmaxf(q[i] - theta, 0.0f);  // max(q - theta, 0); -0 vs +0 aside
}

// ---------------------------------------------------------------------------
// Primal step at one voxel (potts-model/potts-min-partition.cpp:381-480):
//   q = Pi_S(V + tau1 * (div- Xi - lam (u - c)^2)),  Vbar = 2q - V.
// xi are the stored components at x; xin/xir/xic the n/row/col components of
// the backward neighbours; p*/h* say whether the backward/forward neighbour
// exists.  Returns |q - V|^2 over all K labels.
// ---------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void primal_q(float (&q)[K], float (&vv)[K], const float (&v)[K - 1],
                                         const float (&xi)[3 * (K - 1)], const float (&xin)[K - 1],
                                         const float (&xir)[K - 1], const float (&xic)[K - 1], bool pn, bool hn,
                                         bool pr, bool hr, bool pc, bool hc, float u, const float (&c)[K], float lam,
                                         float tau1)
{
    float vk = 1.0f;
    float xk0 = 0.0f, xk1 = 0.0f, xk2 = 0.0f, xkn = 0.0f, xkr = 0.0f, xkc = 0.0f;
    const float fpn = pn ? 1.0f : 0.0f, fhn = hn ? 1.0f : 0.0f, fpr = pr ? 1.0f : 0.0f;
    const float fhr = hr ? 1.0f : 0.0f, fpc = pc ? 1.0f : 0.0f, fhc = hc ? 1.0f : 0.0f;
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
        // div = 0; div -= wn if pn; div += x0 if hn; ... in this order.  A term
        // whose neighbour is missing is multiplied by 0 instead of skipped,
        // which gives the same value as long as the skipped operand is finite
        // (callers pass 0 or finite stale state for missing neighbours).
        float div = fmaf(-fpn, wn, 0.0f);
        div = fmaf(fhn, x0, div);
        div = fmaf(-fpr, wr, div);
        div = fmaf(fhr, x1, div);
        div = fmaf(-fpc, wc, div);
        div = fmaf(fhc, x2, div);
        vv[i] = vi;
        const float dl = u - c[i];
        const float d2 = dl * dl;
        const float w = fmaf(-lam, d2, div);
        q[i] = fmaf(tau1, w, vi);
    }
}

template <int K>
__device__ __forceinline__ float primal_voxel(float (&vnew)[K - 1], float (&vbar)[K - 1], const float (&v)[K - 1],
                                              const float (&xi)[3 * (K - 1)], const float (&xin)[K - 1],
                                              const float (&xir)[K - 1], const float (&xic)[K - 1], bool pn,
                                              bool hn, bool pr, bool hr, bool pc, bool hc, float u,
                                              const float (&c)[K], float lam, float tau1)
{
    float q[K], vv[K];
    primal_q<K>(q, vv, v, xi, xin, xir, xic, pn, hn, pr, hr, pc, hc, u, c, lam, tau1);
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

// ---------------------------------------------------------------------------
// Two voxels at once (consecutive slices of one line) with Blackwell's paired
// FP32 instructions.  Each lane of a pair goes through exactly the operations
// of primal_voxel / dual_build_q / dual_first_sweep_is_identity above, in the
// same order and with the same rounding, so the results are the same bits.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <int K>
__device__ __forceinline__ void dual_build_q_pair(float2 (&q)[K][3], const float2 (&xi)[3 * (K - 1)],
                                                  const float2 (&vb)[K - 1], const float2 (&vbn)[K - 1],
                                                  const float2 (&vbr)[K - 1], const float2 (&vbc)[K - 1], float2 fhn,
                                                  float2 fhr, float2 fhc, float tau2)
{
    float2 vk = f2(1.0f), vkn = f2(1.0f), vkr = f2(1.0f), vkc = f2(1.0f);
    float2 xk0 = f2(0.0f), xk1 = f2(0.0f), xk2 = f2(0.0f);
    const float2 t2 = f2(tau2);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        float2 vi, wn, wr, wc, x0, x1, x2;
        if (i < K - 1) {
            vi = vb[i];
            vk = sub2(vk, vi);
            wn = vbn[i];
            vkn = sub2(vkn, wn);
            wr = vbr[i];
            vkr = sub2(vkr, wr);
            wc = vbc[i];
            vkc = sub2(vkc, wc);
            x0 = xi[3 * i];
            x1 = xi[3 * i + 1];
            x2 = xi[3 * i + 2];
            xk0 = sub2(xk0, x0);
            xk1 = sub2(xk1, x1);
            xk2 = sub2(xk2, x2);
        } else {
            vi = vk;
            wn = vkn;
            wr = vkr;
            wc = vkc;
            x0 = xk0;
            x1 = xk1;
            x2 = xk2;
        }
        q[i][0] = fma2(mul2(fhn, sub2(wn, vi)), t2, x0);
        q[i][1] = fma2(mul2(fhr, sub2(wr, vi)), t2, x1);
        q[i][2] = fma2(mul2(fhc, sub2(wc, vi)), t2, x2);
    }
}

// bit j set: the first sweep of voxel j is not the identity (see
// dual_first_sweep_is_identity)
template <int K>
__device__ __forceinline__ unsigned dual_needs_loop_pair(const float2 (&q)[K][3], DykstraThresholds thr)
{
    bool l0 = false, l1 = false;
#pragma unroll
    for (int i1 = 0; i1 < K - 1; ++i1) {
#pragma unroll
        for (int i2 = i1 + 1; i2 < K; ++i2) {
            const float2 a0 = sub2(q[i2][0], q[i1][0]);
            const float2 a1 = sub2(q[i2][1], q[i1][1]);
            const float2 a2 = sub2(q[i2][2], q[i1][2]);
            float2 s = mul2(a0, a0);
            s = fma2(a1, a1, s);
            s = fma2(a2, a2, s);
            l0 |= (s.x > thr.len_gt_one);
            l1 |= (s.y > thr.len_gt_one);
        }
    }
    return (l0 ? 1u : 0u) | (l1 ? 2u : 0u);
}

template <int K>
__device__ __forceinline__ float2 primal_pair(float2 (&vnew)[K - 1], float2 (&vbar)[K - 1],
                                              const float2 (&v)[K - 1], const float2 (&xi)[3 * (K - 1)],
                                              const float2 (&xin)[K - 1], const float2 (&xir)[K - 1],
                                              const float2 (&xic)[K - 1], float2 fpn, float2 fhn, float2 fpr,
                                              float2 fhr, float2 fpc, float2 fhc, float2 u, const float (&c)[K],
                                              float lam, float tau1)
{
    float2 q[K], vv[K];
    float2 vk = f2(1.0f);
    float2 xk0 = f2(0.0f), xk1 = f2(0.0f), xk2 = f2(0.0f), xkn = f2(0.0f), xkr = f2(0.0f), xkc = f2(0.0f);
    const float2 mfpn = f2(-fpn.x, -fpn.y), mfpr = f2(-fpr.x, -fpr.y), mfpc = f2(-fpc.x, -fpc.y);
    const float2 mlam = f2(-lam), t1 = f2(tau1);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        float2 x0, x1, x2, wn, wr, wc, vi;
        if (i < K - 1) {
            x0 = xi[3 * i];
            x1 = xi[3 * i + 1];
            x2 = xi[3 * i + 2];
            xk0 = sub2(xk0, x0);
            xk1 = sub2(xk1, x1);
            xk2 = sub2(xk2, x2);
            wn = xin[i];
            xkn = sub2(xkn, wn);
            wr = xir[i];
            xkr = sub2(xkr, wr);
            wc = xic[i];
            xkc = sub2(xkc, wc);
            vi = v[i];
            vk = sub2(vk, vi);
        } else {
            x0 = xk0;
            x1 = xk1;
            x2 = xk2;
            wn = xkn;
            wr = xkr;
            wc = xkc;
            vi = vk;
        }
        float2 div = fma2(mfpn, wn, f2(0.0f));
        div = fma2(fhn, x0, div);
        div = fma2(mfpr, wr, div);
        div = fma2(fhr, x1, div);
        div = fma2(mfpc, wc, div);
        div = fma2(fhc, x2, div);
        vv[i] = vi;
        const float2 dl = sub2(u, f2(c[i]));
        const float2 d2 = mul2(dl, dl);
        const float2 w = fma2(mlam, d2, div);
        q[i] = fma2(t1, w, vi);
    }
    // simplex projection of each voxel (the sort and the threshold search are
    // per voxel; the final shift is paired)
    float qa[K], qb[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        qa[i] = q[i].x;
        qb[i] = q[i].y;
    }
    project_simplex<K>(qa);
    project_simplex<K>(qb);
#pragma unroll
    for (int i = 0; i < K; ++i) q[i] = f2(qa[i], qb[i]);
    float2 dq = f2(0.0f);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const float2 e = sub2(q[i], vv[i]);
        dq = (i == 0) ? mul2(e, e) : fma2(e, e, dq);
    }
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        vnew[i] = q[i];
        vbar[i] = sub2(mul2(f2(2.0f), q[i]), vv[i]);
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
