// Per-voxel arithmetic of the "fast" FP32 form (potts_options.arith =
// POTTS_ARITH_FAST): the same iteration as voxel.cuh, with fewer operations.
// It is not bit-identical to the reference's operation order; it is held to
// the FP64 oracle instead (relative L2 of V within 1e-5, labels equal off
// ties, on the 128^3 case).  The differences from the exact form:
//   * terms of the K-th label are derived, not recomputed: div_K = -sum div_i,
//     q_K = -sum q_i (Xi_K = -sum Xi_i, so both identities hold exactly in
//     real arithmetic);
//   * a term for a missing neighbour is not masked where the state is zero
//     there by construction: Xi along an axis stays 0 at a voxel whose forward
//     neighbour along that axis is missing (its gradient is 0 and Dykstra's
//     corrections along that axis are 0), so the forward terms of the
//     divergence need no mask, and the backward terms along n and row read
//     such zeros (the line before a column's first line is the last line of
//     an earlier column; a missing slice reads 0).  Only the backward column
//     term keeps its mask.  Callers that cannot guarantee the zeros (the split
//     kernels) pass zeros for missing neighbours;
//   * the simplex threshold is theta = max_k (S_k - 1) / k over the sums S_k
//     of the k largest values (the sequence rises up to rho and falls after
//     it), for K = 2, 3 without sorting, with multiplications by constant
//     reciprocals;
//   * Dykstra's shrink (l - 1) h / l is h (1 - rsqrt(s)), s = |h|^2, and the
//     exit test sqrt(max |delta|^2) < 1e-6 is max |delta|^2 < 1e-12.
// Every function is written once for F = float (one voxel) and F = float2
// (two consecutive slices with Blackwell's paired FP32 instructions); the two
// lanes of a pair run exactly the operations of the scalar form, so the split
// (one voxel per thread) and fused (two per thread) fast forms give the same
// bits.
#pragma once

#include <cstdint>

namespace potts {
namespace fast {

__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub(float2 a, float2 b)
{
    uint64_t r;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(r)
        : "l"(*reinterpret_cast<const uint64_t *>(&a)), "l"(*reinterpret_cast<const uint64_t *>(&b)));
    return *reinterpret_cast<const float2 *>(&r);
}

template <typename F>
__device__ __forceinline__ F splat(float x);
template <>
__device__ __forceinline__ float splat<float>(float x) { return x; }
template <>
__device__ __forceinline__ float2 splat<float2>(float x) { return make_float2(x, x); }

// 1/k for k = 1..6 (k = 3, 5, 6 rounded; the threshold is not required to be
// the correctly rounded quotient in this form)
__device__ __forceinline__ constexpr float inv_k(int k)
{
    return k == 1 ? 1.0f : k == 2 ? 0.5f : k == 3 ? (1.0f / 3.0f) : k == 4 ? 0.25f : k == 5 ? 0.2f : (1.0f / 6.0f);
}

// Projection of one voxel's K values onto the simplex:
// q_i <- max(q_i - theta, 0), theta = max_k (S_k - 1) / k.
template <int K>
__device__ __forceinline__ void project_simplex(float (&q)[K])
{
    float theta;
    if constexpr (K == 2) {
        const float hi = fmaxf(q[0], q[1]);
        theta = fmaxf(sub(hi, 1.0f), fma(add(q[0], q[1]), 0.5f, -0.5f));
    } else if constexpr (K == 3) {
        const float hi = fmaxf(fmaxf(q[0], q[1]), q[2]);
        const float lo = fminf(fminf(q[0], q[1]), q[2]);
        const float t = add(add(q[0], q[1]), q[2]);
        const float t1 = sub(hi, 1.0f);
        const float t2 = fma(sub(t, lo), 0.5f, -0.5f);
        const float t3 = fma(t, inv_k(3), -inv_k(3));
        theta = fmaxf(t1, fmaxf(t2, t3));
    } else {
        float u[K];
#pragma unroll
        for (int i = 0; i < K; ++i) u[i] = q[i];
#pragma unroll
        for (int r = 0; r < K; ++r) {  // odd-even transposition sort, descending
#pragma unroll
            for (int i = (r & 1); i + 1 < K; i += 2) {
                const float a = u[i], b = u[i + 1];
                u[i] = fmaxf(a, b);
                u[i + 1] = fminf(a, b);
            }
        }
        float s = u[0];
        theta = sub(s, 1.0f);
#pragma unroll
        for (int k = 2; k <= K; ++k) {
            s = add(s, u[k - 1]);
            theta = fmaxf(theta, fma(s, inv_k(k), -inv_k(k)));
        }
    }
#pragma unroll
    for (int i = 0; i < K; ++i) q[i] = fmaxf(sub(q[i], theta), 0.0f);
}

// Primal step of one voxel (F = float) or of two consecutive slices
// (F = float2): q = Pi_S(V + tau1 (div- Xi - lam (u - c)^2)), Vbar = 2q - V;
// returns |q - V|^2 over all K labels.  xi[3 i + axis] at x, xin/xir/xic the
// n/row/col components at the backward neighbours (zero where the neighbour
// is missing along n and row, see above); mpc = -1 where the backward column
// neighbour exists, else -0.
template <int K, typename F>
__device__ __forceinline__ F primal(F (&vnew)[K - 1], F (&vbar)[K - 1], const F (&v)[K - 1],
                                   const F (&xi)[3 * (K - 1)], const F (&xin)[K - 1], const F (&xir)[K - 1],
                                   const F (&xic)[K - 1], F mpc, F u, const float (&c)[K], float lam, float tau1)
{
    F q[K], vv[K];
    F sdiv = splat<F>(0.0f), sv = splat<F>(0.0f);
    const F mlam = splat<F>(-lam), t1 = splat<F>(tau1);
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        const F div = add(add(sub(xi[3 * i], xin[i]), sub(xi[3 * i + 1], xir[i])), fma(mpc, xic[i], xi[3 * i + 2]));
        sdiv = i == 0 ? div : add(sdiv, div);
        sv = i == 0 ? v[i] : add(sv, v[i]);
        const F dl = sub(u, splat<F>(c[i]));
        q[i] = fma(t1, fma(mlam, mul(dl, dl), div), v[i]);
        vv[i] = v[i];
    }
    {  // the K-th label: V_K = 1 - sum V_i, div_K = -sum div_i
        const F vk = sub(splat<F>(1.0f), sv);
        const F dl = sub(u, splat<F>(c[K - 1]));
        q[K - 1] = fma(splat<F>(-tau1), fma(splat<F>(lam), mul(dl, dl), sdiv), vk);
        vv[K - 1] = vk;
    }
    if constexpr (sizeof(F) == 4) {
        project_simplex<K>(q);
    } else {
        float qa[K], qb[K];
#pragma unroll
        for (int i = 0; i < K; ++i) qa[i] = q[i].x, qb[i] = q[i].y;
        project_simplex<K>(qa);
        project_simplex<K>(qb);
#pragma unroll
        for (int i = 0; i < K; ++i) q[i] = make_float2(qa[i], qb[i]);
    }
    F dq;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const F e = sub(q[i], vv[i]);
        dq = i == 0 ? mul(e, e) : fma(e, e, dq);
    }
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        vnew[i] = q[i];
        vbar[i] = sub(add(q[i], q[i]), vv[i]);
    }
    return dq;
}

// q = Xi + tau2 grad+(Vbar) of one voxel or a pair: t2n / t2r / t2c are tau2
// where the forward neighbour along n / row / col exists, else 0; q_K is
// -sum q_i.
template <int K, typename F>
__device__ __forceinline__ void dual_q(F (&q)[K][3], const F (&xi)[3 * (K - 1)], const F (&vb)[K - 1],
                                       const F (&vbn)[K - 1], const F (&vbr)[K - 1], const F (&vbc)[K - 1], F t2n,
                                       F t2r, F t2c)
{
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        q[i][0] = fma(sub(vbn[i], vb[i]), t2n, xi[3 * i]);
        q[i][1] = fma(sub(vbr[i], vb[i]), t2r, xi[3 * i + 1]);
        q[i][2] = fma(sub(vbc[i], vb[i]), t2c, xi[3 * i + 2]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        F s = q[0][a];
#pragma unroll
        for (int i = 1; i < K - 1; ++i) s = add(s, q[i][a]);
        q[K - 1][a] = sub(splat<F>(0.0f), s);
    }
}

// Largest |q_i - q_j|^2 over the pairs (the projection loop is needed only
// where it exceeds 1: otherwise Dykstra's first sweep is the identity).
template <int K, typename F>
__device__ __forceinline__ F max_pair_dist2(const F (&q)[K][3])
{
    F m;
    int p = 0;
#pragma unroll
    for (int i1 = 0; i1 < K - 1; ++i1) {
#pragma unroll
        for (int i2 = i1 + 1; i2 < K; ++i2, ++p) {
            const F a0 = sub(q[i2][0], q[i1][0]), a1 = sub(q[i2][1], q[i1][1]), a2 = sub(q[i2][2], q[i1][2]);
            const F s = fma(a2, a2, fma(a1, a1, mul(a0, a0)));
            if constexpr (sizeof(F) == 4)
                m = p == 0 ? s : fmaxf(m, s);
            else
                m = p == 0 ? s : make_float2(fmaxf(m.x, s.x), fmaxf(m.y, s.y));
        }
    }
    return m;
}

// One sweep of Dykstra's loop over the pairs (i1 < i2); true when the loop
// exits after it (every correction step shorter than 1e-6).
template <int K>
__device__ __forceinline__ bool dykstra_sweep(float (&q)[K][3], float (&P)[K * (K - 1) / 2][3])
{
    float max_dd = 0.0f;
    int p = 0;
#pragma unroll
    for (int i1 = 0; i1 < K - 1; ++i1) {
#pragma unroll
        for (int i2 = i1 + 1; i2 < K; ++i2, ++p) {
            const float h0 = add(sub(q[i2][0], q[i1][0]), P[p][0]);
            const float h1 = add(sub(q[i2][1], q[i1][1]), P[p][1]);
            const float h2 = add(sub(q[i2][2], q[i1][2]), P[p][2]);
            const float s = fma(h2, h2, fma(h1, h1, mul(h0, h0)));
            const float f = s > 1.0f ? sub(1.0f, rsqrtf(s)) : 0.0f;
            const float n0 = mul(h0, f), n1 = mul(h1, f), n2 = mul(h2, f);
            const float d0 = mul(0.5f, sub(n0, P[p][0]));
            const float d1 = mul(0.5f, sub(n1, P[p][1]));
            const float d2 = mul(0.5f, sub(n2, P[p][2]));
            max_dd = fmaxf(max_dd, fma(d2, d2, fma(d1, d1, mul(d0, d0))));
            q[i1][0] = add(q[i1][0], d0);
            q[i1][1] = add(q[i1][1], d1);
            q[i1][2] = add(q[i1][2], d2);
            q[i2][0] = sub(q[i2][0], d0);
            q[i2][1] = sub(q[i2][1], d1);
            q[i2][2] = sub(q[i2][2], d2);
            P[p][0] = n0;
            P[p][1] = n1;
            P[p][2] = n2;
        }
    }
    return max_dd < 1e-12f;
}

// The whole projection loop from zero corrections (at most 20 sweeps).
template <int K>
__device__ __forceinline__ void dual_project(float (&q)[K][3])
{
    constexpr int kPairs = K * (K - 1) / 2;
    float P[kPairs][3];
#pragma unroll
    for (int p = 0; p < kPairs; ++p) P[p][0] = P[p][1] = P[p][2] = 0.0f;
    for (int sweeps = 1; sweeps <= 20; ++sweeps)
        if (dykstra_sweep<K>(q, P)) break;
}

}  // namespace fast
}  // namespace potts
