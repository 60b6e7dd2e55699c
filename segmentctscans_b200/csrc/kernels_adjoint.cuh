// Reverse mode of the unrolled primal-dual iteration (split form, FP32 state).
//
// Forward iteration k (state k -> k+1), per voxel with the K-th label implicit:
//   dual:    Xi^{k+1} = Pi_K(p),  p = E(Xi^k) + tau2 grad+ E(Vbar^k)
//   primal:  V^{k+1}  = Pi_S(q),  q = E(V^k) + tau1 (div- E(Xi^{k+1}) - lam (u - c)^2)
//            Vbar^{k+1} = 2 V^{k+1} - V^k
// where E adds the implicit label (V_K = 1 - sum V_i, Xi_K = -sum Xi_i).  The
// adjoints kept between steps are those of the stored K-1 components
// ("reduced"); a full K-label adjoint a maps to the reduced one by
// E^T a = a_i - a_K, and the adjoint of a projection's output is (reduced, 0)
// because only its first K-1 components are stored.
//
// Backward step k, given A = dL/dV^{k+1}, B = dL/dVbar^{k+1}, X = dL/dXi^{k+1}:
//   adj_primal_kernel:  qbar = J_S(q)^T (A + 2B, 0);  A <- E^T qbar - B;
//                       u, lambda, c gradients from qbar (the data term);
//                       Qbar <- qbar.  B itself is tau2 E^T grad+^T pbar of
//                       the step after (grad+^T = -div-, same masks), read
//                       from Pbar.
//   adj_dual_kernel:    Xtot = X + tau1 E^T div-^T qbar (div-^T = -grad+);
//                       pbar = J_K(p)^T (Xtot, 0);  X <- E^T pbar;  Pbar <- pbar.
// J_S: on the active set A of the simplex projection, a_i - mean_A(a), else 0.
// J_K: Dykstra's loop replayed with every pair step's vector h recorded, then
// run backwards (the numbers of sweeps and the branches are those of the
// forward pass).
#pragma once

#include <cstdint>

#include "geometry.cuh"
#include "kernels_plain.cuh"
#include "voxel.cuh"

namespace potts {

// pbar = J^T ybar for the Dykstra projection at p (the loop of dykstra_sweep).
template <int K>
__device__ void dykstra_vjp(const float (&p)[K][3], const float (&ybar)[K][3], float (&pbar)[K][3],
                            DykstraThresholds thr)
{
    constexpr int kPairs = K * (K - 1) / 2;
    float q[K][3], P[kPairs][3];
    float tape[20][kPairs][3];
#pragma unroll
    for (int i = 0; i < K; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) q[i][a] = p[i][a];
#pragma unroll
    for (int k = 0; k < kPairs; ++k) P[k][0] = P[k][1] = P[k][2] = 0.0f;
    int sweeps = 0;
    for (int s = 0; s < 20; ++s) {
        float max_dd = 0.0f;
        int k = 0;
#pragma unroll
        for (int i1 = 0; i1 < K - 1; ++i1) {
#pragma unroll
            for (int i2 = i1 + 1; i2 < K; ++i2, ++k) {
                const float h0 = (q[i2][0] - q[i1][0]) + P[k][0];
                const float h1 = (q[i2][1] - q[i1][1]) + P[k][1];
                const float h2 = (q[i2][2] - q[i1][2]) + P[k][2];
                tape[s][k][0] = h0;
                tape[s][k][1] = h1;
                tape[s][k][2] = h2;
                float sq = h0 * h0;
                sq = fmaf(h1, h1, sq);
                sq = fmaf(h2, h2, sq);
                float n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
                if (sq > thr.len_gt_one) {
                    const float l = __fsqrt_rn(sq);
                    const float lm1 = l - 1.0f;
                    n0 = __fdiv_rn(lm1 * h0, l);
                    n1 = __fdiv_rn(lm1 * h1, l);
                    n2 = __fdiv_rn(lm1 * h2, l);
                }
                const float d0 = 0.5f * (n0 - P[k][0]);
                const float d1 = 0.5f * (n1 - P[k][1]);
                const float d2 = 0.5f * (n2 - P[k][2]);
                float dd = d0 * d0;
                dd = fmaf(d1, d1, dd);
                dd = fmaf(d2, d2, dd);
                max_dd = fmax_ref(dd, max_dd);
                q[i1][0] += d0, q[i1][1] += d1, q[i1][2] += d2;
                q[i2][0] -= d0, q[i2][1] -= d1, q[i2][2] -= d2;
                P[k][0] = n0, P[k][1] = n1, P[k][2] = n2;
            }
        }
        sweeps = s + 1;
        if (max_dd < thr.exit_below) break;
    }
    // backwards: qb = adjoint of q, Pb = adjoint of each pair's correction
    float qb[K][3], Pb[kPairs][3];
#pragma unroll
    for (int i = 0; i < K; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) qb[i][a] = ybar[i][a];
#pragma unroll
    for (int k = 0; k < kPairs; ++k) Pb[k][0] = Pb[k][1] = Pb[k][2] = 0.0f;
    for (int s = sweeps - 1; s >= 0; --s) {
        int k = kPairs - 1;
#pragma unroll
        for (int i1 = K - 2; i1 >= 0; --i1) {
#pragma unroll
            for (int i2 = K - 1; i2 > i1; --i2, --k) {
                const float h[3] = {tape[s][k][0], tape[s][k][1], tape[s][k][2]};
                float db[3], nb[3], hb[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    db[a] = qb[i1][a] - qb[i2][a];  // d enters q_i1 with +, q_i2 with -
                    nb[a] = Pb[k][a] + 0.5f * db[a];
                    Pb[k][a] = -0.5f * db[a];       // the correction before this step
                }
                float sq = h[0] * h[0];
                sq = fmaf(h[1], h[1], sq);
                sq = fmaf(h[2], h[2], sq);
                if (sq > thr.len_gt_one) {
                    // n = (1 - 1/l) h:  dn/dh = (1 - 1/l) I + h h^T / l^3
                    const float l = sqrtf(sq);
                    const float il = 1.0f / l;
                    const float hn = h[0] * nb[0] + h[1] * nb[1] + h[2] * nb[2];
#pragma unroll
                    for (int a = 0; a < 3; ++a) hb[a] = (1.0f - il) * nb[a] + hn * il * il * il * h[a];
                } else {
                    hb[0] = hb[1] = hb[2] = 0.0f;
                }
#pragma unroll
                for (int a = 0; a < 3; ++a) {  // h = q_i2 - q_i1 + P
                    qb[i2][a] += hb[a];
                    qb[i1][a] -= hb[a];
                    Pb[k][a] += hb[a];
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < K; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) pbar[i][a] = qb[i][a];
}

// qbar = J^T abar for the simplex projection at q.
template <int K>
__device__ __forceinline__ void simplex_vjp(const float (&q)[K], const float (&abar)[K], float (&qbar)[K])
{
    float pr[K];
#pragma unroll
    for (int i = 0; i < K; ++i) pr[i] = q[i];
    project_simplex<K>(pr);
    int cnt = 0;
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < K; ++i)
        if (pr[i] > 0.0f) {
            ++cnt;
            sum += abar[i];
        }
    const float mean = cnt > 0 ? sum / (float)cnt : 0.0f;
#pragma unroll
    for (int i = 0; i < K; ++i) qbar[i] = pr[i] > 0.0f ? abar[i] - mean : 0.0f;
}

// Block sums of up to 8 doubles, then one atomicAdd each into dst.
template <int N>
__device__ __forceinline__ void block_sum_to(double (&v)[N], double *dst)
{
    __shared__ double red[N][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < N; ++j) {
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], s);
        if (lane == 0) red[j][warp] = v[j];
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            double x = lane < nw ? red[j][lane] : 0.0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) x += __shfl_xor_sync(0xffffffffu, x, s);
            if (lane == 0 && x != 0.0) atomicAdd(dst + j, x);
        }
    }
}

// Loss L = -1/count sum_x log(V_t(x) + eps) over the in-mask voxels (t = the
// true label, V_K implicit) and its adjoint A = E^T dL/dV.
template <int K>
__global__ void __launch_bounds__(kPlainThreads)
    adj_loss_kernel(Geometry g, const float *__restrict__ V, const uint8_t *__restrict__ truth, float eps,
                    double inv_count, float *__restrict__ A, double *loss)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    double acc[1] = {0.0};
    if (p.valid) {
        const int64_t o = p.line * g.nstride_w + p.n;
        const int64_t oo = p.line * g.nstride_in + g.slab_start + p.n;
        float v[K];
        float vk = 1.0f;
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            v[i] = V[i * g.plane_w + o];
            vk -= v[i];
        }
        v[K - 1] = vk;
        int t = truth[oo];
        t = t < K ? t : K - 1;
        float vt = v[0];
#pragma unroll
        for (int i = 1; i < K; ++i)
            if (i == t) vt = v[i];
        acc[0] = -inv_count * log((double)vt + (double)eps);
        const float gt = (float)(-inv_count / ((double)vt + (double)eps));
#pragma unroll
        for (int i = 0; i < K - 1; ++i) A[i * g.plane_w + o] = (t == K - 1) ? -gt : (i == t ? gt : 0.0f);
    }
    block_sum_to<1>(acc, loss);
}

// Backward primal step.  V: V^k; xi: Xi^{k+1}; A: in dL/dV^{k+1}, out dL/dV^k;
// pbar: the dual adjoint of the step after (zeros for the last iteration);
// qbar: out; grad_u: += in the input mapping; grads: += {dL/dlam, dL/dc_0..}.
template <int K>
__global__ void __launch_bounds__(kPlainThreads)
    adj_primal_kernel(Geometry g, const float *__restrict__ V, const float *__restrict__ xi,
                      const float *__restrict__ u, PhaseParams<K> pp, float tau2, float *__restrict__ A,
                      const float *__restrict__ pbar, float *__restrict__ qbar, float *__restrict__ grad_u,
                      double *grads)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    double acc[K + 1];
#pragma unroll
    for (int j = 0; j <= K; ++j) acc[j] = 0.0;
    if (p.valid) {
        const LineInfo li = load_line(g, p.line);
        const int64_t o = p.line * g.nstride_w + p.n;
        const bool hn = p.n + 1 < g.ns, pn = p.n > 0;
        const bool hr = li.flags & kHasNextRow, pr = li.flags & kHasPrevRow;
        const bool hc = li.next_col >= 0, pc = li.prev_col >= 0;
        const int64_t opc = pc ? (int64_t)li.prev_col * g.nstride_w + p.n : o;
        float x[3 * (K - 1)], xn[K - 1], xr[K - 1], xc[K - 1], v[K - 1];
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            x[3 * i] = xi[(3 * i) * g.plane_w + o];
            x[3 * i + 1] = xi[(3 * i + 1) * g.plane_w + o];
            x[3 * i + 2] = xi[(3 * i + 2) * g.plane_w + o];
            xn[i] = pn ? xi[(3 * i) * g.plane_w + o - 1] : 0.0f;
            xr[i] = pr ? xi[(3 * i + 1) * g.plane_w + o - g.nstride_w] : 0.0f;
            xc[i] = pc ? xi[(3 * i + 2) * g.plane_w + opc] : 0.0f;
            v[i] = V[i * g.plane_w + o];
        }
        const float uu = u[p.line * g.nstride_in + g.slab_start + p.n];
        float q[K], vv[K];
        primal_q<K>(q, vv, v, x, xn, xr, xc, pn, hn, pr, hr, pc, hc, uu, pp.c, pp.lam, pp.tau1);
        // B = tau2 E^T (-div pbar) at x, pbar of all K labels (3 planes each)
        float bfull[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const float *pb = pbar + (3 * i) * g.plane_w;
            float dv = 0.0f;
            if (pn) dv -= pb[o - 1];
            if (hn) dv += pb[o];
            if (pr) dv -= pb[g.plane_w + o - g.nstride_w];
            if (hr) dv += pb[g.plane_w + o];
            if (pc) dv -= pb[2 * g.plane_w + opc];
            if (hc) dv += pb[2 * g.plane_w + o];
            bfull[i] = -tau2 * dv;
        }
        float ab[K], qb[K], b[K - 1];
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            b[i] = bfull[i] - bfull[K - 1];
            ab[i] = A[i * g.plane_w + o] + 2.0f * b[i];
        }
        ab[K - 1] = 0.0f;
        simplex_vjp<K>(q, ab, qb);
#pragma unroll
        for (int i = 0; i < K - 1; ++i) A[i * g.plane_w + o] = (qb[i] - qb[K - 1]) - b[i];
#pragma unroll
        for (int i = 0; i < K; ++i) qbar[i * g.plane_w + o] = qb[i];
        // data term: q_i = ... - tau1 lam (u - c_i)^2
        float gu = 0.0f;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const float dl = uu - pp.c[i];
            gu += -pp.tau1 * pp.lam * 2.0f * dl * qb[i];
            acc[0] += (double)(-pp.tau1 * qb[i]) * (double)dl * (double)dl;
            acc[1 + i] += 2.0 * (double)pp.tau1 * (double)pp.lam * (double)dl * (double)qb[i];
        }
        grad_u[p.line * g.nstride_in + g.slab_start + p.n] += gu;
    }
    block_sum_to<K + 1>(acc, grads);
}

// Backward dual step.  xi: Xi^k; vb: Vbar^k; X: in dL/dXi^{k+1}, out dL/dXi^k;
// qbar: this step's primal adjoint; pbar: out.
template <int K>
__global__ void __launch_bounds__(kPlainThreads)
    adj_dual_kernel(Geometry g, const float *__restrict__ xi, const float *__restrict__ vb, float tau1, float tau2,
                    DykstraThresholds thr, float *__restrict__ X, const float *__restrict__ qbar,
                    float *__restrict__ pbar)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    if (!p.valid) return;
    const LineInfo li = load_line(g, p.line);
    const int64_t o = p.line * g.nstride_w + p.n;
    const bool hn = p.n + 1 < g.ns;
    const bool hr = li.flags & kHasNextRow;
    const bool hc = li.next_col >= 0;
    const int64_t oc = hc ? (int64_t)li.next_col * g.nstride_w + p.n : o;
    float vx[K - 1], vn[K - 1], vr[K - 1], vc[K - 1], x[3 * (K - 1)];
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        const float *b = vb + i * g.plane_w;
        vx[i] = b[o];
        vn[i] = hn ? b[o + 1] : 0.0f;
        vr[i] = hr ? b[o + g.nstride_w] : 0.0f;
        vc[i] = hc ? b[oc] : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < 3 * (K - 1); ++j) x[j] = xi[j * g.plane_w + o];
    float pq[K][3];
    dual_build_q<K>(pq, x, vx, vn, vr, vc, hn, hr, hc, tau2);
    // Xtot = X + tau1 E^T (-grad+ qbar): (div^T qbar)_a(x) = h_a (qbar(x) - qbar(x + e_a))
    float dt[K][3];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const float *qb = qbar + i * g.plane_w;
        const float q0 = qb[o];
        dt[i][0] = hn ? q0 - qb[o + 1] : 0.0f;
        dt[i][1] = hr ? q0 - qb[o + g.nstride_w] : 0.0f;
        dt[i][2] = hc ? q0 - qb[oc] : 0.0f;
    }
    float yb[K][3];
#pragma unroll
    for (int i = 0; i < K - 1; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) yb[i][a] = X[(3 * i + a) * g.plane_w + o] + tau1 * (dt[i][a] - dt[K - 1][a]);
    yb[K - 1][0] = yb[K - 1][1] = yb[K - 1][2] = 0.0f;
    float pb[K][3];
    if (dual_first_sweep_is_identity<K>(pq, thr)) {
#pragma unroll
        for (int i = 0; i < K; ++i)
#pragma unroll
            for (int a = 0; a < 3; ++a) pb[i][a] = yb[i][a];
    } else {
        dykstra_vjp<K>(pq, yb, pb, thr);
    }
#pragma unroll
    for (int i = 0; i < K - 1; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) X[(3 * i + a) * g.plane_w + o] = pb[i][a] - pb[K - 1][a];
#pragma unroll
    for (int i = 0; i < K; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) pbar[(3 * i + a) * g.plane_w + o] = pb[i][a];
}

}  // namespace potts
