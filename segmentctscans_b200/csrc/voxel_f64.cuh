// FP64 per-voxel arithmetic of the Potts primal-dual iteration, for the
// FP64 solve (state and arithmetic in double precision, split kernels only).
// It is the large-volume counterpart of the CPU oracle: the same operations,
// in the same order, with a multiply and an add fused exactly where the
// reference's clang build contracts them (written as fma()), so on the same
// input it gives the same bits as the FP64 oracle.  The translation unit is
// compiled with -fmad=false; division and square root are the IEEE
// double-precision operations.
//
//   nearest_label_f64   init_v_kernel    potts-model/potts-min-partition.cpp:56-94
//   dual_voxel_f64      grad_kernel      potts-model/potts-min-partition.cpp:96-247
//   project_simplex_f64 project_simplex  potts-model/potts-min-partition.cpp:292-347
//   primal_voxel_f64    div_kernel       potts-model/potts-min-partition.cpp:349-488
//   argmax_label_f64    update_kernel    potts-model/potts-min-partition.cpp:491-538
#pragma once

#include <cfloat>

namespace potts {

// std::max(a, b) as the reference writes it: (a < b) ? b : a
__device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; }

// index of the label nearest to u (strict <, the first of equals wins)
template <int K>
__device__ __forceinline__ int nearest_label_f64(double u, const float (&c)[K])
{
    double best = DBL_MAX;
    int cluster = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double d = fabs((double)c[k] - u);
        if (d < best) {
            best = d;
            cluster = k;
        }
    }
    return cluster;
}

// argmax with strict >, starting from 0 (the first of equal maxima wins)
template <int K>
__device__ __forceinline__ int argmax_label_f64(const double (&v)[K - 1])
{
    double best = 0.0, vk = 1.0;
    int lab = 0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        double vi;
        if (i < K - 1) {
            vi = v[i];
            vk -= vi;
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

// Dykstra's projection onto {|q_i - q_j| <= 1, i < j}: pairs in lexicographic
// order, at most 20 sweeps, exit once every step of a sweep is shorter than
// 1e-6.  q[i][axis].
template <int K>
__device__ __forceinline__ void project_K_f64(double (&q)[K][3])
{
    constexpr int kPairs = K * (K - 1) / 2;
    double P[kPairs][3];
#pragma unroll
    for (int p = 0; p < kPairs; ++p) P[p][0] = P[p][1] = P[p][2] = 0.0;
    for (int sweep = 0; sweep < 20; ++sweep) {
        double max_d = -DBL_MAX;
        int p = 0;
#pragma unroll
        for (int i1 = 0; i1 < K - 1; ++i1) {
#pragma unroll
            for (int i2 = i1 + 1; i2 < K; ++i2, ++p) {
                double qh[3], qhh[3], d[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) qh[a] = q[i2][a] - q[i1][a] + P[p][a];
                double s = qh[0] * qh[0];
                s = fma(qh[1], qh[1], s);
                s = fma(qh[2], qh[2], s);
                const double l = sqrt(s);
#pragma unroll
                for (int a = 0; a < 3; ++a) qhh[a] = (l > 1.0) ? ((l - 1.0) * qh[a]) / l : 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a) d[a] = 0.5 * (qhh[a] - P[p][a]);
                double dd = d[0] * d[0];
                dd = fma(d[1], d[1], dd);
                dd = fma(d[2], d[2], dd);
                max_d = dmax_ref(sqrt(dd), max_d);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    q[i1][a] += d[a];
                    q[i2][a] -= d[a];
                    P[p][a] = qhh[a];
                }
            }
        }
        if (1e-6 > max_d) break;
    }
}

// Dual step at one voxel: q = Xi + tau2 grad+(Vbar) (a missing forward
// neighbour gives a zero difference), then Dykstra.  xi[3 i + axis] are the
// stored K-1 labels; vb* are Vbar at x and at the forward neighbours.
template <int K>
__device__ __forceinline__ void dual_voxel_f64(double (&xo)[3 * (K - 1)], const double (&xi)[3 * (K - 1)],
                                               const double (&vb)[K - 1], const double (&vbn)[K - 1],
                                               const double (&vbr)[K - 1], const double (&vbc)[K - 1], bool hn,
                                               bool hr, bool hc, double tau2)
{
    double q[K][3];
    double vk = 1.0, vkn = 1.0, vkr = 1.0, vkc = 1.0;
    double xk[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < K; ++i) {
        double vi, g[3] = {0.0, 0.0, 0.0}, x[3];
        if (i < K - 1) {
            vi = vb[i];
            vk -= vi;
        } else {
            vi = vk;
        }
        if (hn) {
            double w;
            if (i < K - 1) {
                w = vbn[i];
                vkn -= w;
            } else {
                w = vkn;
            }
            g[0] = w - vi;
        }
        if (hr) {
            double w;
            if (i < K - 1) {
                w = vbr[i];
                vkr -= w;
            } else {
                w = vkr;
            }
            g[1] = w - vi;
        }
        if (hc) {
            double w;
            if (i < K - 1) {
                w = vbc[i];
                vkc -= w;
            } else {
                w = vkc;
            }
            g[2] = w - vi;
        }
        if (i < K - 1) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                x[a] = xi[3 * i + a];
                xk[a] -= x[a];
            }
        } else {
#pragma unroll
            for (int a = 0; a < 3; ++a) x[a] = xk[a];
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) q[i][a] = fma(g[a], tau2, x[a]);
    }
    project_K_f64<K>(q);
#pragma unroll
    for (int i = 0; i < K - 1; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) xo[3 * i + a] = q[i][a];
}

// Projection onto the simplex: descending sort (any sort gives the same
// values), rho = the last i with u_i > (sum_{j<=i} u_j - 1) / i.
template <int K>
__device__ __forceinline__ void project_simplex_f64(double (&q)[K])
{
    double u[K];
#pragma unroll
    for (int i = 0; i < K; ++i) u[i] = q[i];
#pragma unroll
    for (int r = 0; r < K; ++r) {  // odd-even transposition sort, descending
#pragma unroll
        for (int i = (r & 1); i + 1 < K; i += 2) {
            if (u[i] < u[i + 1]) {
                const double t = u[i];
                u[i] = u[i + 1];
                u[i + 1] = t;
            }
        }
    }
    double sum = 0.0, rho_sum = 0.0;
    int rho = 0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        sum += u[i];
        const double theta = (sum - 1.0) / (double)(i + 1);
        if (u[i] > theta) {
            rho = i + 1;
            rho_sum = sum;
        }
    }
    const double theta = (rho_sum - 1.0) / (double)rho;
#pragma unroll
    for (int i = 0; i < K; ++i) q[i] = dmax_ref(q[i] - theta, 0.0);
}

// Primal step at one voxel: q = Pi_S(V + tau1 (div- Xi - lam (u - c)^2)),
// Vbar = 2q - V; returns |q - V|^2 over all K labels.  xin/xir/xic are the
// n/row/col components of Xi at the backward neighbours; p*/h* say whether
// the backward/forward neighbour exists.
template <int K>
__device__ __forceinline__ double primal_voxel_f64(double (&vnew)[K - 1], double (&vbar)[K - 1],
                                                   const double (&v)[K - 1], const double (&xi)[3 * (K - 1)],
                                                   const double (&xin)[K - 1], const double (&xir)[K - 1],
                                                   const double (&xic)[K - 1], bool pn, bool hn, bool pr, bool hr,
                                                   bool pc, bool hc, double u, const float (&c)[K], double lam,
                                                   double tau1)
{
    double q[K], vv[K];
    double vk = 1.0, xk[3] = {0.0, 0.0, 0.0}, xkn = 0.0, xkr = 0.0, xkc = 0.0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        double x[3], div = 0.0, w;
        if (i < K - 1) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                x[a] = xi[3 * i + a];
                xk[a] -= x[a];
            }
        } else {
#pragma unroll
            for (int a = 0; a < 3; ++a) x[a] = xk[a];
        }
        if (pn) {
            if (i < K - 1) {
                w = xin[i];
                xkn -= w;
            } else {
                w = xkn;
            }
            div -= w;
        }
        if (hn) div += x[0];
        if (pr) {
            if (i < K - 1) {
                w = xir[i];
                xkr -= w;
            } else {
                w = xkr;
            }
            div -= w;
        }
        if (hr) div += x[1];
        if (pc) {
            if (i < K - 1) {
                w = xic[i];
                xkc -= w;
            } else {
                w = xkc;
            }
            div -= w;
        }
        if (hc) div += x[2];
        double vi;
        if (i < K - 1) {
            vi = v[i];
            vk -= vi;
        } else {
            vi = vk;
        }
        vv[i] = vi;
        const double dlt = u - (double)c[i];
        const double d2 = dlt * dlt;
        const double wv = fma(-lam, d2, div);
        q[i] = fma(tau1, wv, vi);
    }
    project_simplex_f64<K>(q);
    double dq = 0.0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const double e = q[i] - vv[i];
        dq = (i == 0) ? e * e : fma(e, e, dq);
    }
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        vbar[i] = 2.0 * q[i] - vv[i];
        vnew[i] = q[i];
    }
    return dq;
}

}  // namespace potts
