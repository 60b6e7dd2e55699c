/*
 * CPU oracle for the multiphase Potts primal-dual solve (test infrastructure only).
 *
 * This file is the correctness checker of the project, not part of the product:
 * only tests/, the smoke check and the CPU-baseline leg of bench.py load it.
 * It restates, plainly and per voxel, the Chambolle-Cremers-Pock iteration of
 * the reference solver:
 *
 *   init_v_kernel   potts-model/potts-min-partition.cpp:56-94
 *   grad_kernel     potts-model/potts-min-partition.cpp:96-247   (dual step + Dykstra)
 *   project_simplex potts-model/potts-min-partition.cpp:292-347
 *   div_kernel      potts-model/potts-min-partition.cpp:349-488  (primal step)
 *   update_kernel   potts-model/potts-min-partition.cpp:491-538  (argmax)
 *   host driver     potts-model/potts-min-partition.cpp:540-679  (slabs + halo)
 *   cylinder layout include/layout_cylinder.h:81-97 (offsets, row ranges)
 *
 * Parity unpinned: the reference ships no tests, golden vectors or fixtures for
 * this path and cannot be built in this environment (it needs clang-CUDA,
 * Boost.Hana, mdspan, range-v3 and CCCL 3 launch/buffer APIs), so this
 * restatement is checked against mathematical properties (simplex KKT,
 * projection feasibility, grad/div adjointness) rather than reference outputs.
 *
 * The file is compiled twice: REAL=double (the FP64 oracle) and REAL=float
 * (an FP32 mode).  Where the reference's clang build would contract a multiply
 * and an add into one fused multiply-add, this restatement writes FMA()
 * explicitly, and it is compiled with -ffp-contract=off so that no other
 * contraction happens.  In FP32 mode every operation is therefore an IEEE
 * single-precision operation with a fixed order.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL double
#endif
#ifndef SFX
#define SFX f64
#endif

#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define NAME(x) CAT(x, SFX)

#if defined(ORACLE_REAL_IS_FLOAT)
#define FMA(a, b, c) fmaf((a), (b), (c))
#define SQRT(x) sqrtf(x)
#define FABS(x) fabsf(x)
#define RMAX FLT_MAX
#else
#define FMA(a, b, c) fma((a), (b), (c))
#define SQRT(x) sqrt(x)
#define FABS(x) fabs(x)
#define RMAX DBL_MAX
#endif

#define KMAX 6

/* Host copy of layout_cylinder::mapping (include/layout_cylinder.h:30-112). */
typedef struct {
    uint32_t n_images, rows, cols;
    uint32_t nstride, col_begin, col_end;
    const uint32_t *start_row; /* cols entries   */
    const uint32_t *base;      /* cols+1 entries */
} ocyl;

static inline int64_t row_begin(const ocyl *m, uint32_t col) { return m->start_row[col]; }
static inline int64_t row_end(const ocyl *m, uint32_t col)
{
    return (int64_t)m->start_row[col] + (int64_t)(m->base[col + 1] - m->base[col]) / m->nstride;
}
/* layout_cylinder.h:81-84 */
static inline int64_t offset(const ocyl *m, int64_t n, int64_t row, uint32_t col)
{
    return (int64_t)m->base[col] + (row - (int64_t)m->start_row[col]) * m->nstride + n;
}
static inline int row_in(const ocyl *m, uint32_t col, int64_t row)
{
    return row_begin(m, col) <= row && row < row_end(m, col);
}

/* std::max / cuda::std::max(a, b) as the reference uses it: (a < b) ? b : a */
static inline REAL rmax(REAL a, REAL b) { return (a < b) ? b : a; }

/* ---------------------------------------------------------------------------
 * Projection onto the simplex, potts-min-partition.cpp:292-347.
 * The reference sorts with sorting networks; any correct sort yields the same
 * sorted values, so a plain insertion sort is used here.
 * ------------------------------------------------------------------------- */
void NAME(oracle_project_simplex)(REAL *q, int K)
{
    REAL u[KMAX];
    for (int i = 0; i < K; ++i) u[i] = q[i];
    for (int i = 1; i < K; ++i) {            /* descending */
        REAL x = u[i];
        int j = i - 1;
        while (j >= 0 && u[j] < x) { u[j + 1] = u[j]; --j; }
        u[j + 1] = x;
    }
    REAL sum = 0, rho_sum = 0;
    int rho = 0;
    for (int i = 0; i < K; ++i) {
        sum += u[i];
        REAL theta = (sum - (REAL)1) / (REAL)(i + 1);
        if (u[i] > theta) { rho = i + 1; rho_sum = sum; }
    }
    REAL theta = (rho_sum - (REAL)1) / (REAL)rho;
    for (int i = 0; i < K; ++i) q[i] = rmax(q[i] - theta, (REAL)0);
}

/* ---------------------------------------------------------------------------
 * Dykstra projection onto K = {|q_i - q_j| <= 1, i < j},
 * potts-min-partition.cpp:202-238.  q holds K vectors of 3 components,
 * q[3*i + axis].  Returns the number of sweeps run.
 * ------------------------------------------------------------------------- */
int NAME(oracle_project_K)(REAL *q, int K)
{
    REAL P[KMAX * (KMAX - 1) / 2][3];
    memset(P, 0, sizeof(P));
    int sweep;
    for (sweep = 0; sweep < 20; ++sweep) {
        REAL max_d = -RMAX;
        int p = 0; /* pair index in lexicographic (i1, i2) order, :209 */
        for (int i1 = 0; i1 < K - 1; ++i1) {
            for (int i2 = i1 + 1; i2 < K; ++i2, ++p) {
                REAL qh[3], qhh[3], d[3];
                for (int a = 0; a < 3; ++a) qh[a] = q[3 * i2 + a] - q[3 * i1 + a] + P[p][a];
                REAL s = qh[0] * qh[0];
                s = FMA(qh[1], qh[1], s);
                s = FMA(qh[2], qh[2], s);
                REAL l = SQRT(s);
                for (int a = 0; a < 3; ++a) qhh[a] = (l > (REAL)1) ? ((l - (REAL)1) * qh[a]) / l : (REAL)0;
                for (int a = 0; a < 3; ++a) d[a] = (REAL)0.5 * (qhh[a] - P[p][a]);
                REAL dd = d[0] * d[0];
                dd = FMA(d[1], d[1], dd);
                dd = FMA(d[2], d[2], dd);
                REAL dn = SQRT(dd);
                max_d = rmax(dn, max_d);
                for (int a = 0; a < 3; ++a) {
                    q[3 * i1 + a] += d[a];
                    q[3 * i2 + a] -= d[a];
                    P[p][a] = qhh[a];
                }
            }
        }
        /* `1e-6 > max_δ` compares against the double literal 1e-6 (:235) */
        if (1e-6 > (double)max_d) { ++sweep; break; }
    }
    return sweep;
}

/* ---------------------------------------------------------------------------
 * Solver state for one slab [n_lo, n_hi): arrays are indexed by the input
 * mapping (same offsets as u); only n in [n_lo, n_hi) is touched.
 * ------------------------------------------------------------------------- */
typedef struct {
    const ocyl *m;
    int K;
    int64_t span;
    REAL *xi;  /* 3(K-1) planes of span */
    REAL *V;   /* K-1 planes */
    REAL *Vb;  /* K-1 planes */
    int store; /* 0: state kept in REAL; 1: stored as bfloat16; 2: stored as IEEE binary16 */
    int it;    /* 0-based iteration of the current primal step (keys the stochastic rounding of V) */
} ostate;

/* Rounding of a stored state value to the storage format (round to nearest,
 * ties to even) and back.  bfloat16 keeps the top 16 bits of the binary32
 * pattern; binary16 uses the compiler's _Float16 conversion (IEEE). */
static inline REAL store_round(int store, REAL x)
{
    if (store == 1) {
        float f = (float)x;
        uint32_t b;
        memcpy(&b, &f, 4);
        if ((b & 0x7fffffffu) <= 0x7f800000u) { /* not NaN */
            b += 0x7fffu + ((b >> 16) & 1u);
            b &= 0xffff0000u;
        }
        memcpy(&f, &b, 4);
        return (REAL)f;
    }
    if (store == 2) return (REAL)(float)(_Float16)(float)x;
    return x;
}

/* The stored V of the bfloat16 format is rounded stochastically, with the
 * random bits drawn from a counter-based hash of (line, n, iteration, pair of
 * components): the result is reproducible and the same in every kernel form,
 * and rounding no longer swallows the small updates of a converging solve.
 * The mixer is "lowbias32" of Chris Wellons' hash-prospector (public domain);
 * the key multipliers are the golden-ratio and xxHash32 primes.  The random
 * 16 bits are added to the binary32 pattern before the low half is cut off,
 * which rounds away from zero with probability equal to the cut fraction. */
static inline uint32_t sr_mix(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

static inline uint32_t sr_hash(uint32_t line, uint32_t n, uint32_t it, uint32_t pair)
{
    return sr_mix((line * 0x9e3779b1u) ^ (n * 0x85ebca77u) ^ ((it * 4u + pair) * 0xc2b2ae3du));
}

static inline REAL store_round_v(const ostate *st, REAL x, uint32_t line, uint32_t n, int i)
{
    if (st->store != 1) return store_round(st->store, x);
    float f = (float)x;
    uint32_t b;
    memcpy(&b, &f, 4);
    if ((b & 0x7fffffffu) < 0x7f800000u) { /* finite */
        const uint32_t h = sr_hash(line, n, (uint32_t)st->it, (uint32_t)(i >> 1));
        b += (i & 1) ? (h >> 16) : (h & 0xffffu);
        b &= 0xffff0000u;
    }
    memcpy(&f, &b, 4);
    return (REAL)f;
}

/* init_v_kernel, potts-min-partition.cpp:56-94: V = V_bar = one-hot of the
 * nearest label (strict <, first wins). */
static void init_v(ostate *st, const float *u, const REAL *c, int n_lo, int n_hi)
{
    const ocyl *m = st->m;
    const int K = st->K;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t col = m->col_begin; col < m->col_end; ++col) {
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row) {
            for (int64_t n = n_lo; n < n_hi; ++n) {
                int64_t o = offset(m, n, row, col);
                REAL v = (REAL)u[o];
                REAL best = RMAX;
                int cluster = 0;
                for (int k = 0; k < K; ++k) {
                    REAL d = FABS(c[k] - v);
                    if (d < best) { best = d; cluster = k; }
                }
                for (int i = 0; i < K - 1; ++i) {
                    REAL x = (i == cluster) ? (REAL)1 : (REAL)0;
                    st->V[i * st->span + o] = x;
                    st->Vb[i * st->span + o] = x;
                }
            }
        }
    }
}

/* grad_kernel, potts-min-partition.cpp:96-247 (returns nothing; Xi updated in place). */
static void grad_step(ostate *st, REAL tau2, int n_lo, int n_hi, int *sweep_hist)
{
    const ocyl *m = st->m;
    const int K = st->K;
    const int64_t S = st->span;
    int64_t hist[21];
    memset(hist, 0, sizeof(hist));
#pragma omp parallel
    {
        int64_t lh[21];
        memset(lh, 0, sizeof(lh));
#pragma omp for schedule(dynamic, 4)
        for (int64_t col = m->col_begin; col < m->col_end; ++col) {
            for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row) {
                const int has_r = row_end(m, col) - 1 > row;
                const int has_c = (int64_t)m->col_end - 1 > col && row_in(m, (uint32_t)(col + 1), row);
                for (int64_t n = n_lo; n < n_hi; ++n) {
                    const int has_n = n_hi - 1 > n;
                    const int64_t o = offset(m, n, row, col);
                    const int64_t on = has_n ? offset(m, n + 1, row, col) : 0;
                    const int64_t orr = has_r ? offset(m, n, row + 1, col) : 0;
                    const int64_t oc = has_c ? offset(m, n, row, (uint32_t)(col + 1)) : 0;
                    REAL q[3 * KMAX];
                    REAL vk = 1, vkn = 1, vkr = 1, vkc = 1;
                    REAL xk[3] = {0, 0, 0};
                    for (int i = 0; i < K; ++i) {
                        REAL vi, g[3] = {0, 0, 0}, xi_i[3];
                        if (i < K - 1) { vi = st->Vb[i * S + o]; vk -= vi; } else vi = vk;
                        if (has_n) {
                            REAL w;
                            if (i < K - 1) { w = st->Vb[i * S + on]; vkn -= w; } else w = vkn;
                            g[0] = w - vi;
                        }
                        if (has_r) {
                            REAL w;
                            if (i < K - 1) { w = st->Vb[i * S + orr]; vkr -= w; } else w = vkr;
                            g[1] = w - vi;
                        }
                        if (has_c) {
                            REAL w;
                            if (i < K - 1) { w = st->Vb[i * S + oc]; vkc -= w; } else w = vkc;
                            g[2] = w - vi;
                        }
                        if (i < K - 1) {
                            for (int a = 0; a < 3; ++a) { xi_i[a] = st->xi[(3 * i + a) * S + o]; xk[a] -= xi_i[a]; }
                        } else {
                            for (int a = 0; a < 3; ++a) xi_i[a] = xk[a];
                        }
                        /* q *= tau2; q += xi  (contracted to one FMA) */
                        for (int a = 0; a < 3; ++a) q[3 * i + a] = FMA(g[a], tau2, xi_i[a]);
                    }
                    int sw = NAME(oracle_project_K)(q, K);
                    lh[sw] += 1;
                    for (int i = 0; i < K - 1; ++i)
                        for (int a = 0; a < 3; ++a) st->xi[(3 * i + a) * S + o] = store_round(st->store, q[3 * i + a]);
                }
            }
        }
#pragma omp critical
        for (int i = 0; i < 21; ++i) hist[i] += lh[i];
    }
    if (sweep_hist)
        for (int i = 0; i < 21; ++i) sweep_hist[i] += (int)hist[i];
}

/* div_kernel, potts-min-partition.cpp:349-488.  Returns max_x |V^{k+1}-V^k|^2. */
/* dq_lo/dq_hi: the columns whose voxels enter the returned max |dV|^2 (all
 * columns are updated). */
static REAL div_step(ostate *st, const float *u, const REAL *c, REAL lam, REAL tau1, int n_lo, int n_hi,
                     int64_t dq_lo, int64_t dq_hi)
{
    const ocyl *m = st->m;
    const int K = st->K;
    const int64_t S = st->span;
    REAL dq_max = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(max : dq_max)
    for (int64_t col = m->col_begin; col < m->col_end; ++col) {
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row) {
            const int has_r = row_end(m, col) - 1 > row;
            const int prv_r = row_begin(m, col) < row;
            const int has_c = (int64_t)m->col_end - 1 > col && row_in(m, (uint32_t)(col + 1), row);
            const int prv_c = (int64_t)m->col_begin < col && row_in(m, (uint32_t)(col - 1), row);
            for (int64_t n = n_lo; n < n_hi; ++n) {
                const int has_n = n_hi - 1 > n;
                const int prv_n = n_lo < n;
                const int64_t o = offset(m, n, row, col);
                const int64_t pn = prv_n ? offset(m, n - 1, row, col) : 0;
                const int64_t pr = prv_r ? offset(m, n, row - 1, col) : 0;
                const int64_t pc = prv_c ? offset(m, n, row, (uint32_t)(col - 1)) : 0;
                const REAL g = (REAL)u[o];
                REAL q[KMAX], v[KMAX];
                REAL vk = 1;
                REAL xk[3] = {0, 0, 0};
                REAL xkn = 0, xkr = 0, xkc = 0;
                for (int i = 0; i < K; ++i) {
                    REAL xi_i[3], div = 0, w;
                    if (i < K - 1) {
                        for (int a = 0; a < 3; ++a) { xi_i[a] = st->xi[(3 * i + a) * S + o]; xk[a] -= xi_i[a]; }
                    } else {
                        for (int a = 0; a < 3; ++a) xi_i[a] = xk[a];
                    }
                    if (prv_n) {
                        if (i < K - 1) { w = st->xi[(3 * i + 0) * S + pn]; xkn -= w; } else w = xkn;
                        div -= w;
                    }
                    if (has_n) div += xi_i[0];
                    if (prv_r) {
                        if (i < K - 1) { w = st->xi[(3 * i + 1) * S + pr]; xkr -= w; } else w = xkr;
                        div -= w;
                    }
                    if (has_r) div += xi_i[1];
                    if (prv_c) {
                        if (i < K - 1) { w = st->xi[(3 * i + 2) * S + pc]; xkc -= w; } else w = xkc;
                        div -= w;
                    }
                    if (has_c) div += xi_i[2];
                    REAL vi;
                    if (i < K - 1) { vi = st->V[i * S + o]; vk -= vi; } else vi = vk;
                    v[i] = vi;
                    /* q = v + tau1 * (div - lam * sqr(g - c_i)) */
                    REAL dlt = g - c[i];
                    REAL d2 = dlt * dlt;
                    REAL wv = FMA(-lam, d2, div);
                    q[i] = FMA(tau1, wv, vi);
                }
                NAME(oracle_project_simplex)(q, K);
                REAL dq = 0;
                for (int i = 0; i < K; ++i) {
                    REAL e = q[i] - v[i];
                    dq = (i == 0) ? e * e : FMA(e, e, dq);
                }
                const uint32_t line = m->base[col] / m->nstride + (uint32_t)(row - row_begin(m, col));
                for (int i = 0; i < K - 1; ++i) {
                    st->Vb[i * S + o] = store_round(st->store, (REAL)2 * q[i] - v[i]);
                    st->V[i * S + o] = store_round_v(st, q[i], line, (uint32_t)n, i);
                }
                if (dq > dq_max && col >= dq_lo && col < dq_hi) dq_max = dq;
            }
        }
    }
    return dq_max;
}

/* update_kernel, potts-min-partition.cpp:491-538: argmax (strict >, v starts at 0). */
static void update(const ostate *st, const float *c, int n_lo, int n_hi, float *res, uint8_t *labels)
{
    const ocyl *m = st->m;
    const int K = st->K;
    const int64_t S = st->span;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t col = m->col_begin; col < m->col_end; ++col) {
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row) {
            for (int64_t n = n_lo; n < n_hi; ++n) {
                const int64_t o = offset(m, n, row, col);
                REAL best = 0, vk = 1;
                int lab = 0;
                for (int i = 0; i < K; ++i) {
                    REAL vi;
                    if (i < K - 1) { vi = st->V[i * S + o]; vk -= vi; } else vi = vk;
                    if (vi > best) { best = vi; lab = i; }
                }
                if (res) res[o] = c[lab];
                if (labels) labels[o] = (uint8_t)lab;
            }
        }
    }
}

/* ---------------------------------------------------------------------------
 * FP64 energies of a state (V, Xi) over the voxels of [n_lo, n_hi):
 *   lagrangian = sum_x sum_i V_i (G_i - div Xi_i)
 *   dual       = sum_x min_i (G_i - div Xi_i)
 *   gap        = lagrangian - dual  (>= 0 for V on the simplex)
 * with G_i = lam (u - c_i)^2.  The reference computes no energy; this is the
 * diagnostic reported every few iterations.  Sums are per column over the
 * columns [col_lo, col_hi) (neighbours outside that range still count in the
 * divergence), then added in column order.
 * ------------------------------------------------------------------------- */
static void energies(const ostate *st, const float *u, const REAL *c, REAL lam, int n_lo, int n_hi, int64_t col_lo,
                     int64_t col_hi, double out[3])
{
    const ocyl *m = st->m;
    const int K = st->K;
    const int64_t S = st->span;
    const int64_t ncol = col_hi - col_lo;
    double *part = (double *)calloc((size_t)(2 * (ncol > 0 ? ncol : 1)), sizeof(double));
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t col = col_lo; col < col_hi; ++col) {
        double sl = 0, sd = 0;
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row) {
            const int has_r = row_end(m, col) - 1 > row;
            const int prv_r = row_begin(m, col) < row;
            const int has_c = (int64_t)m->col_end - 1 > col && row_in(m, (uint32_t)(col + 1), row);
            const int prv_c = (int64_t)m->col_begin < col && row_in(m, (uint32_t)(col - 1), row);
            for (int64_t n = n_lo; n < n_hi; ++n) {
                const int has_n = n_hi - 1 > n;
                const int prv_n = n_lo < n;
                const int64_t o = offset(m, n, row, col);
                double dv[KMAX + 1], xk[3] = {0, 0, 0}, xkn = 0, xkr = 0, xkc = 0, vk = 1, lag = 0, mn = DBL_MAX;
                for (int i = 0; i < K; ++i) {
                    double x[3], w, div = 0, vi;
                    if (i < K - 1) {
                        for (int a = 0; a < 3; ++a) { x[a] = (double)st->xi[(3 * i + a) * S + o]; xk[a] -= x[a]; }
                    } else {
                        for (int a = 0; a < 3; ++a) x[a] = xk[a];
                    }
                    if (prv_n) {
                        if (i < K - 1) { w = (double)st->xi[(3 * i) * S + offset(m, n - 1, row, col)]; xkn -= w; } else w = xkn;
                        div -= w;
                    }
                    if (has_n) div += x[0];
                    if (prv_r) {
                        if (i < K - 1) { w = (double)st->xi[(3 * i + 1) * S + offset(m, n, row - 1, col)]; xkr -= w; } else w = xkr;
                        div -= w;
                    }
                    if (has_r) div += x[1];
                    if (prv_c) {
                        if (i < K - 1) { w = (double)st->xi[(3 * i + 2) * S + offset(m, n, row, (uint32_t)(col - 1))]; xkc -= w; } else w = xkc;
                        div -= w;
                    }
                    if (has_c) div += x[2];
                    if (i < K - 1) { vi = (double)st->V[i * S + o]; vk -= vi; } else vi = vk;
                    double dl = (double)u[o] - (double)c[i];
                    double e = (double)lam * dl * dl - div;
                    dv[i] = e;
                    lag += vi * e;
                    if (e < mn) mn = e;
                }
                sl += lag;
                sd += mn;
            }
        }
        part[2 * (col - col_lo)] = sl;
        part[2 * (col - col_lo) + 1] = sd;
    }
    double L = 0, D = 0;
    for (int64_t i = 0; i < ncol; ++i) { L += part[2 * i]; D += part[2 * i + 1]; }
    free(part);
    out[0] = L;
    out[1] = D;
    out[2] = L - D;
}

/* ---------------------------------------------------------------------------
 * Whole solve, potts-min-partition.cpp:540-679.  oracle_solve_store also
 * models reduced-precision storage of the state: every stored value of Xi, V
 * and Vbar is rounded to bfloat16 (store = 1) or binary16 (store = 2).
 *
 * slab_w <= 0 or >= n_images: one slab over the whole volume.  Otherwise the
 * reference's planner: halo = iters, res_w = slab_w - 2*halo, slabs start at
 * i*res_w, the result of each slab is written without its halo (:627-675).
 *
 * Outputs (each optional): res = c[argmax] (span floats, input mapping),
 * labels = argmax index (span bytes), V_out / Xi_out = final state
 * ((K-1)*span and 3(K-1)*span REALs; single-slab runs only), dq_trace = the
 * squared max |dV|^2 of every iteration of the last slab, energy_trace =
 * (lagrangian, dual, gap) after iterations it with (it+1) % gap_every == 0,
 * sweep_hist = histogram of Dykstra sweep counts (21 ints).
 *
 * Returns 0, or -1 on bad arguments / allocation failure / planner failure.
 * ------------------------------------------------------------------------- */
int NAME(oracle_solve_store)(const ocyl *m, const float *u, int K, const float *c_f, float lam_f, float tau1_f,
                             float tau2_f, int iters, int slab_w, float *res, uint8_t *labels, REAL *V_out,
                             REAL *Xi_out, float *dq_trace, int gap_every, double *energy_trace, int *sweep_hist,
                             int store)
{
    if (!m || !u || K < 2 || K > KMAX || iters < 0) return -1;
    const int n = (int)m->n_images;
    const int64_t span = (int64_t)m->base[m->cols];
    REAL c[KMAX];
    for (int i = 0; i < K; ++i) c[i] = (REAL)c_f[i];
    const REAL lam = (REAL)lam_f, tau1 = (REAL)tau1_f, tau2 = (REAL)tau2_f;

    ostate st;
    st.m = m;
    st.K = K;
    st.span = span;
    st.store = store;
    const size_t ns = (size_t)(span > 0 ? span : 1);
    st.xi = (REAL *)calloc(ns * 3 * (size_t)(K - 1), sizeof(REAL));
    st.V = (REAL *)calloc(ns * (size_t)(K - 1), sizeof(REAL));
    st.Vb = (REAL *)calloc(ns * (size_t)(K - 1), sizeof(REAL));
    if (!st.xi || !st.V || !st.Vb) { free(st.xi); free(st.V); free(st.Vb); return -1; }

    int halo = iters, sw = slab_w, n_slabs = 1, res_w = n;
    if (sw <= 0 || sw >= n) {
        sw = n;
    } else {
        res_w = sw - 2 * halo;
        if (res_w <= 0) { free(st.xi); free(st.V); free(st.Vb); return -1; }
        n_slabs = 1 + (n - sw + res_w - 1) / res_w;
    }
    for (int s = 0; s < n_slabs; ++s) {
        const int s0 = s * res_w;
        const int s1 = (s0 + sw < n) ? s0 + sw : n;
        init_v(&st, u, c, s0, s1);
        memset(st.xi, 0, ns * 3 * (size_t)(K - 1) * sizeof(REAL));
        for (int it = 0; it < iters; ++it) {
            grad_step(&st, tau2, s0, s1, sweep_hist);
            st.it = it;
            REAL dq = div_step(&st, u, c, lam, tau1, s0, s1, m->col_begin, m->col_end);
            if (dq_trace) dq_trace[it] = (float)dq;
            if (energy_trace && gap_every > 0 && (it + 1) % gap_every == 0)
                energies(&st, u, c, lam, s0, s1, m->col_begin, m->col_end,
                         energy_trace + 3 * ((it + 1) / gap_every - 1));
        }
        const int r0 = (s0 == 0) ? s0 : s0 + halo;
        const int r1 = (s1 == n) ? s1 : s1 - halo;
        update(&st, c_f, r0, r1, res, labels);
    }
    if (n_slabs == 1) {
        if (V_out) memcpy(V_out, st.V, ns * (size_t)(K - 1) * sizeof(REAL));
        if (Xi_out) memcpy(Xi_out, st.xi, ns * 3 * (size_t)(K - 1) * sizeof(REAL));
    }
    free(st.xi);
    free(st.V);
    free(st.Vb);
    return 0;
}

int NAME(oracle_solve)(const ocyl *m, const float *u, int K, const float *c_f, float lam_f, float tau1_f,
                       float tau2_f, int iters, int slab_w, float *res, uint8_t *labels, REAL *V_out, REAL *Xi_out,
                       float *dq_trace, int gap_every, double *energy_trace, int *sweep_hist)
{
    return NAME(oracle_solve_store)(m, u, K, c_f, lam_f, tau1_f, tau2_f, iters, slab_w, res, labels, V_out, Xi_out,
                                    dq_trace, gap_every, energy_trace, sweep_hist, 0);
}

/* Single steps on caller-owned state (whole volume as one slab), for tests of
 * the adjoint identity and of individual kernels. */
void NAME(oracle_grad_step)(const ocyl *m, int K, REAL *xi, const REAL *Vb, float tau2)
{
    ostate st = {m, K, (int64_t)m->base[m->cols], xi, NULL, (REAL *)Vb, 0, 0};
    grad_step(&st, (REAL)tau2, 0, (int)m->n_images, NULL);
}

REAL NAME(oracle_div_step)(const ocyl *m, int K, const REAL *xi, REAL *V, REAL *Vb, const float *u, const float *c_f,
                           float lam, float tau1)
{
    REAL c[KMAX];
    for (int i = 0; i < K; ++i) c[i] = (REAL)c_f[i];
    ostate st = {m, K, (int64_t)m->base[m->cols], (REAL *)xi, V, Vb, 0, 0};
    return div_step(&st, u, c, (REAL)lam, (REAL)tau1, 0, (int)m->n_images, m->col_begin, m->col_end);
}

void NAME(oracle_energies)(const ocyl *m, int K, const REAL *xi, const REAL *V, const float *u, const float *c_f,
                           float lam, double out[3])
{
    REAL c[KMAX];
    for (int i = 0; i < K; ++i) c[i] = (REAL)c_f[i];
    ostate st = {m, K, (int64_t)m->base[m->cols], (REAL *)xi, (REAL *)V, NULL, 0, 0};
    energies(&st, u, c, (REAL)lam, 0, (int)m->n_images, m->col_begin, m->col_end, out);
}

/* Column-range forms for sharded solves: the primal step updates every column
 * and returns max |dV|^2 over [col_lo, col_hi); the energies sum over the
 * voxels of [col_lo, col_hi). */
REAL NAME(oracle_div_step_cols)(const ocyl *m, int K, const REAL *xi, REAL *V, REAL *Vb, const float *u,
                                const float *c_f, float lam, float tau1, int64_t col_lo, int64_t col_hi)
{
    REAL c[KMAX];
    for (int i = 0; i < K; ++i) c[i] = (REAL)c_f[i];
    ostate st = {m, K, (int64_t)m->base[m->cols], (REAL *)xi, V, Vb, 0, 0};
    return div_step(&st, u, c, (REAL)lam, (REAL)tau1, 0, (int)m->n_images, col_lo, col_hi);
}

void NAME(oracle_energies_cols)(const ocyl *m, int K, const REAL *xi, const REAL *V, const float *u,
                                const float *c_f, float lam, int64_t col_lo, int64_t col_hi, double out[3])
{
    REAL c[KMAX];
    for (int i = 0; i < K; ++i) c[i] = (REAL)c_f[i];
    ostate st = {m, K, (int64_t)m->base[m->cols], (REAL *)xi, (REAL *)V, NULL, 0, 0};
    energies(&st, u, c, (REAL)lam, 0, (int)m->n_images, col_lo, col_hi, out);
}

/* ---------------------------------------------------------------------------
 * TV-L2 (ROF) denoising by Chambolle's projection algorithm,
 * totalvarmin/chambolle.cpp:220-276, on the cylinder.  xi (3 planes) and v
 * start at zero; each iteration
 *   v  = div xi                                   (div_kernel, :33-87)
 *   G  = grad+ v - (grad+ g) / lambda             (grad_kernel, :89-166)
 *   xi = (xi + tau G) / (1 + tau |G|),  dq = max |xi_new - xi|^2
 * and after the last one g <- g - lambda div xi   (update_kernel, :168-218).
 * The differences use the same neighbour tests as the Potts kernels; the
 * multiply-adds are fused where the reference's clang build contracts them
 * (sum of squares, 1 + tau sqrt, xi + tau G, g - lambda d).  g is float and
 * updated in place; dq_trace (optional) receives the per-iteration dq.
 * ------------------------------------------------------------------------- */
static void tv_div(const ocyl *m, REAL *const xi[3], REAL *out, int64_t col, int64_t row, int64_t n, int64_t o)
{
    const int64_t nn = m->n_images;
    REAL d = 0;
    if (0 < n) d -= xi[0][offset(m, n - 1, row, col)];
    if (nn - 1 > n) d += xi[0][o];
    if (row_begin(m, col) < row) d -= xi[1][offset(m, n, row - 1, col)];
    if (row_end(m, col) - 1 > row) d += xi[1][o];
    if ((int64_t)m->col_begin < col && row_in(m, (uint32_t)(col - 1), row)) d -= xi[2][offset(m, n, row, (uint32_t)(col - 1))];
    if ((int64_t)m->col_end - 1 > col && row_in(m, (uint32_t)(col + 1), row)) d += xi[2][o];
    *out = d;
}

int NAME(oracle_tv)(const ocyl *m, float *g, float lam_f, float tau_f, int iters, float *dq_trace)
{
    if (!m || !g || iters < 0) return -1;
    const int64_t span = (int64_t)m->base[m->cols];
    const size_t ns = (size_t)(span > 0 ? span : 1);
    REAL *buf = (REAL *)calloc(ns * 5, sizeof(REAL));
    if (!buf) return -1;
    REAL *xi[3] = {buf, buf + ns, buf + 2 * ns};
    REAL *v = buf + 3 * ns, *gr = buf + 4 * ns;
    const REAL lam = (REAL)lam_f, tau = (REAL)tau_f;
    for (int64_t i = 0; i < span; ++i) gr[i] = (REAL)g[i];
    const int64_t nn = m->n_images;
    for (int it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(dynamic, 4)
        for (int64_t col = m->col_begin; col < m->col_end; ++col)
            for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
                for (int64_t n = 0; n < nn; ++n) {
                    const int64_t o = offset(m, n, row, col);
                    tv_div(m, xi, &v[o], col, row, n, o);
                }
        REAL dq_max = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(max : dq_max)
        for (int64_t col = m->col_begin; col < m->col_end; ++col)
            for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
                for (int64_t n = 0; n < nn; ++n) {
                    const int64_t o = offset(m, n, row, col);
                    REAL g1 = 0, g2 = 0, g3 = 0;
                    if (nn - 1 > n) {
                        const int64_t p = offset(m, n + 1, row, col);
                        g1 = (v[p] - v[o]) - (gr[p] - gr[o]) / lam;
                    }
                    if (row_end(m, col) - 1 > row) {
                        const int64_t p = offset(m, n, row + 1, col);
                        g2 = (v[p] - v[o]) - (gr[p] - gr[o]) / lam;
                    }
                    if ((int64_t)m->col_end - 1 > col && row_in(m, (uint32_t)(col + 1), row)) {
                        const int64_t p = offset(m, n, row, (uint32_t)(col + 1));
                        g3 = (v[p] - v[o]) - (gr[p] - gr[o]) / lam;
                    }
                    REAL s = g1 * g1;
                    s = FMA(g2, g2, s);
                    s = FMA(g3, g3, s);
                    const REAL denom = FMA(tau, SQRT(s), (REAL)1);
                    const REAL q1 = FMA(tau, g1, xi[0][o]) / denom;
                    const REAL q2 = FMA(tau, g2, xi[1][o]) / denom;
                    const REAL q3 = FMA(tau, g3, xi[2][o]) / denom;
                    const REAL e1 = xi[0][o] - q1, e2 = xi[1][o] - q2, e3 = xi[2][o] - q3;
                    REAL dq = e1 * e1;
                    dq = FMA(e2, e2, dq);
                    dq = FMA(e3, e3, dq);
                    if (dq > dq_max) dq_max = dq;
                    xi[0][o] = q1;
                    xi[1][o] = q2;
                    xi[2][o] = q3;
                }
        if (dq_trace) dq_trace[it] = (float)dq_max;
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t col = m->col_begin; col < m->col_end; ++col)
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
            for (int64_t n = 0; n < nn; ++n) {
                const int64_t o = offset(m, n, row, col);
                REAL d;
                tv_div(m, xi, &d, col, row, n, o);
                g[o] = (float)FMA(-lam, d, gr[o]);
            }
    free(buf);
    return 0;
}
