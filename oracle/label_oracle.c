/*
 * CPU oracle for the label-finding inputs (test infrastructure only).
 *
 * This file is a correctness checker, not part of the product: only tests/,
 * the smoke check and the CPU-baseline leg of bench.py load it.  It restates,
 * per in-mask voxel and in single precision, the reference's
 *
 *   min_max_kernel       min_max/min_max.cpp:18-54
 *   grad_min_max_kernel  uv-hist/uv-hist-kernel.cpp:29-68   (strictly positive values)
 *   grad_kernel          grad-magn/grad_magn.cpp:17-58      (gradient magnitude, -1 at the boundary)
 *   calc_hist_kernel     calc_hist/calc_hist.cpp:23-80      (1-D histogram, jitter)
 *   uv_hist bin ids      uv-hist/uv-hist-kernel.cpp:100-197 (2-D histogram)
 *
 * on the cylinder layout of include/layout_cylinder.h:81-97.  Compiled with
 * -ffp-contract=off: where the reference's clang build contracts a multiply
 * and an add, this file writes fmaf() (the sum of squares of the gradient, and
 * nbins * t - 0.5 of the bin index).  The jitter is not the reference's
 * randomly seeded Philox stream but a function of (seed, voxel) (SplitMix64),
 * so that a seed reproduces a histogram; without jitter the histograms are the
 * reference's.
 *
 * Parity unpinned: the reference has no tests or golden vectors for these
 * functions and cannot be built here.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

/* Host copy of layout_cylinder::mapping (include/layout_cylinder.h:30-112); the
 * same layout as in potts_oracle.c. */
typedef struct {
    uint32_t n_images, rows, cols;
    uint32_t nstride, col_begin, col_end;
    const uint32_t *start_row; /* cols entries   */
    const uint32_t *base;      /* cols+1 entries */
} ocyl;

static int64_t row_begin(const ocyl *m, uint32_t col) { return m->start_row[col]; }
static int64_t row_end(const ocyl *m, uint32_t col)
{
    return (int64_t)m->start_row[col] + (int64_t)(m->base[col + 1] - m->base[col]) / m->nstride;
}
static int64_t offset(const ocyl *m, int64_t n, int64_t row, uint32_t col)
{
    return (int64_t)m->base[col] + (row - (int64_t)m->start_row[col]) * m->nstride + n;
}
/* row stored in column col (col may be outside [col_begin, col_end)) */
static int has(const ocyl *m, int64_t col, int64_t row)
{
    if (col < (int64_t)m->col_begin || col >= (int64_t)m->col_end) return 0;
    return row_begin(m, (uint32_t)col) <= row && row < row_end(m, (uint32_t)col);
}

int oracle_min_max(const ocyl *m, const float *f, int positive, float *out)
{
    float lo = FLT_MAX, hi = -FLT_MAX;
    for (uint32_t col = m->col_begin; col < m->col_end; ++col)
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
            for (int64_t n = 0; n < m->n_images; ++n) {
                const float x = f[offset(m, n, row, col)];
                if (!positive || x > 0.0f) {
                    lo = fminf(lo, x);
                    hi = fmaxf(hi, x);
                }
            }
    out[0] = lo;
    out[1] = hi;
    return 0;
}

/* grad_magn.cpp:27-55 */
int oracle_grad_magn(const ocyl *m, const float *u, float *v)
{
    const int64_t N = m->n_images;
    for (uint32_t col = m->col_begin; col < m->col_end; ++col)
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
            for (int64_t n = 0; n < N; ++n) {
                const int64_t o = offset(m, n, row, col);
                if (!(N - 1 > n) || !(row_end(m, col) - 1 > row) || !has(m, (int64_t)col + 1, row) || !(0 < n) ||
                    !(row_begin(m, col) < row) || !has(m, (int64_t)col - 1, row)) {
                    v[o] = -1.0f;
                } else {
                    float q1 = 0.0f, q2 = 0.0f, q3 = 0.0f;
                    q1 += u[offset(m, n + 1, row, col)];
                    q2 += u[offset(m, n, row + 1, col)];
                    q3 += u[offset(m, n, row, col + 1)];
                    q1 -= u[offset(m, n - 1, row, col)];
                    q2 -= u[offset(m, n, row - 1, col)];
                    q3 -= u[offset(m, n, row, col - 1)];
                    float s = q1 * q1;
                    s = fmaf(q2, q2, s);
                    s = fmaf(q3, q3, s);
                    v[o] = 0.5f * sqrtf(s);
                }
            }
    return 0;
}

/* calc_hist.cpp:62-64 / uv-hist-kernel.cpp:139-149: round(nb t - 0.5) clamped to [0, nb-1]
 * (a NaN, from an empty range, gives 0 as the GPU's conversion does) */
static int bin_of(float x, float start, float end, int nb)
{
    const float t = (x - start) / (end - start);
    const float r = roundf(fmaf((float)nb, t, -0.5f));
    if (!(r >= 0.0f)) return 0;
    if (r >= (float)(nb - 1)) return nb - 1;
    return (int)r;
}

/* SplitMix64 (Steele, Lea and Flood, 2014; public domain) */
static uint64_t splitmix64(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
/* uniform in [-delta/2, delta/2) for voxel idx = line * n_images + n */
static float jitter_of(uint64_t seed, uint64_t idx, float delta)
{
    const float u01 = (float)(uint32_t)(splitmix64(seed ^ (idx * 0xd1342543de82ef95ull)) >> 40) * 0x1p-24f;
    const float a = -0.5f * delta;
    const float b = delta * u01;
    return a + b;
}

/* calc_hist.cpp:47-67 */
int oracle_calc_hist(const ocyl *m, const float *f, float rs, float re, uint32_t nb, float delta, uint64_t seed,
                     uint32_t *counts)
{
    memset(counts, 0, sizeof(uint32_t) * nb);
    const float hd = delta * 0.5f;
    const float lo = rs - hd;
    for (uint32_t col = m->col_begin; col < m->col_end; ++col)
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row) {
            const uint64_t line = m->base[col] / m->nstride + (uint64_t)(row - row_begin(m, col));
            for (int64_t n = 0; n < m->n_images; ++n) {
                float x = f[offset(m, n, row, col)];
                if (delta != 0.0f) x = x + jitter_of(seed, line * m->n_images + (uint64_t)n, delta);
                if (lo <= x && x + hd <= re) counts[bin_of(x, rs, re, (int)nb)] += 1u;
            }
        }
    return 0;
}

/* uv-hist-kernel.cpp:133-150: bin ybin * stride + xbin of (u, v) inside the ranges */
int oracle_uv_hist(const ocyl *m, const float *u, const float *v, float us, float ue, float vs, float ve, uint32_t nb,
                   uint32_t stride, uint32_t *hist)
{
    memset(hist, 0, sizeof(uint32_t) * ((size_t)(nb - 1) * stride + nb));
    for (uint32_t col = m->col_begin; col < m->col_end; ++col)
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
            for (int64_t n = 0; n < m->n_images; ++n) {
                const int64_t o = offset(m, n, row, col);
                const float x = u[o], y = v[o];
                if (!(us <= x && x <= ue && vs <= y && y <= ve)) continue;
                const int xb = bin_of(x, us, ue, (int)nb), yb = bin_of(y, vs, ve, (int)nb);
                hist[(size_t)yb * stride + (size_t)xb] += 1u;
            }
    return 0;
}
