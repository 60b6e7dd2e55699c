/* CPU check of the histogram kernels' bin decision (hist_bin_r in
 * segmentctscans_b200/csrc/kernels_hist.cuh), restated here in C with the same IEEE single-precision
 * operations, against the reference's formula (calc_hist.cpp:62-64, uv-hist-kernel.cpp:139-149:
 * t = (x - start) / (end - start), bin = round(nb t - 0.5) clamped to [0, nb - 1]).
 *
 * The kernels replace the division by the product with the correctly rounded reciprocal and decide
 * the rounding from floor(y) and the exact fraction y - floor(y); only when y lies within
 * nb 1e-6 + 1e-6 of a half-integer away from both ends do they divide.  This program draws random
 * values, the values next to both ends and the values next to every rounding boundary of each range,
 * and counts the bins that differ.  Built with -ffp-contract=off, so a * b + c is never contracted
 * and fmaf is the only fused operation, as in the kernels.
 *
 * Output: one line per range, "start end nb values fallbacks mismatches"; exit status 1 on any
 * mismatch. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

static int ref_bin(float x, float start, float end, int nb)
{
    const float t = (x - start) / (end - start);
    const float r = roundf(fmaf((float)nb, t, -0.5f));
    if (!(r >= 0.0f)) return 0;
    if (r >= (float)(nb - 1)) return nb - 1;
    return (int)r;
}

static int fast_bin(float x, float start, float end, float rinv, int nb, long *fallbacks)
{
    const float y = fmaf((float)nb, (x - start) * rinv, -0.5f);
    const float fl = floorf(y);
    const float f = y - fl;
    if (fabsf(f - 0.5f) > fmaf((float)nb, 1e-6f, 1e-6f)) {
        const float r = f > 0.5f ? fl + 1.0f : fl;
        return (int)fminf(fmaxf(r, 0.0f), (float)(nb - 1));
    }
    if (f == f && (fl + 1.0f <= 0.0f || fl >= (float)(nb - 1))) return fl >= 0.0f ? nb - 1 : 0;
    ++*fallbacks;
    return ref_bin(x, start, end, nb);
}

static uint64_t rng_state = 0x9e3779b97f4a7c15ull;
static uint64_t next_u64(void)
{
    uint64_t z = (rng_state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* the histograms count values in [start, end]; the 1-D one also values jittered just below start */
static int check(float start, float end, int nb, long n_random)
{
    const float rinv = 1.0f / (end - start);
    long values = 0, fallbacks = 0, mismatches = 0;
#define TEST(xv)                                                                              \
    do {                                                                                      \
        const float x_ = (xv);                                                                \
        if (x_ == x_ && x_ >= start && x_ <= end) {                                           \
            ++values;                                                                         \
            if (fast_bin(x_, start, end, rinv, nb, &fallbacks) != ref_bin(x_, start, end, nb)) \
                ++mismatches;                                                                 \
        }                                                                                     \
    } while (0)
    for (long i = 0; i < n_random; ++i) {
        const double u = (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0);
        TEST((float)((double)start + u * ((double)end - (double)start)));
    }
    /* both ends and their neighbours */
    float lo = start, hi = end;
    for (int k = 0; k < 2000; ++k) {
        TEST(lo);
        TEST(hi);
        lo = nextafterf(lo, end);
        hi = nextafterf(hi, start);
    }
    /* every rounding boundary (at most 20000 of them, spread over the range), 64 floats each side */
    const int step = nb > 20000 ? nb / 20000 : 1;
    for (int k = 0; k <= nb; k += step) {
        const double xb = (double)start + ((double)k / nb) * ((double)end - (double)start);
        float x = (float)xb;
        for (int j = 0; j < 64; ++j) x = nextafterf(x, -INFINITY);
        for (int j = 0; j < 129; ++j) {
            TEST(x);
            x = nextafterf(x, INFINITY);
        }
    }
#undef TEST
    printf("%.9g %.9g %d %ld %ld %ld\n", start, end, nb, values, fallbacks, mismatches);
    return mismatches != 0;
}

int main(int argc, char **argv)
{
    const long n_random = argc > 1 ? atol(argv[1]) : 1000000;
    int bad = 0;
    bad |= check(0.0f, 1.0f, 512, n_random);
    bad |= check(0.0f, 1.0f, 1024, n_random);
    bad |= check(0.0f, 1.0f, 65535, n_random);
    bad |= check(0.25f, 0.75f, 1000, n_random);
    bad |= check(9.759767e-05f, 0.34773535f, 512, n_random); /* the phantom's gradient range */
    bad |= check(-3.0f, 5.0f, 37, n_random);
    bad |= check(1e-3f, 1.000001e-3f, 256, n_random);        /* a range of a few ulps */
    bad |= check(100.0f, 200.5f, 60000, n_random);
    bad |= check(-1.5e-38f, 2.5e-38f, 7, n_random);           /* subnormal values */
    bad |= check(0.0f, 1.0f, 1, n_random);
    bad |= check(0.0f, 1.0f, 2, n_random);
    return bad;
}
