/*
 * CPU oracle for field I/O and the steps either side of the Potts solve (test
 * infrastructure only).
 *
 * This file is a correctness checker, not part of the product: only tests/
 * and the CPU-baseline leg of bench.py load it.  It restates, one bit or one
 * voxel at a time,
 *
 *   MSB-first bit stream        include/io/outbitstream.h:17-50, include/io/inbitstream.h:35-80
 *   Exp-Golomb ue / se          include/io/writeprimitives.h:55-66, include/io/readprimitives.h:54-76
 *   mapping header              include/layout_cylinder.h:233-312 (mapping_storage::save / load)
 *   Field<T> archive            include/field.h:92-147 (lo/hi for float fields, voxels col -> row -> n)
 *   convert_to_fp_kernel        transpose/convert_to_fp.cpp:11-47
 *   find_intensity_range        transpose/find_intensity_range.cpp:22-110
 *   raw label box (--rawout)    potts-model/potts-model.cpp:184-217
 *   write_png grey levels       potts-model/potts-model.cpp:34-49 (cv::pow, convertTo to 8 bits)
 *
 * on the cylinder layout of include/layout_cylinder.h:81-97.  Compiled with
 * -ffp-contract=off.  The grey levels follow OpenCV's documented semantics
 * (|x|^p for a non-integer p, saturating round-half-even conversion), computed
 * in FP64.
 *
 * Parity unpinned: the reference has no tests, golden files or sample archives
 * for these functions, and its bit-stream headers cannot be compiled here
 * (they need Boost.Hana and Boost.Serialization).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

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
static int64_t offset_of(const ocyl *m, uint32_t n, int64_t row, uint32_t col)
{
    return (int64_t)m->base[col] + (row - (int64_t)m->start_row[col]) * m->nstride + n;
}

/* ---- bit stream ---------------------------------------------------------- */
typedef struct {
    uint8_t *buf; /* NULL: count only */
    uint64_t pos; /* bits written */
} obits;

static void put_bits(obits *w, uint64_t v, int n)
{
    for (int k = n - 1; k >= 0; --k) {
        if (w->buf) {
            uint8_t *b = w->buf + (w->pos >> 3);
            const uint8_t bit = (uint8_t)(0x80u >> (w->pos & 7u));
            if ((v >> k) & 1u)
                *b |= bit;
            else
                *b &= (uint8_t)~bit;
        }
        w->pos++;
    }
}

static void put_ue(obits *w, uint64_t v)
{
    const uint64_t m = v + 1;
    int b = 0;
    while (b < 64 && (m >> b) != 0) ++b; /* bits of m */
    put_bits(w, 0, b - 1);
    put_bits(w, m, b);
}

static void put_se(obits *w, int64_t v) { put_ue(w, v > 0 ? 2 * (uint64_t)v - 1 : 2 * (uint64_t)(-v)); }

typedef struct {
    const uint8_t *buf;
    uint64_t n_bits, pos;
    int overrun;
} ibits;

static uint64_t get_bits(ibits *r, int n)
{
    uint64_t v = 0;
    for (int k = 0; k < n; ++k) {
        if (r->pos >= r->n_bits) {
            r->overrun = 1;
            return 0;
        }
        v = (v << 1) | ((r->buf[r->pos >> 3] >> (7 - (r->pos & 7u))) & 1u);
        r->pos++;
    }
    return v;
}

static uint64_t get_ue(ibits *r)
{
    int zeros = 0;
    while (get_bits(r, 1) == 0) {
        if (r->overrun || ++zeros > 63) {
            r->overrun = 1;
            return 0;
        }
    }
    if (zeros == 0) return 0;
    return ((uint64_t)1 << zeros) + get_bits(r, zeros) - 1;
}

static int64_t get_se(ibits *r)
{
    const uint64_t c = get_ue(r);
    return (c & 1u) ? (int64_t)((c + 1) >> 1) : -(int64_t)(c >> 1);
}

/* ---- archive ------------------------------------------------------------- */
static void put_header(obits *w, const ocyl *m, int bits, float lo, float hi)
{
    put_ue(w, m->n_images);
    put_ue(w, m->rows);
    put_ue(w, m->cols);
    put_ue(w, m->nstride);
    put_ue(w, m->col_begin);
    put_ue(w, m->col_end);
    put_ue(w, m->cols); /* start_row_.size() */
    if (m->cols > 0) {
        put_ue(w, m->start_row[0]);
        for (uint32_t i = 1; i < m->cols; ++i) put_se(w, (int64_t)m->start_row[i] - (int64_t)m->start_row[i - 1]);
    }
    put_ue(w, (uint64_t)m->cols + 1); /* base_.size() */
    put_ue(w, m->base[0]);
    for (uint32_t i = 1; i <= m->cols; ++i) put_se(w, (int64_t)m->base[i] - (int64_t)m->base[i - 1]);
    if (bits == 32) {
        uint32_t b;
        memcpy(&b, &lo, 4);
        put_bits(w, b, 32);
        memcpy(&b, &hi, 4);
        put_bits(w, b, 32);
    }
}

/* Field<T>::save: the archive of `field` (uint32 bit patterns or uint16 values); returns its size in
 * bytes.  out = NULL only counts.  The last byte's unused bits are 0. */
uint64_t oracle_archive_encode(const ocyl *m, int bits, const void *field, float lo, float hi, uint8_t *out,
                               uint64_t *header_bits)
{
    obits w = {out, 0};
    put_header(&w, m, bits, lo, hi);
    if (header_bits) *header_bits = w.pos;
    for (uint32_t col = m->col_begin; col < m->col_end; ++col)
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
            for (uint32_t n = 0; n < m->n_images; ++n) {
                const int64_t o = offset_of(m, n, row, col);
                const uint64_t v = bits == 32 ? ((const uint32_t *)field)[o] : ((const uint16_t *)field)[o];
                put_bits(&w, v, bits);
            }
    if (out && (w.pos & 7u)) put_bits(&w, 0, (int)(8 - (w.pos & 7u)));
    return (w.pos + 7) / 8;
}

/* Field<T>::load.  hdr[6] = n_images, rows, cols, nstride, col_begin, col_end.  start_row / base /
 * field may be NULL (header only; call again with room for cols and cols + 1 entries).  lohi[2] for
 * 32-bit archives.  Returns 0, or -1 when the bytes end early or a table has an unexpected size. */
int oracle_archive_decode(const uint8_t *in, uint64_t n_bytes, int bits, uint32_t *hdr, uint32_t *start_row,
                          uint32_t *base, float *lohi, void *field, uint64_t *header_bits)
{
    ibits r = {in, n_bytes * 8, 0, 0};
    for (int i = 0; i < 6; ++i) hdr[i] = (uint32_t)get_ue(&r);
    const uint32_t cols = hdr[2];
    if ((uint64_t)get_ue(&r) != cols) return -1;
    int64_t prev = 0;
    for (uint32_t i = 0; i < cols; ++i) {
        const int64_t v = i == 0 ? (int64_t)get_ue(&r) : prev + get_se(&r);
        if (start_row) start_row[i] = (uint32_t)v;
        prev = v;
    }
    if (get_ue(&r) != (uint64_t)cols + 1) return -1;
    for (uint32_t i = 0; i <= cols; ++i) {
        const int64_t v = i == 0 ? (int64_t)get_ue(&r) : prev + get_se(&r);
        if (base) base[i] = (uint32_t)v;
        prev = v;
    }
    if (bits == 32) {
        const uint32_t lo = (uint32_t)get_bits(&r, 32), hi = (uint32_t)get_bits(&r, 32);
        if (lohi) {
            memcpy(&lohi[0], &lo, 4);
            memcpy(&lohi[1], &hi, 4);
        }
    }
    if (header_bits) *header_bits = r.pos;
    if (r.overrun) return -1;
    if (!field || !start_row || !base) return 0;
    const ocyl m = {hdr[0], hdr[1], hdr[2], hdr[3], hdr[4], hdr[5], start_row, base};
    for (uint32_t col = m.col_begin; col < m.col_end; ++col)
        for (int64_t row = row_begin(&m, col); row < row_end(&m, col); ++row)
            for (uint32_t n = 0; n < m.n_images; ++n) {
                const uint64_t v = get_bits(&r, bits);
                const int64_t o = offset_of(&m, n, row, col);
                if (bits == 32)
                    ((uint32_t *)field)[o] = (uint32_t)v;
                else
                    ((uint16_t *)field)[o] = (uint16_t)v;
            }
    return r.overrun ? -1 : 0;
}

/* ---- convert_to_fp -------------------------------------------------------- */
void oracle_convert_to_fp(const ocyl *m, int bits, const void *in, float lo, float hi, float *out)
{
    for (uint32_t col = m->col_begin; col < m->col_end; ++col)
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
            for (uint32_t n = 0; n < m->n_images; ++n) {
                const int64_t o = offset_of(m, n, row, col);
                const float v = bits == 32 ? ((const float *)in)[o] : (float)((const uint16_t *)in)[o];
                if (v <= lo)
                    out[o] = 0.0f;
                else if (v >= hi)
                    out[o] = 1.0f;
                else
                    out[o] = (v - lo) / (hi - lo);
            }
}

/* ---- find_intensity_range ------------------------------------------------- */
void oracle_u16_hist(const ocyl *m, const uint16_t *in, uint64_t *hist)
{
    memset(hist, 0, sizeof(uint64_t) * 65536);
    for (uint32_t col = m->col_begin; col < m->col_end; ++col)
        for (int64_t row = row_begin(m, col); row < row_end(m, col); ++row)
            for (uint32_t n = 0; n < m->n_images; ++n) hist[in[offset_of(m, n, row, col)]]++;
}

void oracle_intensity_range(const uint64_t *hist, double tail, uint16_t *lo_out, uint16_t *hi_out)
{
    uint64_t total = 0;
    for (int i = 0; i < 65536; ++i) total += hist[i];
    const double pct_lo = tail * (double)total, pct_hi = (1.0 - tail) * (double)total;
    uint64_t lo = 0, hi = 65536, cum = 0;
    for (uint64_t i = 0; i < 65536; ++i) {
        cum += hist[i];
        if (pct_lo >= (double)cum) lo = i;
        if (pct_hi <= (double)cum) {
            hi = i;
            break;
        }
    }
    *lo_out = (uint16_t)lo;
    *hi_out = (uint16_t)hi;
}

/* ---- raw label box -------------------------------------------------------- */
/* dims[4] = slices, rows, cols, row_begin of the box (potts-model.cpp:186-196, literally: the row
 * range over every column in [col_begin, col_end)).  out = NULL only fills dims. */
void oracle_raw_box(const ocyl *m, const float *f, uint8_t *out, uint32_t *dims)
{
    uint32_t rb = 0xffffffffu, re = 0;
    for (uint32_t col = m->col_begin; col < m->col_end; ++col) {
        if ((uint32_t)row_begin(m, col) < rb) rb = (uint32_t)row_begin(m, col);
        if ((uint32_t)row_end(m, col) > re) re = (uint32_t)row_end(m, col);
    }
    const uint32_t row_size = re - rb, col_size = m->col_end - m->col_begin;
    dims[0] = m->n_images;
    dims[1] = row_size;
    dims[2] = col_size;
    dims[3] = rb;
    if (!out) return;
    uint64_t k = 0;
    for (uint32_t c = 0; c < col_size; ++c)
        for (uint32_t r = 0; r < row_size; ++r)
            for (uint32_t i = 0; i < m->n_images; ++i) {
                const uint32_t col = c + m->col_begin, row = r + rb;
                if (m->col_begin <= col && col < m->col_end && row_begin(m, col) <= row && row < row_end(m, col)) {
                    int x = (int)roundf(255 * f[offset_of(m, i, row, col)]);
                    x = x < 0 ? 0 : x;
                    out[k++] = (uint8_t)(x > 255 ? 255 : x);
                } else {
                    out[k++] = 255;
                }
            }
}

/* ---- PNG slice grey levels ------------------------------------------------ */
/* pix[(row - row_begin(col)) * n_images + n] for the rows of column col. */
void oracle_png_gray(const ocyl *m, const float *f, uint32_t col, uint8_t *pix)
{
    const int64_t rb = row_begin(m, col), re = row_end(m, col);
    for (int64_t row = rb; row < re; ++row)
        for (uint32_t n = 0; n < m->n_images; ++n) {
            const double a = fabs((double)f[offset_of(m, n, row, col)]);
            uint8_t g = 0;
            if (a > 0.0) {
                const double v = nearbyint(pow(a, 1.0 / 2.2) * 255.0);
                g = (uint8_t)(v >= 255.0 ? 255 : v);
            }
            pix[(row - rb) * m->n_images + n] = g;
        }
}
