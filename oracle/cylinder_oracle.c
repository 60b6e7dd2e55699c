/*
 * CPU oracle for the cylindrical-core layout (test infrastructure only).
 *
 * Restates the mask constructor of layout_cylinder::mapping_storage
 * (include/layout_cylinder.h:152-195) and the slab re-mapping
 * (include/layout_cylinder.h:137-149): a (row, col) line is stored iff the
 * row lies strictly inside the circle (col - xc)^2 + (row - yc)^2 < r^2; rows
 * exactly on the boundary are excluded.  Each stored line holds nstride
 * values, columns are stored one after another, rows of a column
 * consecutively.
 */
#include <math.h>
#include <stdint.h>

/* Returns the required span size (base[cols]).  start_row gets cols entries
 * (~0u for empty columns), base gets cols+1 entries. */
uint64_t oracle_cylinder_mask(uint32_t rows, uint32_t cols, double xc, double yc, double r, uint32_t nstride,
                              uint32_t *start_row, uint32_t *base, uint32_t *col_begin, uint32_t *col_end)
{
    const double r2 = r * r;
    uint64_t off = 0;
    uint32_t cb = ~0u, ce = 0;
    for (uint32_t col = 0; col < cols; ++col) {
        double d2 = r2 - ((double)col - xc) * ((double)col - xc);
        base[col] = (uint32_t)off;
        double r0 = 0.0, r1 = 0.0;
        if (0 < d2) {
            double d = sqrt(d2);
            double lo = ceil(yc - d);
            if (yc - d == lo) lo += 1.0;
            double hi = floor(yc + d);
            if (yc + d == hi) hi -= 1.0;
            r0 = lo > 0.0 ? lo : 0.0;
            r1 = hi < (double)(rows - 1) ? hi : (double)(rows - 1);
        }
        if (0 < d2 && r0 <= r1) {
            uint32_t a = (uint32_t)r0, b = (uint32_t)r1;
            if (cb == ~0u) { cb = col; ce = col + 1; } else { ++ce; }
            start_row[col] = a;
            off += (uint64_t)(b - a + 1) * nstride;
        } else {
            start_row[col] = ~0u;
        }
    }
    base[cols] = (uint32_t)off;
    *col_begin = cb;
    *col_end = ce;
    return off;
}

#include <omp.h>

/* Thread count of the oracle's OpenMP loops (0 = leave the default). */
void oracle_set_threads(int n)
{
    if (n > 0) omp_set_num_threads(n);
}

int oracle_max_threads(void) { return omp_get_max_threads(); }
