// Device-side description of one slab of the cylindrical-core volume.
//
// The reference addresses a voxel as base[col] + (row - start_row[col]) *
// nstride + n (include/layout_cylinder.h:81-84).  Every stored (row, col) pair
// is one "line" of nstride values; lines are numbered in storage order
// (column by column, rows of a column consecutively), so line L starts at
// L * nstride.  The solver keeps its state in the same line order with its
// own stride nstride_w (the slab width rounded up to 32) and precomputes, per
// line, the neighbour lines the stencil needs.
#pragma once

#include <cstdint>

namespace potts {

constexpr uint32_t kHasNextRow = 1u;  // row + 1 is stored in the same column
constexpr uint32_t kHasPrevRow = 2u;  // row - 1 is stored in the same column

// One line of the mask: 16 bytes, loaded as one int4.
struct LineInfo {
    int32_t next_col;  // line of (row, col + 1), or -1 when that voxel line is outside the mask
    int32_t prev_col;  // line of (row, col - 1), or -1
    uint32_t flags;    // kHasNextRow | kHasPrevRow
    uint32_t rowcol;   // (col << 16) | row
};

struct Geometry {
    const int4 *lines;  // [n_lines] LineInfo
    int64_t n_lines;    // stored (row, col) lines
    int64_t plane_w;    // n_lines * nstride_w: stride between state components
    int nstride_w;      // stride of n in the state arrays
    int ns;             // n-extent of the slab: n in [0, ns)
    int nstride_in;     // stride of n in u and in the outputs
    int slab_start;     // n of the slab's first slice in u
    // The plain kernels run over the lines [line_begin, n_lines) (a shard's
    // owned lines; 0 = all).  line_base: the line number of line 0 in the
    // whole volume (keys the stochastic rounding of a shard's bfloat16 V).
    int64_t line_begin = 0;
    int64_t line_base = 0;
};

template <int K>
struct PhaseParams {
    float c[K];
    float lam;
    float tau1;
};

__device__ __forceinline__ LineInfo load_line(const Geometry &g, int64_t line)
{
    const int4 v = __ldg(g.lines + line);
    LineInfo li;
    li.next_col = v.x;
    li.prev_col = v.y;
    li.flags = (uint32_t)v.z;
    li.rowcol = (uint32_t)v.w;
    return li;
}

}  // namespace potts
