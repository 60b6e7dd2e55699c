// C-ABI implementation of the B200 Potts solver: device context, fields,
// slab planner and the iteration driver (potts-model/potts-min-partition.cpp:540-679).
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <memory>
#include <mutex>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/potts_b200.h"
#include "geometry.cuh"
#include "kernels_plain.cuh"
#include "kernels_adjoint.cuh"
#include "kernels_tiled.cuh"
#include "tile_shapes.cuh"
#include "kernels_hist.cuh"
#include "kernels_tv.cuh"
#include "kernels_fieldio.cuh"
#include "voxel.cuh"

// Sets the message potts_last_error() returns on this thread; used by the
// library's other translation units.
__attribute__((visibility("hidden"))) void potts_set_last_error(const std::string &msg);

using potts::DykstraThresholds;
using potts::ShapesOf;
using potts::Geometry;
using potts::PhaseParams;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

#define POTTS_CUDA(call)                                                                               \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(e_ == cudaErrorMemoryAllocation ? POTTS_ENOMEM : POTTS_ECUDA,                  \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                           \
    } while (0)

#define POTTS_TRY(expr)              \
    do {                             \
        int s_ = (expr);             \
        if (s_ != POTTS_OK) return s_; \
    } while (0)

inline float bits_to_float(uint32_t b)
{
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

// Bisection over the bit patterns of non-negative floats (which order like
// the floats) for the two Dykstra thresholds; host sqrtf is IEEE like the
// device's __fsqrt_rn.
DykstraThresholds compute_thresholds()
{
    DykstraThresholds t;
    {   // largest s with sqrtf(s) <= 1
        uint32_t lo = 0, hi = 0x7f800000u;
        while (hi - lo > 1) {
            uint32_t mid = lo + (hi - lo) / 2;
            if (std::sqrt(bits_to_float(mid)) > 1.0f) hi = mid; else lo = mid;
        }
        t.len_gt_one = bits_to_float(lo);
    }
    {   // smallest m with (double)sqrtf(m) >= 1e-6
        uint32_t lo = 0, hi = 0x7f800000u;
        while (hi - lo > 1) {
            uint32_t mid = lo + (hi - lo) / 2;
            if ((double)std::sqrt(bits_to_float(mid)) < 1e-6) lo = mid; else hi = mid;
        }
        t.exit_below = bits_to_float(hi);
    }
    return t;
}

uint32_t get_stride(uint32_t n) { return ((n + 31u) / 32u) * 32u; }
uint32_t prev_stride(uint64_t n) { return (uint32_t)std::min<uint64_t>((n / 32u) * 32u, 0x7fffffe0u); }

// Validated host copy of a mapping with its line table.
struct MappingCopy {
    potts_mapping m{};
    std::vector<uint32_t> start_row, base;
    std::vector<int4> lines;
    int64_t n_lines = 0;
    uint64_t span = 0;

    void rebind()
    {
        m.start_row = start_row.data();
        m.base = base.data();
    }
};

int64_t row_end_of(const potts_mapping &m, uint32_t col)
{
    return (int64_t)m.start_row[col] + (int64_t)(m.base[col + 1] - m.base[col]) / m.nstride;
}

bool row_in(const potts_mapping &m, uint32_t col, int64_t row)
{
    return (int64_t)m.start_row[col] <= row && row < row_end_of(m, col);
}

int validate_mapping(const potts_mapping *map)
{
    if (!map || !map->start_row || !map->base) return fail(POTTS_EINVAL, "mapping or its tables is NULL");
    const potts_mapping &m = *map;
    if (m.nstride == 0 || m.nstride % 4 != 0 || m.nstride < m.n_images)
        return fail(POTTS_EINVAL, "nstride must be a multiple of 4 and >= n_images");
    if (m.n_images == 0) return fail(POTTS_EINVAL, "n_images is 0");
    if (m.col_end > m.cols || (m.col_begin > m.col_end && m.col_end != 0))
        return fail(POTTS_EINVAL, "col_begin/col_end out of range");
    if (m.rows > 65535 || m.cols > 65535) return fail(POTTS_EINVAL, "rows and cols are limited to 65535");
    for (uint32_t c = 0; c < m.cols; ++c) {
        if (m.base[c + 1] < m.base[c] || m.base[c] % m.nstride != 0 || (m.base[c + 1] - m.base[c]) % m.nstride != 0)
            return fail(POTTS_EINVAL, "base[] must be non-decreasing multiples of nstride");
        const uint32_t cnt = (m.base[c + 1] - m.base[c]) / m.nstride;
        if (cnt > 0 && ((uint64_t)m.start_row[c] + cnt > m.rows))
            return fail(POTTS_EINVAL, "a column's rows exceed the row extent");
        if (cnt > 0 && (c < m.col_begin || c >= m.col_end))
            return fail(POTTS_EINVAL, "a column outside [col_begin, col_end) holds rows");
    }
    if (m.base[0] != 0) return fail(POTTS_EINVAL, "base[0] must be 0");
    return POTTS_OK;
}

void build_lines(MappingCopy &mc)
{
    const potts_mapping &m = mc.m;
    mc.span = m.base[m.cols];
    mc.n_lines = (int64_t)(mc.span / m.nstride);
    mc.lines.assign((size_t)mc.n_lines, make_int4(-1, -1, 0, 0));
    for (uint32_t col = m.col_begin; col < m.col_end; ++col) {
        const int64_t rb = m.start_row[col], re = row_end_of(m, col);
        const int64_t first = m.base[col] / m.nstride;
        for (int64_t row = rb; row < re; ++row) {
            int4 li;
            li.x = (col + 1 < m.col_end && row_in(m, col + 1, row))
                       ? (int32_t)(m.base[col + 1] / m.nstride + (row - m.start_row[col + 1]))
                       : -1;
            li.y = (col > m.col_begin && row_in(m, col - 1, row))
                       ? (int32_t)(m.base[col - 1] / m.nstride + (row - m.start_row[col - 1]))
                       : -1;
            li.z = (int32_t)((row + 1 < re ? potts::kHasNextRow : 0u) | (row > rb ? potts::kHasPrevRow : 0u));
            li.w = (int32_t)((col << 16) | (uint32_t)row);
            mc.lines[(size_t)(first + row - rb)] = li;
        }
    }
}

int copy_mapping(const potts_mapping *map, MappingCopy &mc)
{
    POTTS_TRY(validate_mapping(map));
    mc.m = *map;
    mc.start_row.assign(map->start_row, map->start_row + map->cols);
    mc.base.assign(map->base, map->base + map->cols + 1);
    mc.rebind();
    build_lines(mc);
    return POTTS_OK;
}

bool same_mapping(const MappingCopy &a, const potts_mapping &b)
{
    if (a.m.n_images != b.n_images || a.m.rows != b.rows || a.m.cols != b.cols || a.m.nstride != b.nstride ||
        a.m.col_begin != b.col_begin || a.m.col_end != b.col_end)
        return false;
    return std::memcmp(a.start_row.data(), b.start_row, sizeof(uint32_t) * b.cols) == 0 &&
           std::memcmp(a.base.data(), b.base, sizeof(uint32_t) * (b.cols + 1)) == 0;
}

// Grow-only device buffer owned by a context.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct potts_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    DykstraThresholds thr{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    MappingCopy mapping;  // last mapping whose line table is on the device
    bool mapping_valid = false;
    DevBuf lines, state, dq, energy, partial, host_u, host_res, host_labels, ustage, err;
    DevBuf hist;      // min/max partials and histogram counters of the label-finding inputs
    DevBuf hist_aux;  // coarse cell counts and cell tables of the 2-D histogram
    DevBuf io, io_tables;  // archive payload / raw label box staging, mask tables of the box kernel
    float *pinned_dq = nullptr;
    // tiled-kernel tables: per column (depends on the mapping) and the work
    // items of the last (slab extent, tile shape) planned
    DevBuf cols, work, vols;
    int n_sm = 0;  // multiprocessors of the device
    bool cols_valid = false;
    int work_key[5] = {-1, -1, -1, -1, -1};
    int gm_segment = 0, gm_ns = -1;  // grad_magn's column segment for this mapping and slice count
    int n_work = 0;
    // Event pairs around runs of consecutive iteration launches (energy
    // evaluations and slab set-up fall outside them), and launch counters.
    std::vector<cudaEvent_t> seg_ev;
    int seg_used = 0;
    bool seg_open = false;
    int loop_launches = 0;
    int64_t total_launches = 0;  // since the last solve began (solves report theirs as int)
    int loop_iters = 0;  // iterations inside the event pairs
    // control words of persistent fused launches (item counters per iteration, grid barrier)
    DevBuf pctl;
};

struct potts_field {
    int device = 0;  // fields may outlive the context that made them
    float *d = nullptr;
    MappingCopy mapping;
};

namespace {

int seg_begin(potts_context *ctx)
{
    if (ctx->seg_open) return POTTS_OK;
    if ((int)ctx->seg_ev.size() < 2 * (ctx->seg_used + 1)) {
        for (int i = 0; i < 2; ++i) {
            cudaEvent_t e;
            POTTS_CUDA(cudaEventCreate(&e));
            ctx->seg_ev.push_back(e);
        }
    }
    POTTS_CUDA(cudaEventRecord(ctx->seg_ev[2 * ctx->seg_used], ctx->stream));
    ctx->seg_open = true;
    return POTTS_OK;
}

int seg_end(potts_context *ctx)
{
    if (!ctx->seg_open) return POTTS_OK;
    POTTS_CUDA(cudaEventRecord(ctx->seg_ev[2 * ctx->seg_used + 1], ctx->stream));
    ctx->seg_open = false;
    ctx->seg_used += 1;
    return POTTS_OK;
}

int seg_total_ms(potts_context *ctx, double *ms)
{
    *ms = 0.0;
    for (int i = 0; i < ctx->seg_used; ++i) {
        float t = 0.0f;
        POTTS_CUDA(cudaEventElapsedTime(&t, ctx->seg_ev[2 * i], ctx->seg_ev[2 * i + 1]));
        *ms += t;
    }
    return POTTS_OK;
}

int ensure(potts_context *ctx, DevBuf &b, size_t bytes)
{
    if (b.bytes >= bytes && b.p) return POTTS_OK;
    if (b.p) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
    }
    if (bytes == 0) return POTTS_OK;
    POTTS_CUDA(cudaMalloc(&b.p, bytes));
    b.bytes = bytes;
    return POTTS_OK;
}

// Frees a context buffer once the stream has finished with it.
int release(potts_context *ctx, DevBuf &b)
{
    if (!b.p) return POTTS_OK;
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    POTTS_CUDA(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
    return POTTS_OK;
}

size_t cached_bytes(const potts_context *ctx)
{
    return ctx->state.bytes + ctx->partial.bytes + ctx->host_u.bytes + ctx->host_res.bytes + ctx->host_labels.bytes +
           ctx->ustage.bytes + ctx->hist.bytes + ctx->io.bytes + ctx->io_tables.bytes;
}

int upload_lines(potts_context *ctx, const potts_mapping *map)
{
    if (ctx->mapping_valid && same_mapping(ctx->mapping, *map)) return POTTS_OK;
    ctx->mapping_valid = false;
    ctx->cols_valid = false;
    ctx->work_key[0] = -1;
    ctx->gm_segment = 0;
    POTTS_TRY(copy_mapping(map, ctx->mapping));
    const size_t bytes = sizeof(int4) * (size_t)std::max<int64_t>(ctx->mapping.n_lines, 1);
    POTTS_TRY(ensure(ctx, ctx->lines, bytes));
    if (ctx->mapping.n_lines > 0)
        POTTS_CUDA(cudaMemcpyAsync(ctx->lines.p, ctx->mapping.lines.data(), sizeof(int4) * ctx->mapping.n_lines,
                                   cudaMemcpyHostToDevice, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->mapping_valid = true;
    return POTTS_OK;
}

// Where the state of one slab lives (stored as ST: float, bfloat16 or binary16).
template <typename ST>
struct SlabState {
    ST *xi[2];  // 3(K-1) planes each (ping-pong for the fused form)
    ST *v[2];   // K-1 planes each (v[1] is Vbar in the split form)
};

// Storage format selected by potts_options::storage.
template <typename ST>
struct StoreInfo;
template <> struct StoreInfo<float> { static constexpr CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; };
template <> struct StoreInfo<__nv_bfloat16> { static constexpr CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; };
template <> struct StoreInfo<__half> { static constexpr CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; };

int state_planes(int K, int variant)
{
    return variant == POTTS_VARIANT_PLAIN ? 5 * (K - 1) : 8 * (K - 1);
}

struct Outputs {
    float *res;
    uint8_t *labels;
    void *V;            // float, or double when v64
    void *Xi;           // float, or double when v64
    bool v64 = false;   // V and Xi are FP64 planes (FP64 state only)
};

inline unsigned plain_blocks(const Geometry &g, int n_begin, int n_end)
{
    const int chunks = (n_end - n_begin + potts::kPlainThreads - 1) / potts::kPlainThreads;
    return (unsigned)((g.n_lines - g.line_begin) * chunks);
}

template <int K, typename ST>
int run_energy(potts_context *ctx, const Geometry &g, const ST *xi, const ST *V, const float *d_u,
               const PhaseParams<K> &pp, double *out)
{
    POTTS_TRY(seg_end(ctx));
    const unsigned nb = plain_blocks(g, 0, g.ns);
    if (nb == 0) return POTTS_OK;
    // one pair of partial sums per block (the buffer is grown outside the iteration loops by the
    // solvers; this keeps every caller safe)
    POTTS_TRY(ensure(ctx, ctx->partial, sizeof(double2) * (size_t)nb));
    ctx->total_launches += 2;
    potts::energy_kernel<K, ST><<<nb, potts::kPlainThreads, 0, ctx->stream>>>(g, xi, V, d_u, pp,
                                                                          (double2 *)ctx->partial.p);
    potts::energy_finish<<<1, 1024, 0, ctx->stream>>>((const double2 *)ctx->partial.p, (int64_t)nb, out);
    POTTS_CUDA(cudaGetLastError());
    return POTTS_OK;
}

// Waits for the stream and reports a bounded device-side wait that gave up.
int check_device_error(potts_context *ctx)
{
    int e = 0;
    POTTS_CUDA(cudaMemcpyAsync(&e, ctx->err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (e != 0) return fail(POTTS_ETIMEOUT, "a device-side wait for a tile load gave up");
    return POTTS_OK;
}

template <int K>
int monitor_sync(potts_context *ctx, int it)
{
    POTTS_CUDA(cudaMemcpyAsync(ctx->pinned_dq, (float *)ctx->dq.p + it, sizeof(float), cudaMemcpyDeviceToHost,
                               ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return POTTS_OK;
}

// ---------------------------------------------------------------------------
// Tiled fused kernel: tensor maps, per-column table, work items.
// ---------------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// A tensor of `rank` dims (dims[0] contiguous), strides in bytes of dims 1.., box per dim.
int encode_map(CUtensorMap *m, CUtensorMapDataType dt, const void *base, int rank, const uint64_t *dims,
               const uint64_t *strides, const uint32_t *box)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return fail(POTTS_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t gd[3], gs[2];
    cuuint32_t bd[3], es[3] = {1, 1, 1};
    for (int i = 0; i < rank; ++i) {
        gd[i] = dims[i];
        bd[i] = box[i];
    }
    for (int i = 0; i + 1 < rank; ++i) gs[i] = strides[i];
    CUresult r = fn(m, dt, (cuuint32_t)rank, const_cast<void *>(base), gd, gs, bd, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(POTTS_ECUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return POTTS_OK;
}

// Planes of L2 prefetch ahead of the fused kernel's load ring by default
// (none: prefetching 2 or 4 planes measured 0.5-3 % slower at 768^2 x 1024).
constexpr int kDefaultPrefetch = 0;

struct TileChoice {
    int rows, slices, vpt, segment;
};

template <int K, typename ST>
int choose_tile(const potts_options &o, TileChoice *tc)
{
    using TS = ShapesOf<K, ST>;
    const int d = o.arith == POTTS_ARITH_FAST ? TS::fast : 0;
    tc->rows = TS::r[d];
    tc->slices = TS::t[d];
    tc->vpt = TS::v[d];
    tc->segment = o.segment_cols > 0 ? o.segment_cols : 64;
    if (tc->segment > 64) return fail(POTTS_EINVAL, "segment_cols must be <= 64");
    if (o.tile_rows > 0 || o.tile_slices > 0 || o.tile_vpt > 0) {
        for (int i = 0; i < TS::n; ++i)
            if ((o.tile_rows <= 0 || o.tile_rows == TS::r[i]) && (o.tile_slices <= 0 || o.tile_slices == TS::t[i]) &&
                (o.tile_vpt <= 0 || o.tile_vpt == TS::v[i])) {
                tc->rows = TS::r[i];
                tc->slices = TS::t[i];
                tc->vpt = TS::v[i];
                return POTTS_OK;
            }
        return fail(POTTS_EINVAL,
                    "tile_rows x tile_slices x tile_vpt is not a compiled tile shape for this K and storage");
    }
    return POTTS_OK;
}

// Per-column table of the fused kernel: x = first line, y/z = row range.
std::vector<int4> column_table(const potts_mapping &m)
{
    std::vector<int4> cols(std::max<uint32_t>(m.cols, 1), make_int4(0, 0, 0, 0));
    for (uint32_t c = 0; c < m.cols; ++c) {
        const int64_t cnt = (int64_t)(m.base[c + 1] - m.base[c]) / m.nstride;
        cols[c].x = (int)(m.base[c] / m.nstride);
        cols[c].y = cnt > 0 ? (int)m.start_row[c] : 0;
        cols[c].z = cnt > 0 ? (int)(m.start_row[c] + cnt) : 0;
    }
    return cols;
}

// Work items of the fused kernel (x = first row, y = first slice, z/w =
// column range), ordered so that items sharing columns run together (halo
// rows of neighbouring tiles meet in L2), the slice tiles of the same rows side
// by side.
std::vector<int4> work_items(const potts_mapping &m, int ns, const TileChoice &tc, int c_begin = -1, int c_end = -1)
{
    // the columns [c_begin, c_end) (default: all active columns)
    const uint32_t cb0 = c_begin < 0 ? m.col_begin : (uint32_t)c_begin;
    const uint32_t ce0 = c_end < 0 ? m.col_end : (uint32_t)c_end;
    int row_lo = INT32_MAX, row_hi = 0;
    for (uint32_t c = cb0; c < ce0; ++c) {
        const int64_t cnt = (int64_t)(m.base[c + 1] - m.base[c]) / m.nstride;
        if (cnt <= 0) continue;
        row_lo = std::min<int>(row_lo, (int)m.start_row[c]);
        row_hi = std::max<int>(row_hi, (int)(m.start_row[c] + cnt));
    }
    struct Item {
        int ca, r0, n0, cb;
    };
    std::vector<Item> items;
    const int tiles = (ns + tc.slices - 1) / tc.slices;
    for (int r0 = row_lo; r0 < row_hi; r0 += tc.rows) {
        int run = -1;
        for (int c = (int)cb0; c <= (int)ce0; ++c) {
            bool active = false;
            if (c < (int)ce0) {
                const int64_t cnt = (int64_t)(m.base[c + 1] - m.base[c]) / m.nstride;
                active = cnt > 0 && (int)m.start_row[c] < r0 + tc.rows && (int)(m.start_row[c] + cnt) > r0;
            }
            if (active && run < 0) run = c;
            if (!active && run >= 0) {
                for (int ca = run; ca < c; ca += tc.segment)
                    for (int t = 0; t < tiles; ++t) items.push_back({ca, r0, t * tc.slices, std::min(c, ca + tc.segment)});
                run = -1;
            }
        }
    }
    std::sort(items.begin(), items.end(), [](const Item &a, const Item &b) {
        if (a.ca != b.ca) return a.ca < b.ca;
        if (a.r0 != b.r0) return a.r0 < b.r0;
        return a.n0 < b.n0;
    });
    std::vector<int4> work(items.size());
    for (size_t i = 0; i < items.size(); ++i) work[i] = make_int4(items[i].r0, items[i].n0, items[i].ca, items[i].cb);
    return work;
}

// Column table and work items of the context's mapping on the device.
int plan_tiles(potts_context *ctx, int ns, const TileChoice &tc)
{
    const MappingCopy &mc = ctx->mapping;
    if (!ctx->cols_valid) {
        const std::vector<int4> cols = column_table(mc.m);
        POTTS_TRY(ensure(ctx, ctx->cols, sizeof(int4) * cols.size()));
        POTTS_CUDA(cudaMemcpy(ctx->cols.p, cols.data(), sizeof(int4) * cols.size(), cudaMemcpyHostToDevice));
        ctx->cols_valid = true;
    }
    const int key[5] = {ns, tc.rows, tc.slices, tc.segment, (int)mc.n_lines};
    if (std::equal(key, key + 5, ctx->work_key)) return POTTS_OK;
    const std::vector<int4> work = work_items(mc.m, ns, tc);
    POTTS_TRY(ensure(ctx, ctx->work, sizeof(int4) * std::max<size_t>(work.size(), 1)));
    if (!work.empty())
        POTTS_CUDA(cudaMemcpy(ctx->work.p, work.data(), sizeof(int4) * work.size(), cudaMemcpyHostToDevice));
    std::copy(key, key + 5, ctx->work_key);
    ctx->n_work = (int)work.size();
    return POTTS_OK;
}

template <int K, typename ST>
struct FusedPlan {
    potts::FusedVolume<K, ST> vol;  // host copy of the volume's descriptor
    int n_work = 0;
    TileChoice tile{};
};

// One launch of the fused kernel over n_work items (work / work_vol on the
// device), volumes in `vols`; `fast` selects the fast arithmetic.
template <int K, typename ST, int I = 0>
int launch_tiled(potts_context *ctx, const TileChoice &tile, bool fast, const potts::FusedVolume<K, ST> *vols,
                 const int4 *work, const int *work_vol, int n_work, int in, int it, float tau2)
{
    using TS = ShapesOf<K, ST>;
    if constexpr (I < TS::n) {
        constexpr int R = TS::r[I], NT = TS::t[I], VPT = TS::v[I];
        if (tile.rows == R && tile.slices == NT && tile.vpt == VPT) {
            const cudaError_t e =
                fast ? potts::launch_fused<K, R, NT, VPT, ST, true>(ctx->stream, vols, work, work_vol, n_work, in, it,
                                                                    tau2, ctx->thr, (int *)ctx->err.p)
                     : potts::launch_fused<K, R, NT, VPT, ST, false>(ctx->stream, vols, work, work_vol, n_work, in,
                                                                     it, tau2, ctx->thr, (int *)ctx->err.p);
            if (e != cudaSuccess)
                return fail(e == cudaErrorMemoryAllocation ? POTTS_ENOMEM : POTTS_ECUDA,
                            std::string("fused kernel launch: ") + cudaGetErrorString(e));
            return POTTS_OK;
        }
        return launch_tiled<K, ST, I + 1>(ctx, tile, fast, vols, work, work_vol, n_work, in, it, tau2);
    } else {
        return fail(POTTS_EINVAL, "no compiled tile shape matches");
    }
}

// One persistent launch of the fused kernel: n_iters iterations (state half
// in0, iteration it0 first) over n_work items; zeroes the launch's control
// words in `ctl` (grown as needed) on the stream first.
template <int K, typename ST, int I = 0>
int launch_tiled_persistent(potts_context *ctx, DevBuf &ctl, const TileChoice &tile, bool fast,
                            const potts::FusedVolume<K, ST> *vols, const int4 *work, const int *work_vol, int n_work,
                            int in0, int it0, int n_iters, float tau2)
{
    using TS = ShapesOf<K, ST>;
    if constexpr (I < TS::n) {
        constexpr int R = TS::r[I], NT = TS::t[I], VPT = TS::v[I];
        if (tile.rows == R && tile.slices == NT && tile.vpt == VPT) {
            const size_t words = (size_t)potts::kPersistentCtlHead + (size_t)std::max(n_iters, 1);
            POTTS_TRY(ensure(ctx, ctl, sizeof(uint32_t) * words));
            POTTS_CUDA(cudaMemsetAsync(ctl.p, 0, sizeof(uint32_t) * words, ctx->stream));
            uint32_t *cw = static_cast<uint32_t *>(ctl.p);
            const cudaError_t e =
                fast ? potts::launch_fused_persistent<K, R, NT, VPT, ST, true>(
                           ctx->stream, vols, work, work_vol, n_work, in0, it0, n_iters, tau2, ctx->thr,
                           (int *)ctx->err.p, cw)
                     : potts::launch_fused_persistent<K, R, NT, VPT, ST, false>(
                           ctx->stream, vols, work, work_vol, n_work, in0, it0, n_iters, tau2, ctx->thr,
                           (int *)ctx->err.p, cw);
            if (e != cudaSuccess)
                return fail(e == cudaErrorMemoryAllocation ? POTTS_ENOMEM : POTTS_ECUDA,
                            std::string("persistent fused kernel launch: ") + cudaGetErrorString(e));
            return POTTS_OK;
        }
        return launch_tiled_persistent<K, ST, I + 1>(ctx, ctl, tile, fast, vols, work, work_vol, n_work, in0, it0,
                                                     n_iters, tau2);
    } else {
        return fail(POTTS_EINVAL, "no compiled tile shape matches");
    }
}

// Descriptor of one volume for the fused kernel: tensor maps of both halves
// of the state and of u (read from ubase with row stride ustride, slice ux0 =
// slice 0 of the volume), its column table and phase parameters.
template <int K, typename ST>
int build_volume(const Geometry &g, const int4 *d_cols, int col_begin, int col_end, const ST *const xi[2],
                 const ST *const v[2], const float *ubase, uint64_t ustride, int ux0, const TileChoice &tile,
                 const PhaseParams<K> &pp, float *dq, int prefetch, potts::FusedVolume<K, ST> *vol)
{
    if (g.plane_w >= (int64_t(1) << 31))
        return fail(POTTS_EINVAL, "a state plane of 2^31 voxels or more needs slabs (set slab_w)");
    std::memset(vol, 0, sizeof(*vol));
    const int R = tile.rows, NT = tile.slices;
    const uint64_t L = (uint64_t)std::max<int64_t>(g.n_lines, 1);
    // boxes as in potts::TileShape: Xi slices n0-XH .. n0+NT+XH-1, V slices
    // n0 .. n0+NT+3 (FP32) or n0+NT+7 (16-bit), whole 16-byte rows
    constexpr uint64_t es = sizeof(ST);
    constexpr int XH = es == 4 ? 4 : 8;
    for (int b = 0; b < 2; ++b) {
        const uint64_t dx[3] = {(uint64_t)g.nstride_w, L, (uint64_t)(3 * (K - 1))};
        const uint64_t sx[2] = {(uint64_t)g.nstride_w * es, (uint64_t)g.plane_w * es};
        const uint32_t bx[3] = {(uint32_t)(NT + 2 * XH), (uint32_t)(R + 2), (uint32_t)(3 * (K - 1))};
        POTTS_TRY(encode_map(&vol->xi[b], StoreInfo<ST>::dt, xi[b], 3, dx, sx, bx));
        const uint64_t dv[3] = {(uint64_t)g.nstride_w, L, (uint64_t)(K - 1)};
        const uint32_t bv[3] = {(uint32_t)(NT + (es == 4 ? 4 : 8)), (uint32_t)(R + 1), (uint32_t)(K - 1)};
        POTTS_TRY(encode_map(&vol->v[b], StoreInfo<ST>::dt, v[b], 3, dv, sx, bv));
        vol->xi_buf[b] = const_cast<ST *>(xi[b]);
        vol->v_buf[b] = const_cast<ST *>(v[b]);
    }
    const uint64_t du[2] = {ustride, L};
    const uint64_t su[1] = {ustride * 4};
    const uint32_t bu[2] = {(uint32_t)(NT + 4), (uint32_t)(R + 1)};
    POTTS_TRY(encode_map(&vol->u, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, ubase, 2, du, su, bu));
    vol->tp.cols = d_cols;
    vol->tp.col_begin = col_begin;
    vol->tp.col_end = col_end;
    vol->tp.ns = g.ns;
    vol->tp.nstride_w = g.nstride_w;
    vol->tp.plane_w = g.plane_w;
    vol->tp.u_x0 = ux0;
    vol->tp.n_base = g.slab_start;
    vol->tp.it = 0;
    vol->tp.prefetch = prefetch < 0 ? 0 : (prefetch == 0 ? kDefaultPrefetch : prefetch);
    vol->pp = pp;
    vol->dq = dq;
    return POTTS_OK;
}

// u of a slab as the fused kernel reads it: in place when the slab's slices
// start on a 16-byte boundary, else staged into `stage` with the state's stride.
int fused_u_source(potts_context *ctx, const Geometry &g, const float *d_u, DevBuf &stage, const float **ubase,
                   uint64_t *ustride, int *ux0)
{
    *ubase = d_u;
    *ustride = (uint64_t)g.nstride_in;
    *ux0 = g.slab_start;
    if (g.slab_start % 4 != 0 || g.nstride_in % 4 != 0 || reinterpret_cast<uintptr_t>(d_u) % 16 != 0) {
        POTTS_TRY(ensure(ctx, stage, sizeof(float) * (size_t)std::max<int64_t>(g.plane_w, 1)));
        const int chunks = (g.ns + potts::kPlainThreads - 1) / potts::kPlainThreads;
        if (g.n_lines > 0)
            potts::stage_u_kernel<<<(unsigned)(g.n_lines * chunks), potts::kPlainThreads, 0, ctx->stream>>>(
                g, d_u, (float *)stage.p);
        ctx->total_launches += 1;
        POTTS_CUDA(cudaGetLastError());
        *ubase = (const float *)stage.p;
        *ustride = (uint64_t)g.nstride_w;
        *ux0 = 0;
    }
    return POTTS_OK;
}

template <int K, typename ST>
int prepare_fused(potts_context *ctx, const Geometry &g, const ST *const xi[2], const ST *const v[2],
                  const float *d_u, const potts_options &o, const PhaseParams<K> &pp, float *dq, FusedPlan<K, ST> *fp)
{
    POTTS_TRY((choose_tile<K, ST>(o, &fp->tile)));
    POTTS_TRY(plan_tiles(ctx, g.ns, fp->tile));
    fp->n_work = ctx->n_work;
    const float *ubase;
    uint64_t ustride;
    int ux0;
    POTTS_TRY(fused_u_source(ctx, g, d_u, ctx->ustage, &ubase, &ustride, &ux0));
    POTTS_TRY((build_volume<K, ST>(g, (const int4 *)ctx->cols.p, (int)ctx->mapping.m.col_begin,
                                   (int)ctx->mapping.m.col_end, xi, v, ubase, ustride, ux0, fp->tile, pp, dq,
                                   o.prefetch, &fp->vol)));
    fp->vol.tp.stall_plane = o.stall_plane;
    return POTTS_OK;
}

// Split-kernel launches in the exact or the fast arithmetic (the FP64 state
// has only the exact one).
template <int K, typename ST>
void launch_dual(bool fast, unsigned nb, cudaStream_t s, const Geometry &g, ST *xi, const ST *vb, float tau2,
                 DykstraThresholds thr)
{
    if constexpr (!std::is_same_v<ST, double>) {
        if (fast) {
            potts::dual_kernel<K, ST, true><<<nb, potts::kPlainThreads, 0, s>>>(g, xi, vb, tau2, thr);
            return;
        }
    }
    potts::dual_kernel<K, ST, false><<<nb, potts::kPlainThreads, 0, s>>>(g, xi, vb, tau2, thr);
}

template <int K, typename ST>
void launch_primal(bool fast, unsigned nb, cudaStream_t s, const Geometry &g, const ST *xi, ST *V, ST *Vb,
                   const float *u, const PhaseParams<K> &pp, float *dq, int it)
{
    if constexpr (!std::is_same_v<ST, double>) {
        if (fast) {
            potts::primal_kernel<K, ST, true><<<nb, potts::kPlainThreads, 0, s>>>(g, xi, V, Vb, u, pp, dq, it);
            return;
        }
    }
    potts::primal_kernel<K, ST, false><<<nb, potts::kPlainThreads, 0, s>>>(g, xi, V, Vb, u, pp, dq, it);
}

// One slab: init, iters iterations, argmax of [res_begin, res_end).
template <int K, typename ST>
int run_slab(potts_context *ctx, const Geometry &g, const float *d_u, const PhaseParams<K> &pp, float tau2,
             int iters, const potts_options &o, const SlabState<ST> &st, int res_begin, int res_end,
             const Outputs &out, int64_t plane_out)
{
    const unsigned nb = plain_blocks(g, 0, g.ns);
    const size_t xi_bytes = sizeof(ST) * 3 * (K - 1) * (size_t)g.plane_w;
    float *dq = o.track_dq ? (float *)ctx->dq.p : nullptr;
    double *energy = (double *)ctx->energy.p;
    const int ge = o.gap_every;
    cudaStream_t s = ctx->stream;
    if (dq && iters > 0) POTTS_CUDA(cudaMemsetAsync(dq, 0, sizeof(float) * iters, s));

    const bool fast = o.arith == POTTS_ARITH_FAST;
    int cur = 0;
    if (o.variant == POTTS_VARIANT_PLAIN || std::is_same_v<ST, double>) {
        ST *xi = st.xi[0], *V = st.v[0], *Vb = st.v[1];
        potts::init_kernel<K, ST><<<nb, potts::kPlainThreads, 0, s>>>(g, d_u, V, Vb, pp);
        ctx->total_launches += 1;
        POTTS_CUDA(cudaMemsetAsync(xi, 0, xi_bytes, s));
        for (int it = 0; it < iters; ++it) {
            POTTS_TRY(seg_begin(ctx));
            launch_dual<K, ST>(fast, nb, s, g, xi, Vb, tau2, ctx->thr);
            launch_primal<K, ST>(fast, nb, s, g, xi, V, Vb, d_u, pp, dq ? dq + it : nullptr, it);
            ctx->loop_launches += 2;
            ctx->total_launches += 2;
            ctx->loop_iters += 1;
            if (ge > 0 && (it + 1) % ge == 0) POTTS_TRY(run_energy<K>(ctx, g, xi, V, d_u, pp, energy + 3 * ((it + 1) / ge - 1)));
            if (o.sync_monitor && dq) POTTS_TRY(monitor_sync<K>(ctx, it));
        }
        POTTS_TRY(seg_end(ctx));
        POTTS_CUDA(cudaGetLastError());
    } else if constexpr (!std::is_same_v<ST, double>) {
        // Fused schedule: a dual step gives Xi^1 from V^0 (= Vbar^0); launch m
        // (m = 1 .. iters-1) turns (Xi^m, V^{m-1}) into (Xi^{m+1}, V^m); a final
        // primal step gives V^iters from Xi^iters.
        // the tiled kernel reads (and multiplies by zero) padding and stale
        // neighbours: keep all of the state finite
        POTTS_CUDA(cudaMemsetAsync(st.xi[0], 0, sizeof(ST) * 8 * (K - 1) * (size_t)g.plane_w, s));
        FusedPlan<K, ST> fp;
        const ST *xs[2] = {st.xi[0], st.xi[1]}, *vs[2] = {st.v[0], st.v[1]};
        if (iters > 1) {
            POTTS_TRY((prepare_fused<K, ST>(ctx, g, xs, vs, d_u, o, pp, dq, &fp)));
            POTTS_TRY(ensure(ctx, ctx->vols, sizeof(fp.vol)));
            POTTS_CUDA(cudaMemcpyAsync(ctx->vols.p, &fp.vol, sizeof(fp.vol), cudaMemcpyHostToDevice, s));
        }
        potts::init_kernel<K, ST><<<nb, potts::kPlainThreads, 0, s>>>(g, d_u, st.v[0], (ST *)nullptr, pp);
        ctx->total_launches += 1;
        POTTS_CUDA(cudaMemsetAsync(st.xi[0], 0, xi_bytes, s));
        if (iters > 0) {
            launch_dual<K, ST>(fast, nb, s, g, st.xi[0], st.v[0], tau2, ctx->thr);
            ctx->total_launches += 1;
        }
        const bool persistent = o.persistent && !o.sync_monitor;
        for (int m = 1; m < iters;) {
            // launches m .. last: one persistent launch up to the next energy
            // evaluation, or a single iteration
            int last = m;
            if (persistent) last = ge > 0 ? std::min(iters - 1, (m + ge - 1) / ge * ge) : iters - 1;
            const int n_it = last - m + 1;
            POTTS_TRY(seg_begin(ctx));
            ctx->loop_launches += 1;
            ctx->total_launches += 1;
            ctx->loop_iters += n_it;
            const auto *vols = (const potts::FusedVolume<K, ST> *)ctx->vols.p;
            if (persistent)
                POTTS_TRY((launch_tiled_persistent<K, ST>)(ctx, ctx->pctl, fp.tile, fast, vols,
                                                           (const int4 *)ctx->work.p, nullptr, fp.n_work, cur, m - 1,
                                                           n_it, tau2));
            else
                POTTS_TRY((launch_tiled<K, ST>)(ctx, fp.tile, fast, vols, (const int4 *)ctx->work.p, nullptr,
                                                fp.n_work, cur, m - 1, tau2));
            cur ^= n_it & 1;
            // launch `last` read Xi^last from half cur ^ 1 and wrote V^last to half cur
            if (ge > 0 && last % ge == 0)
                POTTS_TRY(run_energy<K>(ctx, g, st.xi[cur ^ 1], st.v[cur], d_u, pp, energy + 3 * (last / ge - 1)));
            if (o.sync_monitor && dq) POTTS_TRY(monitor_sync<K>(ctx, m - 1));
            m = last + 1;
        }
        POTTS_TRY(seg_end(ctx));
        if (iters > 0) {
            ctx->total_launches += 1;
            launch_primal<K, ST>(fast, nb, s, g, st.xi[cur], st.v[cur], (ST *)nullptr, d_u, pp,
                                 dq ? dq + (iters - 1) : nullptr, iters - 1);
            if (ge > 0 && iters % ge == 0) POTTS_TRY(run_energy<K>(ctx, g, st.xi[cur], st.v[cur], d_u, pp, energy + 3 * (iters / ge - 1)));
            if (o.sync_monitor && dq) POTTS_TRY(monitor_sync<K>(ctx, iters - 1));
        }
        POTTS_CUDA(cudaGetLastError());
    }
    if (res_end > res_begin) {
        const unsigned nbu = plain_blocks(g, res_begin, res_end);
        ctx->total_launches += 1;
        const bool split = o.variant == POTTS_VARIANT_PLAIN || std::is_same_v<ST, double>;
        const ST *Vf = split ? st.v[0] : st.v[cur];
        const ST *Xf = split ? st.xi[0] : st.xi[cur];
        if (out.v64)
            potts::update_kernel<K, ST, double><<<nbu, potts::kPlainThreads, 0, s>>>(
                g, Vf, Xf, pp, res_begin, res_end, out.res, out.labels, (double *)out.V, (double *)out.Xi, plane_out);
        else
            potts::update_kernel<K, ST, float><<<nbu, potts::kPlainThreads, 0, s>>>(
                g, Vf, Xf, pp, res_begin, res_end, out.res, out.labels, (float *)out.V, (float *)out.Xi, plane_out);
        POTTS_CUDA(cudaGetLastError());
    }
    return POTTS_OK;
}

template <int K, typename ST>
int solve_k(potts_context *ctx, const float *d_u, const float *ci, float lam, float tau1, float tau2, int iters,
            const potts_options &o, const Outputs &out, potts_stats *stats)
{
    const MappingCopy &mc = ctx->mapping;
    const int n = (int)mc.m.n_images;
    const int planes = state_planes(K, o.variant);

    // Slab planner (potts-min-partition.cpp:560-577): as many n-slices as the
    // free memory holds, halo = iters on each side of a slab.  The field-I/O
    // staging buffers are scratch of earlier calls: the solve gets their memory.
    POTTS_TRY(release(ctx, ctx->io));
    POTTS_TRY(release(ctx, ctx->io_tables));
    size_t free_b = 0, total_b = 0;
    POTTS_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t margin = size_t(512) << 20;
    const size_t avail = free_b + ctx->state.bytes > margin ? free_b + ctx->state.bytes - margin : 0;
    const uint64_t bytes_per_slice = sizeof(ST) * (uint64_t)planes * (uint64_t)std::max<int64_t>(mc.n_lines, 1);
    int slab_w = o.slab_w > 0 ? o.slab_w : (int)std::min<uint64_t>(prev_stride(avail / bytes_per_slice), 0x7fffffe0u);
    const int halo = iters;
    int res_w = n, n_slabs = 1;
    if (n <= slab_w) {
        slab_w = n;
    } else {
        res_w = slab_w - 2 * halo;
        if (res_w <= 0)
            return fail(POTTS_ENOMEM, "Not enough memory. Reduce the mask radius or the number of iterations.");
        n_slabs = 1 + (n - slab_w + res_w - 1) / res_w;
    }

    const int nstride_w = (int)get_stride((uint32_t)slab_w);
    const int64_t plane_w = mc.n_lines * (int64_t)nstride_w;
    const size_t state_bytes = sizeof(ST) * (size_t)planes * (size_t)std::max<int64_t>(plane_w, 1);
    POTTS_TRY(ensure(ctx, ctx->state, state_bytes));
    POTTS_TRY(ensure(ctx, ctx->dq, sizeof(float) * (size_t)std::max(iters, 1)));
    const int n_energy = o.gap_every > 0 ? iters / o.gap_every : 0;
    POTTS_TRY(ensure(ctx, ctx->energy, sizeof(double) * 3 * (size_t)std::max(n_energy, 1)));
    if (n_energy > 0) {
        const int chunks = (slab_w + potts::kPlainThreads - 1) / potts::kPlainThreads;
        POTTS_TRY(ensure(ctx, ctx->partial, sizeof(double2) * (size_t)std::max<int64_t>(mc.n_lines * chunks, 1)));
    }

    ST *base = (ST *)ctx->state.p;
    SlabState<ST> st;
    const size_t xi_planes = 3 * (K - 1), v_planes = K - 1;
    st.xi[0] = base;
    if (o.variant == POTTS_VARIANT_PLAIN) {
        st.v[0] = base + xi_planes * plane_w;
        st.v[1] = st.v[0] + v_planes * plane_w;
        st.xi[1] = st.xi[0];
    } else {
        st.xi[1] = base + xi_planes * plane_w;
        st.v[0] = st.xi[1] + xi_planes * plane_w;
        st.v[1] = st.v[0] + v_planes * plane_w;
    }

    PhaseParams<K> pp;
    for (int i = 0; i < K; ++i) pp.c[i] = ci[i];
    pp.lam = lam;
    pp.tau1 = tau1;

    Geometry g;
    g.lines = (const int4 *)ctx->lines.p;
    g.n_lines = mc.n_lines;
    g.plane_w = plane_w;
    g.nstride_w = nstride_w;
    g.nstride_in = (int)mc.m.nstride;

    ctx->seg_used = 0;
    ctx->seg_open = false;
    ctx->loop_launches = ctx->total_launches = ctx->loop_iters = 0;
    POTTS_TRY(ensure(ctx, ctx->err, sizeof(int)));
    POTTS_CUDA(cudaMemsetAsync(ctx->err.p, 0, sizeof(int), ctx->stream));
    POTTS_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int sl = 0; sl < n_slabs; ++sl) {
        const int s0 = sl * res_w;
        const int s1 = std::min(n, s0 + slab_w);
        g.slab_start = s0;
        g.ns = s1 - s0;
        const int r0 = (s0 == 0) ? s0 : s0 + halo;
        const int r1 = (s1 == n) ? s1 : s1 - halo;
        if (mc.n_lines > 0)
            POTTS_TRY((run_slab<K, ST>)(ctx, g, d_u, pp, tau2, iters, o, st, r0 - s0, r1 - s0, out, (int64_t)mc.span));
    }
    POTTS_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));

    if (stats || o.sync_monitor) POTTS_TRY(check_device_error(ctx));
    if (stats) {
        float ms = 0.0f;
        POTTS_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        stats->n_slabs = n_slabs;
        stats->slab_w = slab_w;
        stats->iters = iters;
        stats->solve_ms = ms;
        POTTS_TRY(seg_total_ms(ctx, &stats->loop_ms));
        stats->loop_launches = ctx->loop_launches;
        stats->loop_iters = ctx->loop_iters;
        stats->total_launches = (int)ctx->total_launches;
        stats->state_bytes = state_bytes;
        stats->dq_last = 0.0f;
        if (o.track_dq && iters > 0) {
            std::vector<float> tr((size_t)iters);
            POTTS_CUDA(cudaMemcpy(tr.data(), ctx->dq.p, sizeof(float) * iters, cudaMemcpyDeviceToHost));
            stats->dq_last = std::sqrt(tr.back());
            if (stats->dq_trace) std::memcpy(stats->dq_trace, tr.data(), sizeof(float) * iters);
        }
        if (stats->energy_trace && n_energy > 0)
            POTTS_CUDA(cudaMemcpy(stats->energy_trace, ctx->energy.p, sizeof(double) * 3 * n_energy,
                                  cudaMemcpyDeviceToHost));
    }
    return POTTS_OK;
}

int check_params(int K, const float *ci, float lam, float tau1, float tau2, int iters, const potts_options &o)
{
    if (K < 2 || K > POTTS_MAX_PHASES) return fail(POTTS_EINVAL, "K must be in [2, 6]");
    if (!ci) return fail(POTTS_EINVAL, "ci is NULL");
    for (int i = 0; i < K; ++i)
        if (!std::isfinite(ci[i])) return fail(POTTS_EINVAL, "labels must be finite");
    if (!std::isfinite(lam) || !std::isfinite(tau1) || !std::isfinite(tau2))
        return fail(POTTS_EINVAL, "lambda, tau1 and tau2 must be finite");
    if (iters < 0) return fail(POTTS_EINVAL, "iters must be >= 0");
    if (o.variant != POTTS_VARIANT_FUSED && o.variant != POTTS_VARIANT_PLAIN)
        return fail(POTTS_EINVAL, "unknown variant");
    if (o.storage != POTTS_STORE_F32 && o.storage != POTTS_STORE_BF16 && o.storage != POTTS_STORE_F16 &&
        o.storage != POTTS_STORE_F64)
        return fail(POTTS_EINVAL, "unknown storage");
    if (o.gap_every < 0 || o.slab_w < 0) return fail(POTTS_EINVAL, "gap_every and slab_w must be >= 0");
    if (o.tile_rows < 0 || o.tile_slices < 0 || o.segment_cols < 0 || o.tile_vpt < 0)
        return fail(POTTS_EINVAL, "tile options must be >= 0");
    if (o.prefetch > 16) return fail(POTTS_EINVAL, "prefetch must be <= 16");
    if (o.arith != POTTS_ARITH_EXACT && o.arith != POTTS_ARITH_FAST) return fail(POTTS_EINVAL, "unknown arith");
    if (o.stall_plane < 0) return fail(POTTS_EINVAL, "stall_plane must be >= 0");
    if (o.persistent != 0 && o.persistent != 1) return fail(POTTS_EINVAL, "persistent must be 0 or 1");
    return POTTS_OK;
}

template <typename ST>
int solve_store(potts_context *ctx, const float *d_u, int K, const float *ci, float lam, float tau1, float tau2,
                int iters, const potts_options &o, const Outputs &out, potts_stats *stats)
{
    switch (K) {
    case 2: return solve_k<2, ST>(ctx, d_u, ci, lam, tau1, tau2, iters, o, out, stats);
    case 3: return solve_k<3, ST>(ctx, d_u, ci, lam, tau1, tau2, iters, o, out, stats);
    case 4: return solve_k<4, ST>(ctx, d_u, ci, lam, tau1, tau2, iters, o, out, stats);
    case 5: return solve_k<5, ST>(ctx, d_u, ci, lam, tau1, tau2, iters, o, out, stats);
    case 6: return solve_k<6, ST>(ctx, d_u, ci, lam, tau1, tau2, iters, o, out, stats);
    }
    return fail(POTTS_EINVAL, "K must be in [2, 6]");
}

int solve_dispatch(potts_context *ctx, const potts_mapping *map, const float *d_u, int K, const float *ci,
                   float lam, float tau1, float tau2, int iters, const potts_options *opts, const Outputs &out,
                   potts_stats *stats)
{
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    potts_options o;
    potts_default_options(&o);
    if (opts) o = *opts;
    POTTS_TRY(check_params(K, ci, lam, tau1, tau2, iters, o));
    if (!d_u) return fail(POTTS_EINVAL, "u is NULL");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_TRY(upload_lines(ctx, map));
    if (out.v64 && o.storage != POTTS_STORE_F64) return fail(POTTS_EINVAL, "FP64 outputs need the FP64 state");
    if (o.storage == POTTS_STORE_BF16) return solve_store<__nv_bfloat16>(ctx, d_u, K, ci, lam, tau1, tau2, iters, o, out, stats);
    if (o.storage == POTTS_STORE_F16) return solve_store<__half>(ctx, d_u, K, ci, lam, tau1, tau2, iters, o, out, stats);
    if (o.storage == POTTS_STORE_F64) {
        o.variant = POTTS_VARIANT_PLAIN;  // the FP64 state runs the split kernels only
        return solve_store<double>(ctx, d_u, K, ci, lam, tau1, tau2, iters, o, out, stats);
    }
    return solve_store<float>(ctx, d_u, K, ci, lam, tau1, tau2, iters, o, out, stats);
}

int context_init(int device, void *stream, bool use_stream, potts_context **out)
{
    if (!out) return fail(POTTS_EINVAL, "out is NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(POTTS_ENODEV, "no CUDA device");
    }
    if (device < 0 || device >= count) return fail(POTTS_EINVAL, "device index out of range");
    POTTS_CUDA(cudaSetDevice(device));
    auto *ctx = new potts_context();
    ctx->device = device;
    ctx->thr = compute_thresholds();
    if (cudaDeviceGetAttribute(&ctx->n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) ctx->n_sm = 1;
    if (use_stream) {
        ctx->stream = (cudaStream_t)stream;  // NULL: the device's default stream
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return fail(POTTS_ECUDA, "cudaStreamCreate failed");
        }
        ctx->own_stream = true;
    }
    if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaMallocHost(&ctx->pinned_dq, sizeof(float)) != cudaSuccess) {
        potts_context_destroy(ctx);
        return fail(POTTS_ECUDA, "event/pinned allocation failed");
    }
    *out = ctx;
    return POTTS_OK;
}

#include "adjoint.cuh"
#include "batch.cuh"
#include "label_inputs.cuh"
#include "field_io.cuh"
#include "shard.cuh"

// Work items, shared-memory size and the tensor maps of the two xi buffers (3 planes each,
// boxes of XS slices x XR lines x 3 components) of the tiled TV kernel for TR x TN tiles.
template <int TR, int TN>
int tv_tiled_setup(potts_context *ctx, const Geometry &g, const float *xi_a, const float *xi_b, const float *D,
                   CUtensorMap *maps)
{
    using T = potts::TvTile<TR, TN>;
    POTTS_TRY(plan_tiles(ctx, g.ns, TileChoice{TR, TN, 1, 64}));
    POTTS_CUDA(cudaFuncSetAttribute(potts::tv_tiled_kernel<TR, TN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    T::SMEM_BYTES));
    const uint64_t dims[3] = {(uint64_t)g.nstride_w, (uint64_t)g.n_lines, 3};
    const uint64_t strides[2] = {sizeof(float) * (uint64_t)g.nstride_w, sizeof(float) * (uint64_t)g.plane_w};
    const uint32_t box[3] = {(uint32_t)T::XS, (uint32_t)T::XR, 3};
    POTTS_TRY(encode_map(&maps[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, xi_a, 3, dims, strides, box));
    POTTS_TRY(encode_map(&maps[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, xi_b, 3, dims, strides, box));
    const uint32_t dbox[3] = {(uint32_t)TN, (uint32_t)TR, 3};  // differences of g: L2 prefetch boxes
    POTTS_TRY(encode_map(&maps[2], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, D, 3, dims, strides, dbox));
    return POTTS_OK;
}

template <int TR, int TN>
void tv_tiled_launch(potts_context *ctx, const Geometry &g, const CUtensorMap &xi_map, const CUtensorMap &d_map,
                     const float *D, float *xi_out, float tau, float *dq)
{
    if (ctx->n_work == 0) return;
    const MappingCopy &mc = ctx->mapping;
    potts::tv_tiled_kernel<TR, TN><<<ctx->n_work, potts::kTvThreads, potts::TvTile<TR, TN>::SMEM_BYTES, ctx->stream>>>(
        g, static_cast<const int4 *>(ctx->cols.p), (int)mc.m.col_begin, (int)mc.m.col_end,
        static_cast<const int4 *>(ctx->work.p), xi_map, d_map, D, xi_out, tau, dq, (int *)ctx->err.p);
}

// TV-L2 denoising (chambolle(), totalvarmin/chambolle.cpp:220-276) of d_g in
// place; xi (two halves of 3 planes for the fused forms), v (split form) and the
// differences of g (tiled form) live in the context's state buffer, laid out like g.
int tv_run(potts_context *ctx, float *d_g, float lam, float tau, int iters, int variant, potts_stats *stats)
{
    const MappingCopy &mc = ctx->mapping;
    Geometry g{};
    g.lines = static_cast<const int4 *>(ctx->lines.p);
    g.n_lines = mc.n_lines;
    g.nstride_w = (int)mc.m.nstride;
    g.plane_w = mc.n_lines * (int64_t)mc.m.nstride;
    g.nstride_in = (int)mc.m.nstride;
    g.ns = (int)mc.m.n_images;
    g.slab_start = 0;
    cudaStream_t s = ctx->stream;
    // the tiled kernel's TMA boxes need 16-byte line strides, else the per-voxel fused kernel runs
    const bool tiled = variant == POTTS_VARIANT_FUSED && mc.m.nstride % 4 == 0;
    // split: xi, v; fused forms: xi ping-pong; tiled: and the three difference planes of g
    const size_t planes = variant == POTTS_VARIANT_PLAIN ? 4 : tiled ? 9 : 6;
    POTTS_TRY(ensure(ctx, ctx->state, sizeof(float) * planes * (size_t)std::max<int64_t>(g.plane_w, 1)));
    POTTS_TRY(ensure(ctx, ctx->dq, sizeof(float) * (size_t)std::max(iters, 1)));
    POTTS_TRY(ensure(ctx, ctx->err, sizeof(int)));
    float *xi = static_cast<float *>(ctx->state.p), *v = xi + 3 * g.plane_w;
    float *xi_b = xi + 3 * g.plane_w;  // fused forms: the second half
    float *dgp = xi + 6 * g.plane_w;    // tiled form: differences of g
    float *dq = static_cast<float *>(ctx->dq.p);
    ctx->seg_used = 0;
    ctx->seg_open = false;
    ctx->loop_launches = ctx->total_launches = ctx->loop_iters = 0;
    POTTS_CUDA(cudaEventRecord(ctx->ev0, s));
    // xi starts at zero; every other plane is written at the voxels it is read at before it is read
    POTTS_CUDA(cudaMemsetAsync(ctx->state.p, 0, sizeof(float) * 3 * (size_t)std::max<int64_t>(g.plane_w, 1), s));
    POTTS_CUDA(cudaMemsetAsync(dq, 0, sizeof(float) * (size_t)std::max(iters, 1), s));
    POTTS_CUDA(cudaMemsetAsync(ctx->err.p, 0, sizeof(int), s));
    const unsigned nb = plain_blocks(g, 0, g.ns);
    // tiled form: the Potts kernel's column table and work items for 8 x 128 tiles
    constexpr int kTvRows = 8, kTvSlices = 128;
    CUtensorMap xi_maps[3];  // of xi, xi_b and the differences of g
    int map_in = 0;          // the map of the buffer the next launch reads
    if (tiled && g.n_lines > 0 && iters > 0) {
        POTTS_TRY((tv_tiled_setup<kTvRows, kTvSlices>(ctx, g, xi, xi_b, dgp, xi_maps)));
        potts::tv_gdiff_kernel<<<nb, potts::kPlainThreads, 0, s>>>(g, d_g, dgp, lam);
        ctx->total_launches += 1;
    }
    if (g.n_lines > 0) {
        POTTS_TRY(seg_begin(ctx));
        for (int it = 0; it < iters; ++it) {
            if (tiled) {
                tv_tiled_launch<kTvRows, kTvSlices>(ctx, g, xi_maps[map_in], xi_maps[2], dgp, xi_b, tau, dq + it);
                std::swap(xi, xi_b);
                map_in ^= 1;
                ctx->loop_launches += 1;
                ctx->total_launches += 1;
                ctx->loop_iters += 1;
            } else if (variant == POTTS_VARIANT_PLAIN) {
                potts::tv_div_kernel<<<nb, potts::kPlainThreads, 0, s>>>(g, xi, v);
                potts::tv_grad_kernel<<<nb, potts::kPlainThreads, 0, s>>>(g, d_g, xi, v, lam, tau, dq + it);
                ctx->loop_launches += 2;
                ctx->total_launches += 2;
                ctx->loop_iters += 1;
            } else {
                potts::tv_fused_kernel<<<nb, potts::kPlainThreads, 0, s>>>(g, d_g, xi, xi_b, lam, tau, dq + it);
                std::swap(xi, xi_b);
                ctx->loop_launches += 1;
                ctx->total_launches += 1;
                ctx->loop_iters += 1;
            }
        }
        POTTS_TRY(seg_end(ctx));
        potts::tv_update_kernel<<<nb, potts::kPlainThreads, 0, s>>>(g, d_g, xi, lam);
        ctx->total_launches += 1;
        POTTS_CUDA(cudaGetLastError());
    }
    POTTS_CUDA(cudaEventRecord(ctx->ev1, s));
    if (stats) {
        POTTS_TRY(check_device_error(ctx));
        float ms = 0.0f;
        POTTS_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        stats->n_slabs = 1;
        stats->slab_w = g.ns;
        stats->iters = iters;
        stats->solve_ms = ms;
        POTTS_TRY(seg_total_ms(ctx, &stats->loop_ms));
        stats->loop_launches = ctx->loop_launches;
        stats->loop_iters = ctx->loop_iters;
        stats->total_launches = (int)ctx->total_launches;
        stats->state_bytes = sizeof(float) * planes * (uint64_t)std::max<int64_t>(g.plane_w, 1);
        stats->dq_last = 0.0f;
        if (iters > 0) {
            std::vector<float> tr((size_t)iters);
            POTTS_CUDA(cudaMemcpy(tr.data(), dq, sizeof(float) * iters, cudaMemcpyDeviceToHost));
            stats->dq_last = std::sqrt(tr.back());
            if (stats->dq_trace) std::memcpy(stats->dq_trace, tr.data(), sizeof(float) * iters);
        }
    }
    return POTTS_OK;
}

}  // namespace

__attribute__((visibility("hidden"))) void potts_set_last_error(const std::string &msg) { g_last_error = msg; }

// The mapping checks of every solver entry point, for the library's other
// translation units (host only; sets potts_last_error on failure).
__attribute__((visibility("hidden"))) int potts_check_mapping(const potts_mapping *map)
{
    return validate_mapping(map);
}

extern "C" {

void potts_default_options(potts_options *o)
{
    if (!o) return;
    o->variant = POTTS_VARIANT_FUSED;
    o->storage = POTTS_STORE_F32;
    o->gap_every = 0;
    o->slab_w = 0;
    o->track_dq = 1;
    o->sync_monitor = 0;
    o->tile_rows = 0;
    o->tile_slices = 0;
    o->segment_cols = 0;
    o->tile_vpt = 0;
    o->prefetch = 0;
    o->autotune = 0;
    o->arith = POTTS_ARITH_EXACT;
    o->stall_plane = 0;
    o->persistent = 0;
}

const char *potts_status_string(int s)
{
    switch (s) {
    case POTTS_OK: return "ok";
    case POTTS_EINVAL: return "invalid argument";
    case POTTS_ENOMEM: return "out of device memory";
    case POTTS_ECUDA: return "CUDA error";
    case POTTS_ETIMEOUT: return "device wait timed out";
    case POTTS_ENODEV: return "no CUDA device";
    }
    return "unknown status";
}

const char *potts_last_error(void) { return g_last_error.c_str(); }

int potts_context_create(int device, potts_context **out) { return context_init(device, nullptr, false, out); }

int potts_context_create_on_stream(int device, void *stream, potts_context **out)
{
    return context_init(device, stream, true, out);
}

long long potts_context_launches(const potts_context *ctx) { return ctx ? (long long)ctx->total_launches : 0; }

void potts_context_destroy(potts_context *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (DevBuf *b : {&ctx->lines, &ctx->state, &ctx->dq, &ctx->energy, &ctx->partial, &ctx->host_u,
                      &ctx->host_res, &ctx->host_labels, &ctx->ustage, &ctx->err, &ctx->cols, &ctx->work, &ctx->vols,
                      &ctx->hist, &ctx->hist_aux, &ctx->io, &ctx->io_tables, &ctx->pctl})
        if (b->p) cudaFree(b->p);
    if (ctx->pinned_dq) cudaFreeHost(ctx->pinned_dq);
    for (cudaEvent_t e : ctx->seg_ev) cudaEventDestroy(e);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int potts_context_synchronize(potts_context *ctx)
{
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return POTTS_OK;
}

int potts_device_memory(potts_context *ctx, size_t *available, size_t *total)
{
    if (!ctx || !available || !total) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    size_t f = 0, t = 0;
    POTTS_CUDA(cudaMemGetInfo(&f, &t));
    *available = f + cached_bytes(ctx);
    *total = t;
    return POTTS_OK;
}

int potts_field_create(potts_context *ctx, const potts_mapping *map, potts_field **out)
{
    if (!ctx || !out) return fail(POTTS_EINVAL, "NULL argument");
    *out = nullptr;
    auto *f = new potts_field();
    int s = copy_mapping(map, f->mapping);
    if (s != POTTS_OK) {
        delete f;
        return s;
    }
    f->device = ctx->device;
    cudaSetDevice(ctx->device);
    const size_t bytes = sizeof(float) * (size_t)std::max<uint64_t>(f->mapping.span, 1);
    cudaError_t e = cudaMalloc(&f->d, bytes);
    if (e != cudaSuccess) {
        delete f;
        return fail(e == cudaErrorMemoryAllocation ? POTTS_ENOMEM : POTTS_ECUDA, cudaGetErrorString(e));
    }
    *out = f;
    return POTTS_OK;
}

int potts_field_upload(potts_context *ctx, const potts_mapping *map, const float *host, potts_field **out)
{
    if (!host) return fail(POTTS_EINVAL, "host is NULL");
    POTTS_TRY(potts_field_create(ctx, map, out));
    potts_field *f = *out;
    cudaError_t e = cudaMemcpyAsync(f->d, host, sizeof(float) * f->mapping.span, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        potts_field_destroy(f);
        *out = nullptr;
        return fail(POTTS_ECUDA, cudaGetErrorString(e));
    }
    return POTTS_OK;
}

int potts_field_download(potts_context *ctx, const potts_field *f, float *host, uint64_t span)
{
    if (!ctx || !f || !host) return fail(POTTS_EINVAL, "NULL argument");
    if (span != f->mapping.span) return fail(POTTS_EINVAL, "Host and device images have different sizes.");
    POTTS_CUDA(cudaMemcpyAsync(host, f->d, sizeof(float) * span, cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return POTTS_OK;
}

float *potts_field_data(potts_field *f) { return f ? f->d : nullptr; }
uint64_t potts_field_span(const potts_field *f) { return f ? f->mapping.span : 0; }

void potts_field_destroy(potts_field *f)
{
    if (!f) return;
    if (f->d) {
        cudaSetDevice(f->device);
        cudaFree(f->d);  // waits for work on the device that may still use it
    }
    delete f;
}

int potts_solve_device(potts_context *ctx, const potts_mapping *map, const float *d_u, int K, const float *ci,
                       float lambda, float tau1, float tau2, int iters, const potts_options *opts, float *d_res,
                       uint8_t *d_labels, float *d_V, float *d_Xi, potts_stats *stats)
{
    Outputs out{d_res, d_labels, d_V, d_Xi};
    return solve_dispatch(ctx, map, d_u, K, ci, lambda, tau1, tau2, iters, opts, out, stats);
}

int potts_solve_device_f64(potts_context *ctx, const potts_mapping *map, const float *d_u, int K, const float *ci,
                           float lambda, float tau1, float tau2, int iters, const potts_options *opts, float *d_res,
                           uint8_t *d_labels, double *d_V, double *d_Xi, potts_stats *stats)
{
    potts_options o;
    potts_default_options(&o);
    if (opts) o = *opts;
    o.storage = POTTS_STORE_F64;
    Outputs out{d_res, d_labels, d_V, d_Xi, true};
    return solve_dispatch(ctx, map, d_u, K, ci, lambda, tau1, tau2, iters, &o, out, stats);
}

int potts_min_partition(potts_context *ctx, const potts_field *g, const potts_mapping *cpu_map, int K,
                        const float *ci, float lambda, float tau1, float tau2, int iters,
                        const potts_options *opts, potts_field **result, potts_stats *stats)
{
    if (!ctx || !g || !result) return fail(POTTS_EINVAL, "NULL argument");
    *result = nullptr;
    const potts_mapping *map = cpu_map ? cpu_map : &g->mapping.m;
    if (cpu_map && (cpu_map->base == nullptr || cpu_map->base[cpu_map->cols] != g->mapping.span))
        return fail(POTTS_EINVAL, "cpu_map does not describe g");
    potts_field *res = nullptr;
    POTTS_TRY(potts_field_create(ctx, map, &res));
    cudaError_t e = cudaMemsetAsync(res->d, 0, sizeof(float) * res->mapping.span, ctx->stream);
    if (e != cudaSuccess) {
        potts_field_destroy(res);
        return fail(POTTS_ECUDA, cudaGetErrorString(e));
    }
    Outputs out{res->d, nullptr, nullptr, nullptr};
    int s = solve_dispatch(ctx, map, g->d, K, ci, lambda, tau1, tau2, iters, opts, out, stats);
    if (s != POTTS_OK) {
        potts_field_destroy(res);
        return s;
    }
    *result = res;
    return POTTS_OK;
}

int potts_solve_host(potts_context *ctx, const potts_mapping *map, const float *h_u, int K, const float *ci,
                     float lambda, float tau1, float tau2, int iters, const potts_options *opts, float *h_res,
                     uint8_t *h_labels, potts_stats *stats)
{
    if (!ctx || !map || !h_u) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_TRY(validate_mapping(map));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    const uint64_t span = map->base[map->cols];
    POTTS_TRY(ensure(ctx, ctx->host_u, sizeof(float) * std::max<uint64_t>(span, 1)));
    if (h_res) POTTS_TRY(ensure(ctx, ctx->host_res, sizeof(float) * std::max<uint64_t>(span, 1)));
    if (h_labels) POTTS_TRY(ensure(ctx, ctx->host_labels, std::max<uint64_t>(span, 1)));
    POTTS_CUDA(cudaMemcpyAsync(ctx->host_u.p, h_u, sizeof(float) * span, cudaMemcpyHostToDevice, ctx->stream));
    Outputs out{h_res ? (float *)ctx->host_res.p : nullptr, h_labels ? (uint8_t *)ctx->host_labels.p : nullptr,
                nullptr, nullptr};
    POTTS_TRY(solve_dispatch(ctx, map, (const float *)ctx->host_u.p, K, ci, lambda, tau1, tau2, iters, opts, out,
                             stats));
    if (h_res)
        POTTS_CUDA(cudaMemcpyAsync(h_res, ctx->host_res.p, sizeof(float) * span, cudaMemcpyDeviceToHost, ctx->stream));
    if (h_labels)
        POTTS_CUDA(cudaMemcpyAsync(h_labels, ctx->host_labels.p, span, cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return POTTS_OK;
}

uint64_t potts_cylinder_mapping(uint32_t rows, uint32_t cols, double xc, double yc, double r, uint32_t nstride,
                                uint32_t *start_row, uint32_t *base, uint32_t *col_begin, uint32_t *col_end)
{
    // include/layout_cylinder.h:152-195: a row is kept iff it lies strictly
    // inside the circle; columns are stored in order.
    const double r2 = r * r;
    uint64_t off = 0;
    uint32_t cb = ~0u, ce = 0;
    for (uint32_t col = 0; col < cols; ++col) {
        const double dx = (double)col - xc;
        const double d2 = r2 - dx * dx;
        base[col] = (uint32_t)off;
        start_row[col] = ~0u;
        if (!(d2 > 0.0)) continue;
        const double d = std::sqrt(d2);
        double lo = std::ceil(yc - d);
        if (yc - d == lo) lo += 1.0;  // on the circle: outside
        double hi = std::floor(yc + d);
        if (yc + d == hi) hi -= 1.0;
        lo = std::max(0.0, lo);
        hi = std::min((double)rows - 1.0, hi);
        if (lo > hi) continue;
        if (cb == ~0u) cb = col, ce = col;
        ce = col + 1;
        start_row[col] = (uint32_t)lo;
        off += (uint64_t)((uint32_t)hi - (uint32_t)lo + 1) * nstride;
    }
    base[cols] = (uint32_t)off;
    if (col_begin) *col_begin = cb;
    if (col_end) *col_end = ce;
    return off;
}

uint32_t potts_get_stride(uint32_t n) { return get_stride(n); }

int potts_batch_create(potts_context *ctx, int n_volumes, const potts_batch_volume *volumes, int K, float tau1,
                       float tau2, int iters, const potts_options *opts, potts_batch **out)
{
    if (!out) return fail(POTTS_EINVAL, "out is NULL");
    *out = nullptr;
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    if (n_volumes <= 0 || !volumes) return fail(POTTS_EINVAL, "a batch needs at least one volume");
    potts_options o;
    potts_default_options(&o);
    if (opts) o = *opts;
    o.variant = POTTS_VARIANT_FUSED;
    o.gap_every = 0;
    o.slab_w = 0;
    for (int i = 0; i < n_volumes; ++i) {
        POTTS_TRY(check_params(K, volumes[i].ci, volumes[i].lambda, tau1, tau2, iters, o));
        if (!volumes[i].d_u) return fail(POTTS_EINVAL, "a volume's u is NULL");
    }
    POTTS_CUDA(cudaSetDevice(ctx->device));
    auto *b = new potts_batch();
    b->ctx = ctx;
    b->K = K;
    b->storage = o.storage;
    b->iters = iters;
    b->tau1 = tau1;
    b->tau2 = tau2;
    b->opts = o;
    b->vols.resize((size_t)n_volumes);
    int rc = POTTS_OK;
    for (int i = 0; i < n_volumes && rc == POTTS_OK; ++i) {
        BatchVolume &bv = b->vols[(size_t)i];
        rc = copy_mapping(&volumes[i].map, bv.mc);
        bv.d_u = volumes[i].d_u;
        bv.res = volumes[i].d_res;
        bv.labels = volumes[i].d_labels;
        bv.V = volumes[i].d_V;
        for (int k = 0; k < K; ++k) bv.c[k] = volumes[i].ci[k];
        bv.lambda = volumes[i].lambda;
    }
    if (rc == POTTS_OK) {
        if (o.storage == POTTS_STORE_BF16)
            rc = batch_build_store<__nv_bfloat16>(b);
        else if (o.storage == POTTS_STORE_F16)
            rc = batch_build_store<__half>(b);
        else
            rc = batch_build_store<float>(b);
    }
    if (rc != POTTS_OK) {
        const std::string msg = g_last_error;
        batch_free(b);
        g_last_error = msg;
        return rc;
    }
    *out = b;
    return POTTS_OK;
}

int potts_batch_run(potts_batch *b, potts_stats *stats)
{
    if (!b || !b->exec[0]) return fail(POTTS_EINVAL, "batch is NULL");
    potts_context *ctx = b->ctx;
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_CUDA(cudaEventRecord(b->ev[0], ctx->stream));
    POTTS_CUDA(cudaGraphLaunch(b->exec[0], ctx->stream));
    POTTS_CUDA(cudaEventRecord(b->ev[2], ctx->stream));
    POTTS_CUDA(cudaGraphLaunch(b->exec[1], ctx->stream));
    POTTS_CUDA(cudaEventRecord(b->ev[3], ctx->stream));
    POTTS_CUDA(cudaGraphLaunch(b->exec[2], ctx->stream));
    POTTS_CUDA(cudaEventRecord(b->ev[1], ctx->stream));
    if (!stats) return POTTS_OK;
    POTTS_TRY(check_device_error(ctx));
    float ms = 0.0f, lms = 0.0f;
    POTTS_CUDA(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
    POTTS_CUDA(cudaEventElapsedTime(&lms, b->ev[2], b->ev[3]));
    stats->n_slabs = (int)b->vols.size();
    stats->slab_w = 0;
    stats->iters = b->iters;
    stats->solve_ms = ms;
    stats->loop_ms = lms;
    stats->loop_launches = b->loop_launches;
    stats->loop_iters = b->iters > 1 ? b->iters - 1 : 0;
    stats->total_launches = b->graph_launches;
    stats->state_bytes = b->state_bytes;
    stats->dq_last = 0.0f;
    if (b->dq.p && b->iters > 0) {
        std::vector<float> all((size_t)b->iters * b->vols.size());
        POTTS_CUDA(cudaMemcpy(all.data(), b->dq.p, sizeof(float) * all.size(), cudaMemcpyDeviceToHost));
        std::vector<float> mx((size_t)b->iters, 0.0f);
        for (size_t v = 0; v < b->vols.size(); ++v)
            for (int i = 0; i < b->iters; ++i) mx[(size_t)i] = std::max(mx[(size_t)i], all[v * b->iters + i]);
        stats->dq_last = std::sqrt(mx.back());
        if (stats->dq_trace) std::memcpy(stats->dq_trace, mx.data(), sizeof(float) * mx.size());
    }
    return POTTS_OK;
}

int potts_batch_get_info(const potts_batch *b, potts_batch_info *info)
{
    if (!b || !info) return fail(POTTS_EINVAL, "batch or info is NULL");
    info->n_volumes = (int)b->vols.size();
    info->n_work = b->n_work;
    info->tile_rows = b->tile.rows;
    info->tile_slices = b->tile.slices;
    info->tile_vpt = b->tile.vpt;
    info->segment_cols = b->tile.segment;
    info->voxels = b->voxels;
    info->state_bytes = b->state_bytes;
    info->graph_launches = b->graph_launches;
    info->autotune_ms = b->autotune_ms;
    info->persistent = b->opts.persistent;
    return POTTS_OK;
}

int potts_batch_read_dq(potts_batch *b, float *host)
{
    if (!b || !host) return fail(POTTS_EINVAL, "batch or host is NULL");
    if (!b->dq.p) return fail(POTTS_EINVAL, "the batch was created without track_dq");
    POTTS_CUDA(cudaSetDevice(b->ctx->device));
    POTTS_CUDA(cudaStreamSynchronize(b->ctx->stream));
    POTTS_CUDA(cudaMemcpy(host, b->dq.p, sizeof(float) * (size_t)b->iters * b->vols.size(), cudaMemcpyDeviceToHost));
    return POTTS_OK;
}

void potts_batch_destroy(potts_batch *b) { batch_free(b); }

int potts_forward_ckpt(potts_context *ctx, const potts_mapping *map, const float *d_u, const uint8_t *d_truth, int K,
                       const float *ci, float lambda, float tau1, float tau2, int iters, int ckpt_every, float eps,
                       float *d_V, double *loss, potts_tape **out)
{
    if (!out) return fail(POTTS_EINVAL, "out is NULL");
    *out = nullptr;
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    potts_options o;
    potts_default_options(&o);
    POTTS_TRY(check_params(K, ci, lambda, tau1, tau2, iters, o));
    if (!d_u || !d_truth) return fail(POTTS_EINVAL, "u or truth is NULL");
    if (ckpt_every <= 0) return fail(POTTS_EINVAL, "ckpt_every must be >= 1");
    if (!(eps > 0.0f) || !std::isfinite(eps)) return fail(POTTS_EINVAL, "eps must be positive");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    auto *t = new potts_tape();
    t->ctx = ctx;
    int rc = copy_mapping(map, t->mc);
    if (rc == POTTS_OK) {
        t->K = K;
        t->iters = iters;
        t->every = std::min(ckpt_every, std::max(iters, 1));
        t->n_ckpt = (iters + t->every - 1) / t->every + 1;
        t->tau1 = tau1;
        t->tau2 = tau2;
        t->lambda = lambda;
        t->eps = eps;
        for (int i = 0; i < K; ++i) t->c[i] = ci[i];
        t->d_u = d_u;
        t->d_truth = d_truth;
        const potts_mapping &m = t->mc.m;
        t->g.n_lines = t->mc.n_lines;
        t->g.nstride_w = (int)get_stride(m.n_images);
        t->g.plane_w = t->mc.n_lines * (int64_t)t->g.nstride_w;
        t->g.nstride_in = (int)m.nstride;
        t->g.ns = (int)m.n_images;
        t->g.slab_start = 0;
        uint64_t vox = (uint64_t)t->mc.n_lines * m.n_images;
        t->inv_count = vox > 0 ? 1.0 / (double)vox : 0.0;
        rc = ensure(ctx, t->lines, sizeof(int4) * (size_t)std::max<int64_t>(t->mc.n_lines, 1));
        if (rc == POTTS_OK && t->mc.n_lines > 0 &&
            cudaMemcpy(t->lines.p, t->mc.lines.data(), sizeof(int4) * t->mc.n_lines, cudaMemcpyHostToDevice) !=
                cudaSuccess)
            rc = fail(POTTS_ECUDA, "copying the line table failed");
        t->g.lines = static_cast<const int4 *>(t->lines.p);
    }
    if (rc == POTTS_OK) rc = tape_alloc(t);
    if (rc == POTTS_OK && t->mc.n_lines > 0) {
        switch (K) {
        case 2: rc = tape_forward<2>(t, d_V, loss); break;
        case 3: rc = tape_forward<3>(t, d_V, loss); break;
        case 4: rc = tape_forward<4>(t, d_V, loss); break;
        case 5: rc = tape_forward<5>(t, d_V, loss); break;
        case 6: rc = tape_forward<6>(t, d_V, loss); break;
        }
    } else if (rc == POTTS_OK && loss) {
        *loss = 0.0;
    }
    if (rc != POTTS_OK) {
        const std::string msg = g_last_error;
        tape_free(t);
        g_last_error = msg;
        return rc;
    }
    *out = t;
    return POTTS_OK;
}

int potts_backward(potts_tape *t, float *d_grad_u, double *grad_ci, double *grad_lambda)
{
    if (!t || !d_grad_u) return fail(POTTS_EINVAL, "tape or grad_u is NULL");
    POTTS_CUDA(cudaSetDevice(t->ctx->device));
    if (t->mc.n_lines == 0) {
        if (grad_lambda) *grad_lambda = 0.0;
        if (grad_ci)
            for (int i = 0; i < t->K; ++i) grad_ci[i] = 0.0;
        return POTTS_OK;
    }
    switch (t->K) {
    case 2: return tape_backward<2>(t, d_grad_u, grad_ci, grad_lambda);
    case 3: return tape_backward<3>(t, d_grad_u, grad_ci, grad_lambda);
    case 4: return tape_backward<4>(t, d_grad_u, grad_ci, grad_lambda);
    case 5: return tape_backward<5>(t, d_grad_u, grad_ci, grad_lambda);
    case 6: return tape_backward<6>(t, d_grad_u, grad_ci, grad_lambda);
    }
    return fail(POTTS_EINVAL, "K must be in [2, 6]");
}

void potts_tape_destroy(potts_tape *t) { tape_free(t); }


int potts_tv_denoise(potts_context *ctx, const potts_mapping *map, float *d_g, float lambda, float tau, int iters,
                     int variant, potts_stats *stats)
{
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    if (!d_g) return fail(POTTS_EINVAL, "g is NULL");
    if (!std::isfinite(lambda) || lambda == 0.0f || !std::isfinite(tau))
        return fail(POTTS_EINVAL, "lambda must be finite and non-zero, tau finite");
    if (iters < 0) return fail(POTTS_EINVAL, "iters must be >= 0");
    if (variant < 0 || variant > 2) return fail(POTTS_EINVAL, "unknown variant");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_TRY(upload_lines(ctx, map));
    return tv_run(ctx, d_g, lambda, tau, iters, variant, stats);
}

int potts_min_max(potts_context *ctx, const potts_mapping *map, const float *d_field, float *out_min, float *out_max)
{
    if (!ctx || !map || !d_field || !out_min || !out_max) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_TRY(upload_lines(ctx, map));
    return minmax_run(ctx, d_field, false, out_min, out_max);
}

int potts_min_max_positive(potts_context *ctx, const potts_mapping *map, const float *d_field, float *out_min,
                           float *out_max)
{
    if (!ctx || !map || !d_field || !out_min || !out_max) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_TRY(upload_lines(ctx, map));
    return minmax_run(ctx, d_field, true, out_min, out_max);
}

int potts_grad_magn(potts_context *ctx, const potts_mapping *map, const float *d_u, float *d_v)
{
    if (!ctx || !map || !d_u || !d_v) return fail(POTTS_EINVAL, "NULL argument");
    if (d_u == d_v) return fail(POTTS_EINVAL, "u and v must be different fields");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_TRY(upload_lines(ctx, map));
    return grad_magn_run(ctx, d_u, d_v);
}

int potts_calc_hist(potts_context *ctx, const potts_mapping *map, const float *d_field, float range_start,
                    float range_end, uint32_t nbins, float jitter, uint64_t seed, uint32_t *out_counts,
                    double *out_density)
{
    if (!ctx || !map || !d_field || !out_counts) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_TRY(check_nbins(nbins));
    if (!std::isfinite(jitter) || jitter < 0.0f) return fail(POTTS_EINVAL, "jitter must be finite and >= 0");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_TRY(upload_lines(ctx, map));
    POTTS_TRY(hist1d_run(ctx, d_field, range_start, range_end, (int)nbins, jitter, seed, out_counts));
    if (out_density) {
        // calc_hist.cpp:129-135: counts / (in-mask voxels x bin width), in double
        const double bin_width = ((double)range_end - (double)range_start) / nbins;
        const double voxels = (double)ctx->mapping.n_lines * (double)ctx->mapping.m.n_images;
        const double scale = 1.0 / (voxels * bin_width);
        for (uint32_t i = 0; i < nbins; ++i) out_density[i] = out_counts[i] * scale;
    }
    return POTTS_OK;
}

int potts_calc_hist_auto(potts_context *ctx, const potts_mapping *map, const float *d_field, uint32_t nbins,
                         float jitter, uint64_t seed, uint32_t *out_counts, double *out_density, float *out_min,
                         float *out_max)
{
    if (!ctx || !map || !d_field || !out_counts || !out_min || !out_max) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_TRY(check_nbins(nbins));
    POTTS_TRY(potts_min_max(ctx, map, d_field, out_min, out_max));
    return potts_calc_hist(ctx, map, d_field, *out_min, *out_max, nbins, jitter, seed, out_counts, out_density);
}

uint32_t potts_uv_hist_stride(uint32_t nbins) { return nbins ? uv_stride((int)nbins) : 0u; }

uint64_t potts_uv_hist_span(uint32_t nbins) { return nbins ? uv_span((int)nbins) : 0u; }

int potts_uv_hist(potts_context *ctx, const potts_mapping *map, const float *d_u, const float *d_v, float u_start,
                  float u_end, float v_start, float v_end, uint32_t nbins, uint32_t *out_hist)
{
    if (!ctx || !map || !d_u || !d_v || !out_hist) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_TRY(check_nbins(nbins));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_TRY(upload_lines(ctx, map));
    const potts::UvRange r{u_start, u_end, v_start, v_end, (int)nbins, (int)uv_stride((int)nbins)};
    return uv_hist_run(ctx, d_u, d_v, r, out_hist);
}

int potts_uv_hist_auto(potts_context *ctx, const potts_mapping *map, const float *d_u, const float *d_v,
                       uint32_t nbins, uint32_t *out_hist, float *out_ranges)
{
    if (!ctx || !map || !d_u || !d_v || !out_hist || !out_ranges) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_TRY(check_nbins(nbins));
    // uv-hist-kernel.cpp:70-98: v over its strictly positive values, u over all (one pass)
    POTTS_CUDA(cudaSetDevice(ctx->device));
    POTTS_TRY(upload_lines(ctx, map));
    POTTS_TRY(minmax_pair_run(ctx, d_u, d_v, out_ranges));
    return potts_uv_hist(ctx, map, d_u, d_v, out_ranges[0], out_ranges[1], out_ranges[2], out_ranges[3], nbins,
                         out_hist);
}

int potts_archive_read_header(const uint8_t *bytes, uint64_t n_bytes, int elem, potts_archive_info *info,
                              uint32_t *start_row, uint32_t *base)
{
    const int bits = elem_bits_of(elem);
    if (!bits) return fail(POTTS_EINVAL, "unknown element type");
    ArchiveHeader h;
    POTTS_TRY(decode_header(bytes, n_bytes, bits, h));
    fill_info(h, info);
    if (start_row) std::memcpy(start_row, h.mc.start_row.data(), sizeof(uint32_t) * h.mc.m.cols);
    if (base) std::memcpy(base, h.mc.base.data(), sizeof(uint32_t) * ((size_t)h.mc.m.cols + 1));
    return POTTS_OK;
}

int potts_archive_size(const potts_mapping *map, int elem, uint64_t *total_bytes, uint64_t *header_bits)
{
    const int bits = elem_bits_of(elem);
    if (!bits) return fail(POTTS_EINVAL, "unknown element type");
    POTTS_TRY(validate_mapping(map));
    BitWriter w;
    encode_header(*map, bits, 0.0f, 0.0f, w);
    const uint64_t voxels = (uint64_t)(map->base[map->cols] / map->nstride) * map->n_images;
    if (total_bytes) *total_bytes = (w.bits + voxels * (uint64_t)bits + 7) / 8;
    if (header_bits) *header_bits = w.bits;
    return POTTS_OK;
}

int potts_archive_load(potts_context *ctx, const uint8_t *bytes, uint64_t n_bytes, int elem, void *d_field,
                       uint64_t capacity, potts_archive_info *info, potts_io_stats *stats)
{
    io_stats_reset(stats);
    const int bits = elem_bits_of(elem);
    if (!ctx || !d_field) return fail(POTTS_EINVAL, "NULL argument");
    if (!bits) return fail(POTTS_EINVAL, "unknown element type");
    POTTS_CUDA(cudaSetDevice(ctx->device));
    return archive_load_run(ctx, bytes, n_bytes, bits, d_field, capacity, info, stats);
}

int potts_archive_save(potts_context *ctx, const potts_mapping *map, int elem, const void *d_field, float lo,
                       float hi, uint8_t *out, uint64_t capacity, uint64_t *out_bytes, potts_io_stats *stats)
{
    io_stats_reset(stats);
    const int bits = elem_bits_of(elem);
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    if (!bits) return fail(POTTS_EINVAL, "unknown element type");
    POTTS_TRY(validate_mapping(map));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    return archive_save_run(ctx, map, bits, d_field, lo, hi, out, capacity, out_bytes, stats);
}

int potts_convert_to_fp(potts_context *ctx, const potts_mapping *map, int elem, const void *d_in, float lo, float hi,
                        float *d_out)
{
    const int bits = elem_bits_of(elem);
    if (!ctx || !d_in || !d_out) return fail(POTTS_EINVAL, "NULL argument");
    if (!bits) return fail(POTTS_EINVAL, "unknown element type");
    if (bits == 32 && d_in == (const void *)d_out) return fail(POTTS_EINVAL, "input and output must differ");
    POTTS_TRY(validate_mapping(map));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    return convert_to_fp_run(ctx, map, bits, d_in, lo, hi, d_out);
}

int potts_find_intensity_range(potts_context *ctx, const potts_mapping *map, const uint16_t *d_field,
                               double tail_thr, uint16_t *out_lo, uint16_t *out_hi, uint64_t *out_hist)
{
    if (!ctx || !d_field || !out_lo || !out_hi) return fail(POTTS_EINVAL, "NULL argument");
    if (!std::isfinite(tail_thr)) return fail(POTTS_EINVAL, "tail_thr must be finite");
    POTTS_TRY(validate_mapping(map));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    return intensity_range_run(ctx, map, d_field, tail_thr, out_lo, out_hi, out_hist);
}

int potts_raw_labels_dims(const potts_mapping *map, uint32_t *slices, uint32_t *rows, uint32_t *cols,
                          uint32_t *row_begin)
{
    POTTS_TRY(validate_mapping(map));
    uint32_t rb = 0, r = 0, c = 0;
    POTTS_TRY(raw_box_dims(*map, &rb, &r, &c));
    if (slices) *slices = map->n_images;
    if (rows) *rows = r;
    if (cols) *cols = c;
    if (row_begin) *row_begin = rb;
    return POTTS_OK;
}

int potts_raw_labels(potts_context *ctx, const potts_mapping *map, const float *d_field, uint8_t *d_box)
{
    if (!ctx || !d_field || !d_box) return fail(POTTS_EINVAL, "NULL argument");
    POTTS_TRY(validate_mapping(map));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    return raw_box_run(ctx, map, d_field, d_box);
}

int potts_vtk_labels(potts_context *ctx, const potts_mapping *map, const float *d_field, uint8_t *out,
                     uint64_t capacity, uint64_t *out_bytes, potts_io_stats *stats)
{
    io_stats_reset(stats);
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    POTTS_TRY(validate_mapping(map));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    return vtk_labels_run(ctx, map, d_field, out, capacity, out_bytes, stats);
}

int potts_png_slice(potts_context *ctx, const potts_mapping *map, const float *d_field, uint32_t col, uint8_t *out,
                    uint64_t capacity, uint64_t *out_bytes)
{
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    POTTS_TRY(validate_mapping(map));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    return png_slice_run(ctx, map, d_field, col, out, capacity, out_bytes);
}

int potts_shard_partition(const potts_mapping *map, int world, uint32_t *cuts)
{
    if (!cuts) return fail(POTTS_EINVAL, "cuts is NULL");
    POTTS_TRY(validate_mapping(map));
    return shard_partition(*map, world, cuts);
}

int potts_shard_bounds(const potts_mapping *map, const uint32_t *cuts, int world, int rank, uint32_t *cols,
                       uint64_t *span)
{
    POTTS_TRY(validate_mapping(map));
    ShardColumns sc;
    POTTS_TRY(shard_columns(*map, cuts, world, rank, &sc));
    if (cols) {
        cols[0] = sc.first;
        cols[1] = sc.last;
        cols[2] = sc.own_begin;
        cols[3] = sc.own_end;
    }
    if (span) {
        span[0] = map->base[sc.first];
        span[1] = map->base[sc.last];
    }
    return POTTS_OK;
}

int potts_shard_create(potts_context *ctx, const potts_mapping *map, const uint32_t *cuts, int world, int rank,
                       const float *d_u, int K, const float *ci, float lambda, float tau1, float tau2,
                       const potts_options *opts, potts_shard **out)
{
    if (!out) return fail(POTTS_EINVAL, "out is NULL");
    *out = nullptr;
    if (!ctx) return fail(POTTS_EINVAL, "context is NULL");
    potts_options o;
    potts_default_options(&o);
    if (opts) o = *opts;
    return shard_create(ctx, map, cuts, world, rank, d_u, K, ci, lambda, tau1, tau2, o, out);
}

int potts_shard_link(potts_shard *left, potts_shard *right)
{
    if (!left || !right) return fail(POTTS_EINVAL, "shard is NULL");
    if (left->ctx != right->ctx) return fail(POTTS_EINVAL, "linked shards share one context");
    if (left->world != right->world || right->rank != left->rank + 1)
        return fail(POTTS_EINVAL, "only neighbouring ranks are linked");
    if (left->nccl || right->nccl) return fail(POTTS_EINVAL, "a shard on NCCL is not linked");
    left->right = right;
    right->left = left;
    return POTTS_OK;
}

int potts_nccl_unique_id(void *id)
{
    if (!id) return fail(POTTS_EINVAL, "id is NULL");
    const NcclApi *api;
    POTTS_TRY(nccl_api(&api));
    ncclUniqueId u;
    POTTS_NCCL(api, api->GetUniqueId(&u));
    std::memcpy(id, &u, sizeof(u));
    return POTTS_OK;
}

int potts_nccl_comm_create(const void *id, int world, int rank, int device, void **comm)
{
    if (!id || !comm) return fail(POTTS_EINVAL, "id or comm is NULL");
    *comm = nullptr;
    if (world < 1 || rank < 0 || rank >= world) return fail(POTTS_EINVAL, "rank must be in [0, world)");
    const NcclApi *api;
    POTTS_TRY(nccl_api(&api));
    POTTS_CUDA(cudaSetDevice(device));
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    ncclComm_t c = nullptr;
    POTTS_NCCL(api, api->CommInitRank(&c, world, u, rank));
    *comm = c;
    return POTTS_OK;
}

int potts_nccl_comm_destroy(void *comm)
{
    if (!comm) return POTTS_OK;
    const NcclApi *api;
    POTTS_TRY(nccl_api(&api));
    POTTS_NCCL(api, api->CommDestroy(static_cast<ncclComm_t>(comm)));
    return POTTS_OK;
}

int potts_shard_set_nccl(potts_shard *s, void *comm)
{
    if (!s || !comm) return fail(POTTS_EINVAL, "shard or comm is NULL");
    if (s->left || s->right) return fail(POTTS_EINVAL, "a linked shard does not use NCCL");
    const NcclApi *api;
    POTTS_TRY(nccl_api(&api));
    int count = 0, rank = -1;
    POTTS_NCCL(api, api->CommCount(static_cast<ncclComm_t>(comm), &count));
    POTTS_NCCL(api, api->CommUserRank(static_cast<ncclComm_t>(comm), &rank));
    if (count != s->world || rank != s->rank)
        return fail(POTTS_EINVAL, "the communicator's size and rank differ from the shard's");
    s->nccl = static_cast<ncclComm_t>(comm);
    return POTTS_OK;
}

int potts_shard_solve(potts_shard *const *shards, int n, int iters, float *const *d_res, uint8_t *const *d_labels,
                      float *const *d_V, potts_stats *stats)
{
    POTTS_TRY(shard_check(shards, n, iters));
    POTTS_CUDA(cudaSetDevice(shards[0]->ctx->device));
    switch (shards[0]->opts.storage) {
    case POTTS_STORE_BF16: return shard_solve_store<__nv_bfloat16>(shards, n, iters, d_res, d_labels, d_V, stats);
    case POTTS_STORE_F16: return shard_solve_store<__half>(shards, n, iters, d_res, d_labels, d_V, stats);
    default: return shard_solve_store<float>(shards, n, iters, d_res, d_labels, d_V, stats);
    }
}

void potts_shard_destroy(potts_shard *s) { shard_free(s); }

}  // extern "C"
