// Host side of the label-finding inputs (kernels_hist.cuh): min/max, gradient
// magnitude, 1-D and 2-D histograms of fields laid out like the context's
// mapping.  Included by potts_b200.cu inside its internal namespace.
#pragma once

// Geometry of a whole field of the context's mapping (one slab: every slice).
Geometry field_geometry(const potts_context *ctx)
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
    return g;
}

// Blocks of a line-strided field kernel: `per_sm` per multiprocessor, at most one per line.
unsigned field_blocks(const potts_context *ctx, int64_t n_lines, int per_sm)
{
    const int64_t want = (int64_t)std::max(ctx->n_sm, 1) * per_sm;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(n_lines, want));
}

bool field_empty(const Geometry &g) { return g.n_lines == 0 || g.ns == 0; }

// 16-byte loads along a line: lines of a multiple of 4 values and stride, aligned field.
bool field_vec(const Geometry &g, const float *d_f)
{
    return ((uintptr_t)d_f & 15u) == 0 && g.ns % 4 == 0 && g.nstride_w % 4 == 0;
}

// min_max (min_max/min_max.cpp:56-81) and, with positive, the min/max of the strictly positive
// values (uv-hist-kernel.cpp:70-92).  FLT_MAX / -FLT_MAX when there is no such value.
int minmax_run(potts_context *ctx, const float *d_f, bool positive, float *out_min, float *out_max)
{
    const Geometry g = field_geometry(ctx);
    float res[2] = {FLT_MAX, -FLT_MAX};
    if (!field_empty(g)) {
        const unsigned nb = field_blocks(ctx, g.n_lines, 8);
        POTTS_TRY(ensure(ctx, ctx->hist, sizeof(float2) * nb + 2 * sizeof(float)));
        float2 *part = static_cast<float2 *>(ctx->hist.p);
        float *d_res = reinterpret_cast<float *>(part + nb);
        const bool vec = ((uintptr_t)d_f & 15u) == 0 && g.ns % 4 == 0 && g.nstride_w % 4 == 0;
        if (positive && vec)
            potts::minmax_partial_kernel<true, true><<<nb, potts::kHistThreads, 0, ctx->stream>>>(g, d_f, part);
        else if (positive)
            potts::minmax_partial_kernel<true, false><<<nb, potts::kHistThreads, 0, ctx->stream>>>(g, d_f, part);
        else if (vec)
            potts::minmax_partial_kernel<false, true><<<nb, potts::kHistThreads, 0, ctx->stream>>>(g, d_f, part);
        else
            potts::minmax_partial_kernel<false, false><<<nb, potts::kHistThreads, 0, ctx->stream>>>(g, d_f, part);
        potts::minmax_final_kernel<<<1, potts::kHistThreads, 0, ctx->stream>>>(part, (int)nb, d_res);
        ctx->total_launches += 2;
        POTTS_CUDA(cudaGetLastError());
        POTTS_CUDA(cudaMemcpyAsync(res, d_res, sizeof(res), cudaMemcpyDeviceToHost, ctx->stream));
        POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    *out_min = res[0];
    *out_max = res[1];
    return POTTS_OK;
}

// The ranges of uv_hist_auto in one pass: out = (min u, max u, min v, max v) over every u and the
// strictly positive v (uv-hist-kernel.cpp:70-98); FLT_MAX / -FLT_MAX where there is no value.
int minmax_pair_run(potts_context *ctx, const float *d_u, const float *d_v, float *out)
{
    const Geometry g = field_geometry(ctx);
    float res[4] = {FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX};
    if (!field_empty(g)) {
        const unsigned nb = field_blocks(ctx, g.n_lines, 8);
        POTTS_TRY(ensure(ctx, ctx->hist, sizeof(float4) * nb + 4 * sizeof(float)));
        float4 *part = static_cast<float4 *>(ctx->hist.p);
        float *d_res = reinterpret_cast<float *>(part + nb);
        if (field_vec(g, d_u) && field_vec(g, d_v))
            potts::minmax_pair_partial_kernel<true><<<nb, potts::kHistThreads, 0, ctx->stream>>>(g, d_u, d_v, part);
        else
            potts::minmax_pair_partial_kernel<false><<<nb, potts::kHistThreads, 0, ctx->stream>>>(g, d_u, d_v, part);
        potts::minmax_pair_final_kernel<<<1, potts::kHistThreads, 0, ctx->stream>>>(part, (int)nb, d_res);
        ctx->total_launches += 2;
        POTTS_CUDA(cudaGetLastError());
        POTTS_CUDA(cudaMemcpyAsync(res, d_res, sizeof(res), cudaMemcpyDeviceToHost, ctx->stream));
        POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    std::copy(res, res + 4, out);
    return POTTS_OK;
}

// The column march of grad_magn_tiled_kernel over the work items of GmTile tiles: one TMA box
// of u per column plane; waits for the stream to report a device-side wait that gave up.
int grad_magn_tiled(potts_context *ctx, const Geometry &g, const float *d_u, float *d_v)
{
    using T = potts::GmTile;
    // segments of 64 columns; of 16 when 64 leave fewer than four blocks per multiprocessor (decided
    // once per mapping and slice count)
    if (ctx->gm_segment == 0 || ctx->gm_ns != g.ns) {
        const size_t items = work_items(ctx->mapping.m, g.ns, TileChoice{T::TR, T::TN, 1, 64}).size();
        ctx->gm_segment = items < (size_t)4 * std::max(ctx->n_sm, 1) ? 16 : 64;
        ctx->gm_ns = g.ns;
    }
    POTTS_TRY(plan_tiles(ctx, g.ns, TileChoice{T::TR, T::TN, 1, ctx->gm_segment}));
    if (ctx->n_work == 0) return POTTS_OK;
    POTTS_TRY(ensure(ctx, ctx->err, sizeof(int)));
    CUtensorMap map;
    const uint64_t dims[2] = {(uint64_t)g.nstride_w, (uint64_t)g.n_lines};
    const uint64_t strides[1] = {sizeof(float) * (uint64_t)g.nstride_w};
    const uint32_t box[2] = {(uint32_t)T::XS, (uint32_t)T::XR};
    POTTS_TRY(encode_map(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, d_u, 2, dims, strides, box));
    POTTS_CUDA(cudaFuncSetAttribute(potts::grad_magn_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    T::SMEM_BYTES));
    POTTS_CUDA(cudaMemsetAsync(ctx->err.p, 0, sizeof(int), ctx->stream));
    const MappingCopy &mc = ctx->mapping;
    potts::grad_magn_tiled_kernel<<<ctx->n_work, potts::kGmThreads, T::SMEM_BYTES, ctx->stream>>>(
        g, static_cast<const int4 *>(ctx->cols.p), (int)mc.m.col_begin, (int)mc.m.col_end,
        static_cast<const int4 *>(ctx->work.p), map, d_v, (int *)ctx->err.p);
    ctx->total_launches += 1;
    POTTS_CUDA(cudaGetLastError());
    return check_device_error(ctx);
}

// grad_magn (grad-magn/grad_magn.cpp:60-79): v at every in-mask voxel.  Fields of 16-byte lines
// and stride march along the columns (grad_magn_tiled: 0.76 ms at 768^2 x 1024 against 1.09 ms
// for one warp per line with 16-byte loads of the line and its four neighbour lines, which
// waited on those loads); others take one thread per voxel.
int grad_magn_run(potts_context *ctx, const float *d_u, float *d_v)
{
    const Geometry g = field_geometry(ctx);
    if (field_empty(g)) return POTTS_OK;
    if (field_vec(g, d_u) && field_vec(g, d_v)) return grad_magn_tiled(ctx, g, d_u, d_v);
    potts::grad_magn_kernel<<<field_blocks(ctx, g.n_lines, 8), potts::kHistThreads, 0, ctx->stream>>>(g, d_u, d_v);
    ctx->total_launches += 1;
    POTTS_CUDA(cudaGetLastError());
    return POTTS_OK;
}

constexpr int kHist1dSharedMax = 50 * 1024;  // bins kept in shared memory (200 KB)
constexpr int kHist1dPerWarpMax = 100 * 1024;  // shared bytes of per-warp copies (two blocks per SM)

// calc_hist (calc_hist/calc_hist.cpp:93-138): counts of nb bins over [rs, re] to the host.
int hist1d_run(potts_context *ctx, const float *d_f, float rs, float re, int nb, float delta, uint64_t seed,
               uint32_t *h_counts)
{
    const Geometry g = field_geometry(ctx);
    POTTS_TRY(ensure(ctx, ctx->hist, sizeof(uint32_t) * nb));
    uint32_t *d_counts = static_cast<uint32_t *>(ctx->hist.p);
    POTTS_CUDA(cudaMemsetAsync(d_counts, 0, sizeof(uint32_t) * nb, ctx->stream));
    if (!field_empty(g)) {
        const bool jitter = delta != 0.0f;
        if (nb <= kHist1dSharedMax) {
            // a copy per warp while the copies fit 100 KB (at most 3200 bins), else one per block
            const int warps = potts::kHistThreads / 32;
            const int copies = (size_t)sizeof(uint32_t) * nb * warps <= (size_t)kHist1dPerWarpMax ? warps : 1;
            const int smem = (int)sizeof(uint32_t) * nb * copies;
            const int per_sm = std::max(1, std::min(8, (200 * 1024) / std::max(smem, 1)));
            // one warp per line
            const unsigned blocks = field_blocks(ctx, (g.n_lines + 7) / 8, per_sm);
            const bool vec = field_vec(g, d_f);
            auto launch = [&](auto kern) -> int {
                POTTS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
                kern<<<blocks, potts::kHistThreads, smem, ctx->stream>>>(g, d_f, rs, re, nb, copies, delta, seed,
                                                                         d_counts);
                return POTTS_OK;
            };
            if (jitter)
                POTTS_TRY(vec ? launch(potts::hist1d_kernel<true, true>) : launch(potts::hist1d_kernel<true, false>));
            else
                POTTS_TRY(vec ? launch(potts::hist1d_kernel<false, true>) : launch(potts::hist1d_kernel<false, false>));
        } else {
            const unsigned blocks = field_blocks(ctx, g.n_lines, 8);
            if (jitter)
                potts::hist1d_global_kernel<true><<<blocks, potts::kHistThreads, 0, ctx->stream>>>(
                    g, d_f, rs, re, nb, delta, seed, d_counts);
            else
                potts::hist1d_global_kernel<false><<<blocks, potts::kHistThreads, 0, ctx->stream>>>(
                    g, d_f, rs, re, nb, delta, seed, d_counts);
        }
        ctx->total_launches += 1;
        POTTS_CUDA(cudaGetLastError());
    }
    POTTS_CUDA(cudaMemcpyAsync(h_counts, d_counts, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return POTTS_OK;
}

// Row stride and span of the 2-D histogram (uv-hist-kernel.cpp:112-118): rows padded to 128 bytes.
uint32_t uv_stride(int nb) { return (uint32_t)((nb + 31) / 32 * 32); }
uint64_t uv_span(int nb) { return (uint64_t)(nb - 1) * uv_stride(nb) + (uint64_t)nb; }

// The 2-D histogram through the hot-cell kernels (kernels_hist.cuh): a coarse pass over every
// 8th line, the densest cells to shared memory, the rest to global atomics.
int uv_hist_hot(potts_context *ctx, const Geometry &g, const float *d_u, const float *d_v, const potts::UvRange &r,
                uint32_t *d_hist)
{
    int cs = 0;
    while (((r.nb + (1 << cs) - 1) >> cs) > potts::kUvCoarseMax) ++cs;
    const int cdim = (r.nb + (1 << cs) - 1) >> cs;
    const int cells = cdim * cdim;
    const int n_slots = std::min(cells, potts::kUvHotBins >> (2 * cs));
    // device: coarse counts (cells uint32), cell -> slot table (cells int16), slot -> cell (n_slots int16)
    const size_t bytes = sizeof(uint32_t) * cells + sizeof(int16_t) * (cells + n_slots) + 16;
    POTTS_TRY(ensure(ctx, ctx->hist_aux, bytes));
    uint32_t *d_coarse = static_cast<uint32_t *>(ctx->hist_aux.p);
    int16_t *d_table = reinterpret_cast<int16_t *>(d_coarse + cells);
    int16_t *d_cells = d_table + cells;
    POTTS_CUDA(cudaMemsetAsync(d_coarse, 0, sizeof(uint32_t) * cells, ctx->stream));
    // every step-th line, at least 4096 lines where the field has them (the cell ranking needs no
    // more; which cells get slots changes only the speed)
    const int step = (int)std::min<int64_t>(32, std::max<int64_t>(1, g.n_lines / 4096));
    const bool vec = field_vec(g, d_u) && field_vec(g, d_v);
    const unsigned cblocks = field_blocks(ctx, ((g.n_lines + step - 1) / step + 7) / 8, 8);
    if (vec)
        potts::uv_coarse_kernel<true><<<cblocks, potts::kHistThreads, 0, ctx->stream>>>(g, d_u, d_v, r, cs, cdim,
                                                                                       step, d_coarse);
    else
        potts::uv_coarse_kernel<false><<<cblocks, potts::kHistThreads, 0, ctx->stream>>>(g, d_u, d_v, r, cs, cdim,
                                                                                        step, d_coarse);
    ctx->total_launches += 1;
    POTTS_CUDA(cudaGetLastError());
    std::vector<uint32_t> counts((size_t)cells);
    POTTS_CUDA(cudaMemcpyAsync(counts.data(), d_coarse, sizeof(uint32_t) * cells, cudaMemcpyDeviceToHost,
                               ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<int> order((size_t)cells);
    for (int i = 0; i < cells; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return counts[(size_t)a] > counts[(size_t)b]; });
    std::vector<int16_t> table((size_t)cells, (int16_t)-1), slot_cell((size_t)std::max(n_slots, 1), (int16_t)0);
    for (int s = 0; s < n_slots; ++s) {
        table[(size_t)order[(size_t)s]] = (int16_t)s;
        slot_cell[(size_t)s] = (int16_t)order[(size_t)s];
    }
    POTTS_CUDA(cudaMemcpyAsync(d_table, table.data(), sizeof(int16_t) * cells, cudaMemcpyHostToDevice, ctx->stream));
    POTTS_CUDA(cudaMemcpyAsync(d_cells, slot_cell.data(), sizeof(int16_t) * n_slots, cudaMemcpyHostToDevice,
                               ctx->stream));
    const int smem = (int)(sizeof(uint32_t) * ((size_t)n_slots << (2 * cs)) + sizeof(int16_t) * cells);
    auto hot = vec ? potts::uv_hist_hot_kernel<true> : potts::uv_hist_hot_kernel<false>;
    POTTS_CUDA(cudaFuncSetAttribute(hot, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const unsigned hblocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(std::max(ctx->n_sm, 1), (g.n_lines + potts::kUvThreads / 32 - 1) / (potts::kUvThreads / 32)));
    hot<<<hblocks, potts::kUvThreads, smem, ctx->stream>>>(g, d_u, d_v, r, cs, cdim, d_table, d_cells, n_slots,
                                                           d_hist);
    ctx->total_launches += 1;
    POTTS_CUDA(cudaGetLastError());
    // the host vectors above are pageable: wait for the copies before they go out of scope
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return POTTS_OK;
}

// uv_hist (uv-hist-kernel.cpp:100-197): the 2-D histogram of (u, v) to the host.
int uv_hist_run(potts_context *ctx, const float *d_u, const float *d_v, const potts::UvRange &r, uint32_t *h_hist)
{
    const Geometry g = field_geometry(ctx);
    const uint64_t span = uv_span(r.nb);
    POTTS_TRY(ensure(ctx, ctx->hist, sizeof(uint32_t) * span));
    uint32_t *d_hist = static_cast<uint32_t *>(ctx->hist.p);
    POTTS_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(uint32_t) * span, ctx->stream));
    if (!field_empty(g)) POTTS_TRY(uv_hist_hot(ctx, g, d_u, d_v, r, d_hist));
    POTTS_CUDA(cudaMemcpyAsync(h_hist, d_hist, sizeof(uint32_t) * span, cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return POTTS_OK;
}

int check_nbins(uint32_t nbins)
{
    if (nbins < 1 || nbins > 65535) return fail(POTTS_EINVAL, "nbins must be in [1, 65535]");
    return POTTS_OK;
}
