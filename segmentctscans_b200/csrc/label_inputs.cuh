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

// grad_magn (grad-magn/grad_magn.cpp:60-79): v at every in-mask voxel.
int grad_magn_run(potts_context *ctx, const float *d_u, float *d_v)
{
    const Geometry g = field_geometry(ctx);
    if (field_empty(g)) return POTTS_OK;
    potts::grad_magn_kernel<<<field_blocks(ctx, g.n_lines, 8), potts::kHistThreads, 0, ctx->stream>>>(g, d_u, d_v);
    ctx->total_launches += 1;
    POTTS_CUDA(cudaGetLastError());
    return POTTS_OK;
}

constexpr int kHist1dSharedMax = 50 * 1024;  // bins kept in shared memory (200 KB)

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
            const int smem = (int)sizeof(uint32_t) * nb;
            const int per_sm = std::max(1, std::min(8, (200 * 1024) / std::max(smem, 1)));
            const unsigned blocks = field_blocks(ctx, g.n_lines, per_sm);
            if (jitter) {
                POTTS_CUDA(cudaFuncSetAttribute(potts::hist1d_kernel<true>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
                potts::hist1d_kernel<true><<<blocks, potts::kHistThreads, smem, ctx->stream>>>(g, d_f, rs, re, nb,
                                                                                             delta, seed, d_counts);
            } else {
                POTTS_CUDA(cudaFuncSetAttribute(potts::hist1d_kernel<false>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
                potts::hist1d_kernel<false><<<blocks, potts::kHistThreads, smem, ctx->stream>>>(g, d_f, rs, re, nb,
                                                                                              delta, seed, d_counts);
            }
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

// uv_hist (uv-hist-kernel.cpp:100-197): the 2-D histogram of (u, v) to the host.
int uv_hist_run(potts_context *ctx, const float *d_u, const float *d_v, const potts::UvRange &r, uint32_t *h_hist)
{
    const Geometry g = field_geometry(ctx);
    const uint64_t span = uv_span(r.nb);
    POTTS_TRY(ensure(ctx, ctx->hist, sizeof(uint32_t) * span));
    uint32_t *d_hist = static_cast<uint32_t *>(ctx->hist.p);
    POTTS_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(uint32_t) * span, ctx->stream));
    if (!field_empty(g)) {
        if (span <= (uint64_t)potts::kUvCluster * potts::kUvSlice) {
            const int smem = (int)sizeof(uint32_t) * potts::kUvSlice;
            POTTS_CUDA(cudaFuncSetAttribute(potts::uv_hist_cluster_kernel,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            // one block per multiprocessor: as many whole clusters as fit at once
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3((unsigned)(std::max(ctx->n_sm, 1) / potts::kUvCluster * potts::kUvCluster));
            cfg.blockDim = dim3(potts::kUvThreads);
            cfg.dynamicSmemBytes = (size_t)smem;
            cfg.stream = ctx->stream;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, (void *)potts::uv_hist_cluster_kernel, &cfg) != cudaSuccess ||
                clusters < 1) {
                cudaGetLastError();
                clusters = 1;
            }
            const unsigned blocks = (unsigned)(clusters * potts::kUvCluster);
            potts::uv_hist_cluster_kernel<<<blocks, potts::kUvThreads, smem, ctx->stream>>>(g, d_u, d_v, r, (int)span,
                                                                                           d_hist);
        } else {
            potts::uv_hist_global_kernel<<<field_blocks(ctx, g.n_lines, 8), potts::kHistThreads, 0, ctx->stream>>>(
                g, d_u, d_v, r, d_hist);
        }
        ctx->total_launches += 1;
        POTTS_CUDA(cudaGetLastError());
    }
    POTTS_CUDA(cudaMemcpyAsync(h_hist, d_hist, sizeof(uint32_t) * span, cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return POTTS_OK;
}

int check_nbins(uint32_t nbins)
{
    if (nbins < 1 || nbins > 65535) return fail(POTTS_EINVAL, "nbins must be in [1, 65535]");
    return POTTS_OK;
}
