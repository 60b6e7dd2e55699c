// Batched solves: many independent volumes (own mapping, u, labels and
// lambda; common K, step sizes, iteration count and storage) planned once and
// run as captured CUDA graphs: set-up (u staging, init and first dual step of
// every volume), iterations (one persistent launch of the fused kernel that
// runs every iteration over the work items of all volumes, one volume
// descriptor each; or, with persistent = 0, one launch per iteration) and
// finish (last primal step and argmax of every volume), replayed back to back
// so that the iterations can be timed apart.  Included by potts_b200.cu inside its
// internal namespace.
#pragma once

struct BatchVolume {
    MappingCopy mc;
    Geometry g{};
    int64_t lines_off = 0, cols_off = 0;  // offsets into the batch's tables
    size_t state_off = 0;                 // byte offset of the volume's state
    bool staged = false;                  // u is copied to an aligned buffer each run
    size_t stage_off = 0;                 // float offset of that buffer
    const float *d_u = nullptr;
    float *res = nullptr, *V = nullptr;
    uint8_t *labels = nullptr;
    float c[POTTS_MAX_PHASES] = {};
    float lambda = 0.0f;
    uint64_t voxels = 0;
};

}  // namespace

struct potts_batch {
    potts_context *ctx = nullptr;
    int K = 0, storage = 0, iters = 0;
    float tau1 = 0.0f, tau2 = 0.0f;
    potts_options opts{};
    std::vector<BatchVolume> vols;
    DevBuf lines, cols, state, desc, work, work_vol, dq, ustage, pctl;
    TileChoice tile{};
    int n_work = 0;
    cudaGraph_t graph[3] = {nullptr, nullptr, nullptr};  // set-up, iterations, finish
    cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // run start/end, iterations start/end
    uint64_t voxels = 0, state_bytes = 0;
    int graph_launches = 0;
    int loop_launches = 0;  // launches of the iterations graph
    double autotune_ms = 0.0;
};

namespace {

void batch_free(potts_batch *b)
{
    if (!b) return;
    if (b->ctx) {
        cudaSetDevice(b->ctx->device);
        cudaStreamSynchronize(b->ctx->stream);
    }
    for (int i = 0; i < 3; ++i) {
        if (b->exec[i]) cudaGraphExecDestroy(b->exec[i]);
        if (b->graph[i]) cudaGraphDestroy(b->graph[i]);
    }
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    for (DevBuf *d : {&b->lines, &b->cols, &b->state, &b->desc, &b->work, &b->work_vol, &b->dq, &b->ustage,
                      &b->pctl})
        if (d->p) cudaFree(d->p);
    delete b;
}

template <int K>
PhaseParams<K> batch_params(const BatchVolume &bv, float tau1)
{
    PhaseParams<K> pp;
    for (int i = 0; i < K; ++i) pp.c[i] = bv.c[i];
    pp.lam = bv.lambda;
    pp.tau1 = tau1;
    return pp;
}

template <typename ST>
SlabState<ST> batch_state(const potts_batch *b, const BatchVolume &bv, int K)
{
    ST *base = reinterpret_cast<ST *>(static_cast<uint8_t *>(b->state.p) + bv.state_off);
    const size_t xi_planes = 3 * (size_t)(K - 1), v_planes = (size_t)(K - 1);
    SlabState<ST> st;
    st.xi[0] = base;
    st.xi[1] = base + xi_planes * bv.g.plane_w;
    st.v[0] = st.xi[1] + xi_planes * bv.g.plane_w;
    st.v[1] = st.v[0] + v_planes * bv.g.plane_w;
    return st;
}

// Work items and volume descriptors of the batch for one tile shape.
template <int K, typename ST>
int batch_plan_tiles(potts_batch *b, const TileChoice &tile)
{
    potts_context *ctx = b->ctx;
    std::vector<int4> work;
    std::vector<int> work_vol;
    std::vector<potts::FusedVolume<K, ST>> desc(b->vols.size());
    for (size_t v = 0; v < b->vols.size(); ++v) {
        const BatchVolume &bv = b->vols[v];
        const std::vector<int4> w = work_items(bv.mc.m, bv.g.ns, tile);
        work.insert(work.end(), w.begin(), w.end());
        work_vol.insert(work_vol.end(), w.size(), (int)v);
        const SlabState<ST> st = batch_state<ST>(b, bv, K);
        const ST *xs[2] = {st.xi[0], st.xi[1]}, *vs[2] = {st.v[0], st.v[1]};
        const float *ubase = bv.staged ? static_cast<const float *>(b->ustage.p) + bv.stage_off : bv.d_u;
        const uint64_t ustride = bv.staged ? (uint64_t)bv.g.nstride_w : (uint64_t)bv.g.nstride_in;
        float *dq = b->dq.p ? static_cast<float *>(b->dq.p) + v * (size_t)b->iters : nullptr;
        POTTS_TRY((build_volume<K, ST>(bv.g, static_cast<const int4 *>(b->cols.p) + bv.cols_off,
                                       (int)bv.mc.m.col_begin, (int)bv.mc.m.col_end, xs, vs, ubase, ustride, 0, tile,
                                       batch_params<K>(bv, b->tau1), dq, b->opts.prefetch, &desc[v])));
    }
    POTTS_TRY(ensure(ctx, b->work, sizeof(int4) * std::max<size_t>(work.size(), 1)));
    POTTS_TRY(ensure(ctx, b->work_vol, sizeof(int) * std::max<size_t>(work.size(), 1)));
    POTTS_TRY(ensure(ctx, b->desc, sizeof(potts::FusedVolume<K, ST>) * desc.size()));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (!work.empty()) {
        POTTS_CUDA(cudaMemcpy(b->work.p, work.data(), sizeof(int4) * work.size(), cudaMemcpyHostToDevice));
        POTTS_CUDA(cudaMemcpy(b->work_vol.p, work_vol.data(), sizeof(int) * work.size(), cudaMemcpyHostToDevice));
    }
    POTTS_CUDA(cudaMemcpy(b->desc.p, desc.data(), sizeof(potts::FusedVolume<K, ST>) * desc.size(),
                          cudaMemcpyHostToDevice));
    b->n_work = (int)work.size();
    b->tile = tile;
    return POTTS_OK;
}

// Everything before the iteration launches: u staging, zeroed state, init
// and the first dual step of every volume.
template <int K, typename ST>
int batch_enqueue_head(potts_batch *b)
{
    potts_context *ctx = b->ctx;
    cudaStream_t s = ctx->stream;
    POTTS_CUDA(cudaMemsetAsync(ctx->err.p, 0, sizeof(int), s));
    if (b->dq.p) POTTS_CUDA(cudaMemsetAsync(b->dq.p, 0, b->dq.bytes, s));
    POTTS_CUDA(cudaMemsetAsync(b->state.p, 0, b->state_bytes, s));
    for (const BatchVolume &bv : b->vols) {
        if (bv.g.n_lines == 0) continue;
        const unsigned nb = plain_blocks(bv.g, 0, bv.g.ns);
        if (bv.staged) {
            potts::stage_u_kernel<<<nb, potts::kPlainThreads, 0, s>>>(bv.g, bv.d_u,
                                                                       static_cast<float *>(b->ustage.p) + bv.stage_off);
            ctx->total_launches += 1;
        }
        const SlabState<ST> st = batch_state<ST>(b, bv, K);
        potts::init_kernel<K, ST><<<nb, potts::kPlainThreads, 0, s>>>(bv.g, bv.d_u, st.v[0], (ST *)nullptr,
                                                                      batch_params<K>(bv, b->tau1));
        ctx->total_launches += 1;
        if (b->iters > 0) {
            launch_dual<K, ST>(b->opts.arith == POTTS_ARITH_FAST, nb, s, bv.g, st.xi[0], st.v[0], b->tau2, ctx->thr);
            ctx->total_launches += 1;
        }
    }
    POTTS_CUDA(cudaGetLastError());
    return POTTS_OK;
}

template <int K, typename ST>
int batch_enqueue_tail(potts_batch *b, int cur)
{
    potts_context *ctx = b->ctx;
    cudaStream_t s = ctx->stream;
    for (size_t v = 0; v < b->vols.size(); ++v) {
        const BatchVolume &bv = b->vols[v];
        if (bv.g.n_lines == 0) continue;
        const unsigned nb = plain_blocks(bv.g, 0, bv.g.ns);
        const SlabState<ST> st = batch_state<ST>(b, bv, K);
        const PhaseParams<K> pp = batch_params<K>(bv, b->tau1);
        if (b->iters > 0) {
            float *dq = b->dq.p ? static_cast<float *>(b->dq.p) + v * (size_t)b->iters + (b->iters - 1) : nullptr;
            launch_primal<K, ST>(b->opts.arith == POTTS_ARITH_FAST, nb, s, bv.g, st.xi[cur], st.v[cur],
                                 (ST *)nullptr, bv.d_u, pp, dq, b->iters - 1);
            ctx->total_launches += 1;
        }
        if (bv.res || bv.labels || bv.V) {
            potts::update_kernel<K, ST><<<nb, potts::kPlainThreads, 0, s>>>(
                bv.g, st.v[cur], st.xi[cur], pp, 0, bv.g.ns, bv.res, bv.labels, bv.V, nullptr,
                (int64_t)bv.mc.span);
            ctx->total_launches += 1;
        }
    }
    POTTS_CUDA(cudaGetLastError());
    return POTTS_OK;
}

// Tile autotuner: time a few iterations of every compiled tile shape (and
// three segment lengths), as one launch per iteration and as the persistent
// launch, on the batch itself; keep the fastest.  The solution depends on
// neither, so the choice only changes speed.
template <int K, typename ST>
int batch_autotune(potts_batch *b, TileChoice *best, int *best_persistent)
{
    potts_context *ctx = b->ctx;
    using TS = ShapesOf<K, ST>;
    constexpr int kTrials = 3;
    cudaEvent_t e0, e1, t0, t1;
    POTTS_CUDA(cudaEventCreate(&e0));
    POTTS_CUDA(cudaEventCreate(&e1));
    POTTS_CUDA(cudaEventCreate(&t0));
    POTTS_CUDA(cudaEventCreate(&t1));
    POTTS_CUDA(cudaEventRecord(t0, ctx->stream));
    float best_ms = 0.0f;
    bool have = false;
    int rc = POTTS_OK;
    const int segments[3] = {16, 32, 64};
    for (int i = 0; i < TS::n && rc == POTTS_OK; ++i)
        for (int sgi = 0; sgi < 3 && rc == POTTS_OK; ++sgi) {
            TileChoice tc{TS::r[i], TS::t[i], TS::v[i], segments[sgi]};
            rc = batch_plan_tiles<K, ST>(b, tc);
            if (rc != POTTS_OK) break;
            rc = batch_enqueue_head<K, ST>(b);
            if (rc != POTTS_OK) break;
            const bool fast = b->opts.arith == POTTS_ARITH_FAST;
            const auto *vols = static_cast<const potts::FusedVolume<K, ST> *>(b->desc.p);
            const auto *work = static_cast<const int4 *>(b->work.p);
            const auto *work_vol = static_cast<const int *>(b->work_vol.p);
            // form 0: one launch per iteration (one untimed, then kTrials timed);
            // form 1: the persistent launch (one iteration untimed, then kTrials in one launch)
            for (int form = 0; form < 2 && rc == POTTS_OK; ++form) {
                if (form == 0) {
                    for (int m = 0; m <= kTrials && rc == POTTS_OK; ++m) {
                        if (m == 1) cudaEventRecord(e0, ctx->stream);
                        rc = launch_tiled<K, ST>(ctx, tc, fast, vols, work, work_vol, b->n_work, m & 1, m, b->tau2);
                    }
                } else {
                    rc = launch_tiled_persistent<K, ST>(ctx, b->pctl, tc, fast, vols, work, work_vol, b->n_work, 0, 0,
                                                        1, b->tau2);
                    cudaEventRecord(e0, ctx->stream);
                    if (rc == POTTS_OK)
                        rc = launch_tiled_persistent<K, ST>(ctx, b->pctl, tc, fast, vols, work, work_vol, b->n_work,
                                                            1, 1, kTrials, b->tau2);
                }
                if (rc != POTTS_OK) break;
                cudaEventRecord(e1, ctx->stream);
                if (cudaEventSynchronize(e1) != cudaSuccess) {
                    rc = fail(POTTS_ECUDA, "autotune timing failed");
                    break;
                }
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (!have || ms < best_ms) {
                    best_ms = ms;
                    *best = tc;
                    *best_persistent = form;
                    have = true;
                }
            }
        }
    cudaEventRecord(t1, ctx->stream);
    cudaEventSynchronize(t1);
    float total = 0.0f;
    cudaEventElapsedTime(&total, t0, t1);
    b->autotune_ms = total;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc == POTTS_OK) rc = check_device_error(ctx);
    return rc;
}

template <int K, typename ST>
int batch_capture(potts_batch *b, const TileChoice &tile);

template <int K, typename ST>
int batch_build(potts_batch *b)
{
    potts_context *ctx = b->ctx;
    const size_t planes = 8 * (size_t)(K - 1);
    // tables, state and staging offsets
    int64_t n_lines = 0, n_cols = 0;
    size_t state = 0, stage = 0;
    for (BatchVolume &bv : b->vols) {
        const potts_mapping &m = bv.mc.m;
        bv.g.n_lines = bv.mc.n_lines;
        bv.g.nstride_w = (int)get_stride(m.n_images);
        bv.g.plane_w = bv.mc.n_lines * (int64_t)bv.g.nstride_w;
        if (bv.g.plane_w >= (int64_t(1) << 31))
            return fail(POTTS_EINVAL, "a batch volume of 2^31 state voxels or more: solve it alone");
        bv.g.nstride_in = (int)m.nstride;
        bv.g.ns = (int)m.n_images;
        bv.g.slab_start = 0;
        bv.lines_off = n_lines;
        bv.cols_off = n_cols;
        n_lines += std::max<int64_t>(bv.mc.n_lines, 1);
        n_cols += std::max<int64_t>(m.cols, 1);
        bv.state_off = state;
        state += (sizeof(ST) * planes * (size_t)std::max<int64_t>(bv.g.plane_w, 1) + 255) / 256 * 256;
        bv.staged = m.nstride % 4 != 0 || reinterpret_cast<uintptr_t>(bv.d_u) % 16 != 0;
        bv.stage_off = stage;
        if (bv.staged) stage += ((size_t)std::max<int64_t>(bv.g.plane_w, 1) + 63) / 64 * 64;
        bv.voxels = 0;
        for (uint32_t c = m.col_begin; c < m.col_end; ++c)
            bv.voxels += (uint64_t)((m.base[c + 1] - m.base[c]) / m.nstride) * m.n_images;
        b->voxels += bv.voxels;
    }
    size_t free_b = 0, total_b = 0;
    POTTS_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (state + (size_t(512) << 20) > free_b) return fail(POTTS_ENOMEM, "the batch's state does not fit in memory");
    b->state_bytes = state;
    POTTS_TRY(ensure(ctx, b->state, state));
    POTTS_TRY(ensure(ctx, b->lines, sizeof(int4) * (size_t)n_lines));
    POTTS_TRY(ensure(ctx, b->cols, sizeof(int4) * (size_t)n_cols));
    if (stage > 0) POTTS_TRY(ensure(ctx, b->ustage, sizeof(float) * stage));
    if (b->opts.track_dq && b->iters > 0)
        POTTS_TRY(ensure(ctx, b->dq, sizeof(float) * (size_t)b->iters * b->vols.size()));
    POTTS_TRY(ensure(ctx, ctx->err, sizeof(int)));
    for (BatchVolume &bv : b->vols) {
        int4 *dl = static_cast<int4 *>(b->lines.p) + bv.lines_off;
        if (bv.mc.n_lines > 0)
            POTTS_CUDA(cudaMemcpy(dl, bv.mc.lines.data(), sizeof(int4) * bv.mc.n_lines, cudaMemcpyHostToDevice));
        bv.g.lines = dl;
        const std::vector<int4> cols = column_table(bv.mc.m);
        POTTS_CUDA(cudaMemcpy(static_cast<int4 *>(b->cols.p) + bv.cols_off, cols.data(), sizeof(int4) * cols.size(),
                              cudaMemcpyHostToDevice));
    }

    // tile shape: the options', or the autotuner's
    TileChoice tile;
    const potts_options &o = b->opts;
    if (o.autotune && o.tile_rows <= 0 && o.tile_slices <= 0 && o.tile_vpt <= 0 && o.segment_cols <= 0 &&
        b->iters > 1) {
        POTTS_TRY((batch_autotune<K, ST>(b, &tile, &b->opts.persistent)));
    } else {
        POTTS_TRY((choose_tile<K, ST>(o, &tile)));
    }
    POTTS_TRY((batch_plan_tiles<K, ST>(b, tile)));
    // the kernel's shared-memory attribute is set (and the persistent launch's
    // control words allocated) outside the capture
    POTTS_TRY((launch_tiled<K, ST>(ctx, tile, b->opts.arith == POTTS_ARITH_FAST, nullptr, nullptr, nullptr, 0, 0, 0, b->tau2)));
    if (b->opts.persistent && b->iters > 1)
        POTTS_TRY((launch_tiled_persistent<K, ST>(ctx, b->pctl, tile, b->opts.arith == POTTS_ARITH_FAST, nullptr,
                                                  nullptr, nullptr, 0, 0, 0, b->iters - 1, b->tau2)));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));

    for (cudaEvent_t &e : b->ev) POTTS_CUDA(cudaEventCreate(&e));
    // capture on a stream of our own (the context's may be the legacy default
    // stream, which cannot be captured); the graphs run on the context's
    cudaStream_t run_stream = ctx->stream, cap = nullptr;
    POTTS_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    ctx->stream = cap;
    const int rc_cap = batch_capture<K, ST>(b, tile);
    ctx->stream = run_stream;
    cudaStreamDestroy(cap);
    return rc_cap;
}

template <int K, typename ST>
int batch_capture(potts_batch *b, const TileChoice &tile)
{
    potts_context *ctx = b->ctx;
    const int64_t launches0 = ctx->total_launches;
    int cur = 0;
    for (int part = 0; part < 3; ++part) {
        POTTS_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = POTTS_OK;
        if (part == 0) {
            rc = batch_enqueue_head<K, ST>(b);
        } else if (part == 1) {
            const bool fast = b->opts.arith == POTTS_ARITH_FAST;
            const auto *vols = static_cast<const potts::FusedVolume<K, ST> *>(b->desc.p);
            const auto *work = static_cast<const int4 *>(b->work.p);
            const auto *work_vol = static_cast<const int *>(b->work_vol.p);
            if (b->opts.persistent && b->iters > 1) {
                // every iteration of every volume in one launch
                rc = launch_tiled_persistent<K, ST>(ctx, b->pctl, tile, fast, vols, work, work_vol, b->n_work, 0, 0,
                                                    b->iters - 1, b->tau2);
                ctx->total_launches += 1;
                b->loop_launches = 1;
                cur = (b->iters - 1) & 1;
            } else {
                for (int m = 1; m < b->iters && rc == POTTS_OK; ++m) {
                    rc = launch_tiled<K, ST>(ctx, tile, fast, vols, work, work_vol, b->n_work, cur, m - 1, b->tau2);
                    ctx->total_launches += 1;
                    cur ^= 1;
                }
                b->loop_launches = b->iters > 1 ? b->iters - 1 : 0;
            }
        } else {
            rc = batch_enqueue_tail<K, ST>(b, cur);
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        if (rc != POTTS_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess)
            return fail(POTTS_ECUDA, std::string("graph capture failed: ") + cudaGetErrorString(ce));
        b->graph[part] = graph;
        POTTS_CUDA(cudaGraphInstantiate(&b->exec[part], graph, 0));
    }
    b->graph_launches = (int)(ctx->total_launches - launches0);
    return POTTS_OK;
}

template <typename ST>
int batch_build_store(potts_batch *b)
{
    switch (b->K) {
    case 2: return batch_build<2, ST>(b);
    case 3: return batch_build<3, ST>(b);
    case 4: return batch_build<4, ST>(b);
    case 5: return batch_build<5, ST>(b);
    case 6: return batch_build<6, ST>(b);
    }
    return fail(POTTS_EINVAL, "K must be in [2, 6]");
}
