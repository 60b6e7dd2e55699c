// Column sharding of one volume (potts_shard_*): the sharded form of the
// iteration driver potts-min-partition.cpp:625-660.  The volume's columns are
// split into contiguous ranges (one per shard: a rank with its own GPU, or
// several shards held by one process), and every shard runs the fused
// iteration on its columns plus halo columns:
//
//   a-1        the left neighbour's last column: the primal step at a needs
//              Xi^m there (the backward difference along col);
//   b, b+1     the right neighbour's first two columns: the dual step at b-1
//              needs Vbar^m at b, and the primal step at b (computed here,
//              it needs Xi^m at b and b-1, V^{m-1} and u at b, and the row
//              range of column b+1 for its mask) gives that Vbar and V^m(b).
//
// A fused launch over the columns [a, b+1) turns (Xi^m, V^{m-1}) into
// (Xi^{m+1}, V^m) exactly on [a, b) and V^m exactly on b; Xi^{m+1} on b and
// on a-1 comes from the neighbours after the launch (one column of the Xi
// planes each way), and nothing else crosses.  The set-up's dual step is
// exact on [a-1, b] without an exchange (V^0 is local).  So every owned voxel
// goes through the operations of the single-volume fused solve and gets its
// bits; the convergence trace is the max and the FP64 energies the sums over
// the shards (potts-min-partition.cpp:648-659 prints the max; the energies
// are this library's diagnostic).  Included by potts_b200.cu inside its
// internal namespace.
#pragma once

// NCCL entry points, resolved at run time from the libnccl.so.2 that the
// process has loaded already (PyTorch's) or from the system's.
struct NcclApi {
    ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*CommCount)(const ncclComm_t, int *) = nullptr;
    ncclResult_t (*CommUserRank)(const ncclComm_t, int *) = nullptr;
    ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

int nccl_api(const NcclApi **out)
{
    static NcclApi api;
    static int status = -1;  // -1 not tried, else POTTS_OK or the failure
    static std::string why;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (status < 0) {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW);
        if (!h) {
            status = POTTS_ENODEV;
            why = std::string("NCCL is not available: ") + dlerror();
        } else {
            bool ok = true;
            auto get = [&](auto &fn, const char *name) {
                fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
                ok = ok && fn != nullptr;
            };
            get(api.GetUniqueId, "ncclGetUniqueId");
            get(api.CommInitRank, "ncclCommInitRank");
            get(api.CommDestroy, "ncclCommDestroy");
            get(api.CommCount, "ncclCommCount");
            get(api.CommUserRank, "ncclCommUserRank");
            get(api.Send, "ncclSend");
            get(api.Recv, "ncclRecv");
            get(api.GroupStart, "ncclGroupStart");
            get(api.GroupEnd, "ncclGroupEnd");
            get(api.AllReduce, "ncclAllReduce");
            get(api.GetErrorString, "ncclGetErrorString");
            status = ok ? POTTS_OK : POTTS_ENODEV;
            if (!ok) why = "libnccl.so.2 lacks an entry point this library uses";
        }
    }
    if (status != POTTS_OK) return fail(status, why);
    *out = &api;
    return POTTS_OK;
}

#define POTTS_NCCL(api, call)                                                                           \
    do {                                                                                                \
        ncclResult_t r_ = (call);                                                                       \
        if (r_ != ncclSuccess) return fail(POTTS_ECUDA, std::string("NCCL: ") + (api)->GetErrorString(r_)); \
    } while (0)

// Global columns of shard `rank`: held [first, last), owned [own_begin, own_end).
struct ShardColumns {
    uint32_t first, last, own_begin, own_end;
};

int shard_columns(const potts_mapping &m, const uint32_t *cuts, int world, int rank, ShardColumns *sc)
{
    if (!cuts) return fail(POTTS_EINVAL, "cuts is NULL");
    if (world < 1 || rank < 0 || rank >= world) return fail(POTTS_EINVAL, "rank must be in [0, world)");
    if (cuts[0] != m.col_begin || cuts[world] != m.col_end)
        return fail(POTTS_EINVAL, "cuts must start at col_begin and end at col_end");
    for (int r = 0; r < world; ++r)
        if (cuts[r + 1] <= cuts[r]) return fail(POTTS_EINVAL, "every shard needs at least one column");
    sc->own_begin = cuts[rank];
    sc->own_end = cuts[rank + 1];
    sc->first = rank > 0 ? sc->own_begin - 1 : sc->own_begin;
    sc->last = rank + 1 < world ? std::min<uint32_t>(sc->own_end + 2, m.col_end) : sc->own_end;
    return POTTS_OK;
}

}  // namespace

struct potts_shard {
    potts_context *ctx = nullptr;
    MappingCopy mc;  // the local volume: global columns [first, last) renumbered from 0
    ShardColumns sc{};
    int rank = 0, world = 1;
    int K = 0;
    float tau1 = 0.0f, tau2 = 0.0f, lambda = 0.0f;
    float c[POTTS_MAX_PHASES] = {};
    potts_options opts{};
    const float *d_u = nullptr;  // local u, in the local mapping's layout
    int64_t line_base = 0;       // global line of local line 0
    int64_t own_line_begin = 0, own_line_end = 0;
    DevBuf lines, cols, state, work, vol, dq, energy, ustage;
    TileChoice tile{};
    int n_work = 0;
    size_t state_bytes = 0;
    potts_shard *left = nullptr, *right = nullptr;  // neighbours held by this process
    ncclComm_t nccl = nullptr;                      // or the communicator of all ranks
};

namespace {

void shard_free(potts_shard *s)
{
    if (!s) return;
    if (s->ctx) {
        cudaSetDevice(s->ctx->device);
        cudaStreamSynchronize(s->ctx->stream);
    }
    if (s->left) s->left->right = nullptr;
    if (s->right) s->right->left = nullptr;
    for (DevBuf *d : {&s->lines, &s->cols, &s->state, &s->work, &s->vol, &s->dq, &s->energy, &s->ustage})
        if (d->p) cudaFree(d->p);
    delete s;
}

// Split [col_begin, col_end) into `world` ranges of about equal in-mask voxels
// (cuts at the prefix sums), each at least one column.
int shard_partition(const potts_mapping &m, int world, uint32_t *cuts)
{
    const uint32_t lo = m.col_begin, hi = m.col_end;
    if (world < 1 || hi - lo < (uint32_t)world)
        return fail(POTTS_EINVAL, "cannot split the active columns over that many shards");
    std::vector<double> cum(hi - lo + 1, 0.0);
    for (uint32_t c = lo; c < hi; ++c)
        cum[c - lo + 1] = cum[c - lo] + (double)((m.base[c + 1] - m.base[c]) / m.nstride) * m.n_images;
    cuts[0] = lo;
    for (int r = 1; r < world; ++r) {
        const double target = cum.back() * r / world;
        uint32_t c = lo + (uint32_t)(std::lower_bound(cum.begin(), cum.end(), target) - cum.begin());
        c = std::max(c, cuts[r - 1] + 1);
        c = std::min(c, hi - (uint32_t)(world - r));
        cuts[r] = c;
    }
    cuts[world] = hi;
    return POTTS_OK;
}

// The shard's local mapping: global columns [first, last) renumbered from 0.
void shard_local_mapping(const potts_mapping &m, const ShardColumns &sc, potts_mapping *lm,
                         std::vector<uint32_t> &start_row, std::vector<uint32_t> &base)
{
    const uint32_t cols = sc.last - sc.first;
    start_row.assign(m.start_row + sc.first, m.start_row + sc.last);
    base.resize(cols + 1);
    for (uint32_t c = 0; c <= cols; ++c) base[c] = m.base[sc.first + c] - m.base[sc.first];
    *lm = m;
    lm->cols = cols;
    lm->col_begin = 0;
    lm->col_end = cols;
    lm->start_row = start_row.data();
    lm->base = base.data();
}

inline uint32_t shard_local_col(const potts_shard *s, uint32_t global_col) { return global_col - s->sc.first; }

// Lines [L0, L1) of local column c.
inline void shard_col_lines(const potts_shard *s, uint32_t c, int64_t *L0, int64_t *L1)
{
    const potts_mapping &m = s->mc.m;
    *L0 = m.base[c] / m.nstride;
    *L1 = m.base[c + 1] / m.nstride;
}

template <typename ST>
SlabState<ST> shard_state(const potts_shard *s, const Geometry &g)
{
    ST *base = static_cast<ST *>(s->state.p);
    const size_t xi_planes = 3 * (size_t)(s->K - 1), v_planes = (size_t)(s->K - 1);
    SlabState<ST> st;
    st.xi[0] = base;
    st.xi[1] = base + xi_planes * g.plane_w;
    st.v[0] = st.xi[1] + xi_planes * g.plane_w;
    st.v[1] = st.v[0] + v_planes * g.plane_w;
    return st;
}

Geometry shard_geometry(const potts_shard *s)
{
    Geometry g{};
    const potts_mapping &m = s->mc.m;
    g.lines = static_cast<const int4 *>(s->lines.p);
    g.n_lines = s->mc.n_lines;
    g.nstride_w = (int)get_stride(m.n_images);
    g.plane_w = g.n_lines * (int64_t)g.nstride_w;
    g.nstride_in = (int)m.nstride;
    g.ns = (int)m.n_images;
    g.slab_start = 0;
    g.line_begin = 0;
    g.line_base = s->line_base;
    return g;
}

size_t store_bytes(int storage) { return storage == POTTS_STORE_F32 ? 4 : 2; }

template <typename ST>
int choose_tile_k(int K, const potts_options &o, TileChoice *tc)
{
    switch (K) {
    case 2: return choose_tile<2, ST>(o, tc);
    case 3: return choose_tile<3, ST>(o, tc);
    case 4: return choose_tile<4, ST>(o, tc);
    case 5: return choose_tile<5, ST>(o, tc);
    case 6: return choose_tile<6, ST>(o, tc);
    }
    return fail(POTTS_EINVAL, "K must be in [2, 6]");
}

int shard_create(potts_context *ctx, const potts_mapping *map, const uint32_t *cuts, int world, int rank,
                 const float *d_u, int K, const float *ci, float lambda, float tau1, float tau2,
                 const potts_options &o, potts_shard **out)
{
    POTTS_TRY(check_params(K, ci, lambda, tau1, tau2, 0, o));
    if (!d_u) return fail(POTTS_EINVAL, "u is NULL");
    if (o.variant != POTTS_VARIANT_FUSED) return fail(POTTS_EINVAL, "shards run the fused form");
    if (o.storage == POTTS_STORE_F64) return fail(POTTS_EINVAL, "shards store FP32, bfloat16 or binary16");
    if (o.sync_monitor) return fail(POTTS_EINVAL, "shards keep the monitor on the device (sync_monitor = 0)");
    POTTS_TRY(validate_mapping(map));
    ShardColumns sc;
    POTTS_TRY(shard_columns(*map, cuts, world, rank, &sc));
    POTTS_CUDA(cudaSetDevice(ctx->device));
    std::unique_ptr<potts_shard, void (*)(potts_shard *)> s(new potts_shard(), shard_free);
    s->ctx = ctx;
    s->sc = sc;
    s->rank = rank;
    s->world = world;
    s->K = K;
    s->tau1 = tau1;
    s->tau2 = tau2;
    s->lambda = lambda;
    for (int i = 0; i < K; ++i) s->c[i] = ci[i];
    s->opts = o;
    s->d_u = d_u;
    potts_mapping lm;
    std::vector<uint32_t> sr, bs;
    shard_local_mapping(*map, sc, &lm, sr, bs);
    POTTS_TRY(copy_mapping(&lm, s->mc));
    s->line_base = map->base[sc.first] / map->nstride;
    int64_t l0, l1;
    shard_col_lines(s.get(), shard_local_col(s.get(), sc.own_begin), &l0, &l1);
    s->own_line_begin = l0;
    shard_col_lines(s.get(), shard_local_col(s.get(), sc.own_end - 1), &l0, &l1);
    s->own_line_end = l1;
    const int64_t n_lines = s->mc.n_lines;
    POTTS_TRY(ensure(ctx, s->lines, sizeof(int4) * (size_t)std::max<int64_t>(n_lines, 1)));
    if (n_lines > 0)
        POTTS_CUDA(cudaMemcpy(s->lines.p, s->mc.lines.data(), sizeof(int4) * n_lines, cudaMemcpyHostToDevice));
    const std::vector<int4> cols = column_table(s->mc.m);
    POTTS_TRY(ensure(ctx, s->cols, sizeof(int4) * cols.size()));
    POTTS_CUDA(cudaMemcpy(s->cols.p, cols.data(), sizeof(int4) * cols.size(), cudaMemcpyHostToDevice));
    // tile and work items: the owned columns and, with a right neighbour, its first column
    // (the primal step there gives Vbar and V at b; see the top of this file)
    switch (o.storage) {
    case POTTS_STORE_BF16: POTTS_TRY(choose_tile_k<__nv_bfloat16>(K, o, &s->tile)); break;
    case POTTS_STORE_F16: POTTS_TRY(choose_tile_k<__half>(K, o, &s->tile)); break;
    default: POTTS_TRY(choose_tile_k<float>(K, o, &s->tile)); break;
    }
    const uint32_t a = shard_local_col(s.get(), sc.own_begin);
    const uint32_t b1 = std::min<uint32_t>(shard_local_col(s.get(), sc.own_end) + 1, s->mc.m.cols);
    const std::vector<int4> work = work_items(s->mc.m, (int)lm.n_images, s->tile, (int)a, (int)b1);
    POTTS_TRY(ensure(ctx, s->work, sizeof(int4) * std::max<size_t>(work.size(), 1)));
    if (!work.empty())
        POTTS_CUDA(cudaMemcpy(s->work.p, work.data(), sizeof(int4) * work.size(), cudaMemcpyHostToDevice));
    s->n_work = (int)work.size();
    const Geometry g = shard_geometry(s.get());
    s->state_bytes = store_bytes(o.storage) * 8 * (size_t)(K - 1) * (size_t)std::max<int64_t>(g.plane_w, 1);
    if (g.plane_w >= (int64_t(1) << 31))
        return fail(POTTS_EINVAL, "a shard of 2^31 state voxels or more: use more shards");
    POTTS_TRY(ensure(ctx, s->state, s->state_bytes));
    *out = s.release();
    return POTTS_OK;
}

// Pointer to the Xi planes of local column c in half h, and the column's bytes per plane.
template <typename ST>
ST *shard_col_xi(const potts_shard *s, int h, uint32_t c, size_t *bytes)
{
    const Geometry g = shard_geometry(s);
    int64_t L0, L1;
    shard_col_lines(s, c, &L0, &L1);
    *bytes = sizeof(ST) * (size_t)(L1 - L0) * (size_t)g.nstride_w;
    return shard_state<ST>(s, g).xi[h] + L0 * g.nstride_w;
}

// After a launch: Xi^{m+1} (state half h) of the boundary columns goes to the
// neighbours' halo columns, by NCCL between ranks or by device copies between
// shards of this process, all on the context's stream.
template <typename ST>
int shard_exchange(potts_shard *const *sh, int n, int h)
{
    potts_context *ctx = sh[0]->ctx;
    const NcclApi *api = nullptr;
    const bool nccl = sh[0]->nccl != nullptr;
    if (nccl) {
        POTTS_TRY(nccl_api(&api));
        POTTS_NCCL(api, api->GroupStart());
    }
    for (int i = 0; i < n; ++i) {
        potts_shard *s = sh[i];
        const int planes = 3 * (s->K - 1);
        const int64_t pw = shard_geometry(s).plane_w;
        size_t bytes = 0;
        if (nccl) {
            // the left neighbour holds our first owned column as its right halo and
            // sends its last owned column for our left halo (local column 0);
            // the right neighbour the other way round
            struct Side {
                int peer;
                uint32_t send_col, recv_col;
            } sides[2];
            int ns = 0;
            if (s->rank > 0) sides[ns++] = {s->rank - 1, shard_local_col(s, s->sc.own_begin), 0u};
            if (s->rank + 1 < s->world)
                sides[ns++] = {s->rank + 1, shard_local_col(s, s->sc.own_end - 1), shard_local_col(s, s->sc.own_end)};
            for (int k = 0; k < ns; ++k) {
                ST *src = shard_col_xi<ST>(s, h, sides[k].send_col, &bytes);
                size_t rbytes = 0;
                ST *dst = shard_col_xi<ST>(s, h, sides[k].recv_col, &rbytes);
                for (int p = 0; p < planes; ++p) {
                    POTTS_NCCL(api, api->Send(src + p * pw, bytes, ncclUint8, sides[k].peer, s->nccl, ctx->stream));
                    POTTS_NCCL(api, api->Recv(dst + p * pw, rbytes, ncclUint8, sides[k].peer, s->nccl, ctx->stream));
                }
            }
        } else if (s->right) {
            potts_shard *r = s->right;
            const int64_t rpw = shard_geometry(r).plane_w;
            // our last owned column -> the right shard's left halo (its local column 0)
            ST *src = shard_col_xi<ST>(s, h, shard_local_col(s, s->sc.own_end - 1), &bytes);
            size_t b2 = 0;
            ST *dst = shard_col_xi<ST>(r, h, 0u, &b2);
            if (bytes != b2) return fail(POTTS_EINVAL, "linked shards disagree on a column");
            if (bytes > 0)
                POTTS_CUDA(cudaMemcpy2DAsync(dst, sizeof(ST) * rpw, src, sizeof(ST) * pw, bytes, planes,
                                             cudaMemcpyDeviceToDevice, ctx->stream));
            // the right shard's first owned column -> our right halo
            src = shard_col_xi<ST>(r, h, shard_local_col(r, r->sc.own_begin), &bytes);
            dst = shard_col_xi<ST>(s, h, shard_local_col(s, s->sc.own_end), &b2);
            if (bytes != b2) return fail(POTTS_EINVAL, "linked shards disagree on a column");
            if (bytes > 0)
                POTTS_CUDA(cudaMemcpy2DAsync(dst, sizeof(ST) * pw, src, sizeof(ST) * rpw, bytes, planes,
                                             cudaMemcpyDeviceToDevice, ctx->stream));
        }
    }
    if (nccl) POTTS_NCCL(api, api->GroupEnd());
    return POTTS_OK;
}

template <int K, typename ST>
int shard_solve_k(potts_shard *const *sh, int n, int iters, float *const *d_res, uint8_t *const *d_labels,
                  float *const *d_V, potts_stats *stats)
{
    potts_context *ctx = sh[0]->ctx;
    cudaStream_t st = ctx->stream;
    const potts_options &o = sh[0]->opts;
    const bool fast = o.arith == POTTS_ARITH_FAST;
    const int ge = o.gap_every;
    const int n_en = ge > 0 ? iters / ge : 0;
    ctx->seg_used = 0;
    ctx->seg_open = false;
    ctx->loop_launches = ctx->total_launches = ctx->loop_iters = 0;
    POTTS_TRY(ensure(ctx, ctx->err, sizeof(int)));
    POTTS_CUDA(cudaMemsetAsync(ctx->err.p, 0, sizeof(int), st));
    POTTS_CUDA(cudaEventRecord(ctx->ev0, st));
    std::vector<Geometry> g(n), gown(n);
    std::vector<SlabState<ST>> ss(n);
    std::vector<PhaseParams<K>> pp(n);
    for (int i = 0; i < n; ++i) {
        potts_shard *s = sh[i];
        g[i] = shard_geometry(s);
        gown[i] = g[i];
        gown[i].line_begin = s->own_line_begin;
        gown[i].n_lines = s->own_line_end;
        if (ge > 0)  // the energies' partial sums (one pair per block), allocated before the loop
            POTTS_TRY(ensure(ctx, ctx->partial, sizeof(double2) * (size_t)std::max(plain_blocks(gown[i], 0, g[i].ns), 1u)));
        ss[i] = shard_state<ST>(s, g[i]);
        for (int k = 0; k < K; ++k) pp[i].c[k] = s->c[k];
        pp[i].lam = s->lambda;
        pp[i].tau1 = s->tau1;
        POTTS_TRY(ensure(ctx, s->dq, sizeof(float) * (size_t)std::max(iters, 1)));
        POTTS_TRY(ensure(ctx, s->energy, sizeof(double) * 3 * (size_t)std::max(n_en, 1)));
        POTTS_CUDA(cudaMemsetAsync(s->dq.p, 0, sizeof(float) * (size_t)std::max(iters, 1), st));
        POTTS_CUDA(cudaMemsetAsync(s->energy.p, 0, sizeof(double) * 3 * (size_t)std::max(n_en, 1), st));
        // the fused kernel reads (and multiplies by zero) padding and stale halos: all of it finite
        POTTS_CUDA(cudaMemsetAsync(s->state.p, 0, s->state_bytes, st));
        if (iters > 1) {
            const float *ubase;
            uint64_t ustride;
            int ux0;
            POTTS_TRY(fused_u_source(ctx, g[i], s->d_u, s->ustage, &ubase, &ustride, &ux0));
            potts::FusedVolume<K, ST> vol;
            const ST *xs[2] = {ss[i].xi[0], ss[i].xi[1]}, *vs[2] = {ss[i].v[0], ss[i].v[1]};
            POTTS_TRY((build_volume<K, ST>(g[i], static_cast<const int4 *>(s->cols.p), 0, (int)s->mc.m.cols, xs, vs,
                                           ubase, ustride, ux0, s->tile, pp[i], static_cast<float *>(s->dq.p),
                                           o.prefetch, &vol)));
            vol.tp.line_base = s->line_base;
            POTTS_TRY(ensure(ctx, s->vol, sizeof(vol)));
            // pageable source: the call returns once the bytes are staged
            POTTS_CUDA(cudaMemcpyAsync(s->vol.p, &vol, sizeof(vol), cudaMemcpyHostToDevice, st));
        }
        if (g[i].n_lines == 0) continue;
        const unsigned nb = plain_blocks(g[i], 0, g[i].ns);
        potts::init_kernel<K, ST><<<nb, potts::kPlainThreads, 0, st>>>(g[i], s->d_u, ss[i].v[0], (ST *)nullptr, pp[i]);
        ctx->total_launches += 1;
        if (iters > 0) {
            launch_dual<K, ST>(fast, nb, st, g[i], ss[i].xi[0], ss[i].v[0], s->tau2, ctx->thr);
            ctx->total_launches += 1;
        }
    }
    POTTS_CUDA(cudaGetLastError());
    int cur = 0;
    for (int m = 1; m < iters; ++m) {
        POTTS_TRY(seg_begin(ctx));
        for (int i = 0; i < n; ++i) {
            potts_shard *s = sh[i];
            POTTS_TRY((launch_tiled<K, ST>)(ctx, s->tile, fast, static_cast<const potts::FusedVolume<K, ST> *>(s->vol.p),
                                            static_cast<const int4 *>(s->work.p), nullptr, s->n_work, cur, m - 1,
                                            s->tau2));
            ctx->loop_launches += 1;
            ctx->total_launches += 1;
        }
        ctx->loop_iters += 1;
        cur ^= 1;
        POTTS_TRY(shard_exchange<ST>(sh, n, cur));
        if (ge > 0 && m % ge == 0)
            for (int i = 0; i < n; ++i)
                if (gown[i].n_lines > gown[i].line_begin)
                    POTTS_TRY(run_energy<K>(ctx, gown[i], ss[i].xi[cur ^ 1], ss[i].v[cur], sh[i]->d_u, pp[i],
                                        static_cast<double *>(sh[i]->energy.p) + 3 * (m / ge - 1)));
    }
    POTTS_TRY(seg_end(ctx));
    for (int i = 0; i < n; ++i) {
        potts_shard *s = sh[i];
        if (gown[i].n_lines <= gown[i].line_begin) continue;
        const unsigned nb = plain_blocks(gown[i], 0, gown[i].ns);
        if (iters > 0) {
            launch_primal<K, ST>(fast, nb, st, gown[i], ss[i].xi[cur], ss[i].v[cur], (ST *)nullptr, s->d_u, pp[i],
                                 static_cast<float *>(s->dq.p) + (iters - 1), iters - 1);
            ctx->total_launches += 1;
            if (ge > 0 && iters % ge == 0)
                POTTS_TRY(run_energy<K>(ctx, gown[i], ss[i].xi[cur], ss[i].v[cur], s->d_u, pp[i],
                                        static_cast<double *>(s->energy.p) + 3 * (iters / ge - 1)));
        }
        float *res = d_res ? d_res[i] : nullptr, *V = d_V ? d_V[i] : nullptr;
        uint8_t *lab = d_labels ? d_labels[i] : nullptr;
        if (res || lab || V) {
            potts::update_kernel<K, ST, float><<<nb, potts::kPlainThreads, 0, st>>>(
                gown[i], ss[i].v[cur], ss[i].xi[cur], pp[i], 0, gown[i].ns, res, lab, V, (float *)nullptr,
                (int64_t)s->mc.span);
            ctx->total_launches += 1;
        }
    }
    POTTS_CUDA(cudaGetLastError());
    // the convergence trace (max over the shards) and the energies (sums)
    const NcclApi *api = nullptr;
    if (sh[0]->nccl) {
        POTTS_TRY(nccl_api(&api));
        POTTS_NCCL(api, api->AllReduce(sh[0]->dq.p, sh[0]->dq.p, (size_t)std::max(iters, 1), ncclFloat, ncclMax,
                                       sh[0]->nccl, st));
        POTTS_NCCL(api, api->AllReduce(sh[0]->energy.p, sh[0]->energy.p, 3 * (size_t)std::max(n_en, 1), ncclDouble,
                                       ncclSum, sh[0]->nccl, st));
    }
    POTTS_CUDA(cudaEventRecord(ctx->ev1, st));
    POTTS_TRY(check_device_error(ctx));
    if (!stats) return POTTS_OK;
    std::vector<float> dq((size_t)std::max(iters, 1), 0.0f), part(dq.size());
    std::vector<double> en(3 * (size_t)std::max(n_en, 1), 0.0), epart(en.size());
    const int n_sum = sh[0]->nccl ? 1 : n;  // after the all-reduce one copy holds everything
    for (int i = 0; i < n_sum; ++i) {
        POTTS_CUDA(cudaMemcpy(part.data(), sh[i]->dq.p, sizeof(float) * part.size(), cudaMemcpyDeviceToHost));
        POTTS_CUDA(cudaMemcpy(epart.data(), sh[i]->energy.p, sizeof(double) * epart.size(), cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < dq.size(); ++k) dq[k] = std::max(dq[k], part[k]);
        for (size_t k = 0; k < en.size(); ++k) en[k] += epart[k];
    }
    for (int k = 0; k < n_en; ++k) en[3 * k + 2] = en[3 * k] - en[3 * k + 1];
    float ms = 0.0f;
    POTTS_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    stats->n_slabs = n;
    stats->slab_w = (int)sh[0]->mc.m.n_images;
    stats->iters = iters;
    stats->solve_ms = ms;
    POTTS_TRY(seg_total_ms(ctx, &stats->loop_ms));
    stats->loop_launches = ctx->loop_launches;
    stats->loop_iters = ctx->loop_iters;
    stats->total_launches = (int)ctx->total_launches;
    stats->state_bytes = 0;
    for (int i = 0; i < n; ++i) stats->state_bytes += sh[i]->state_bytes;
    stats->dq_last = iters > 0 ? std::sqrt(dq[(size_t)iters - 1]) : 0.0f;
    if (stats->dq_trace && iters > 0) std::memcpy(stats->dq_trace, dq.data(), sizeof(float) * (size_t)iters);
    if (stats->energy_trace && n_en > 0) std::memcpy(stats->energy_trace, en.data(), sizeof(double) * 3 * n_en);
    return POTTS_OK;
}

template <typename ST>
int shard_solve_store(potts_shard *const *sh, int n, int iters, float *const *r, uint8_t *const *l, float *const *v,
                      potts_stats *stats)
{
    switch (sh[0]->K) {
    case 2: return shard_solve_k<2, ST>(sh, n, iters, r, l, v, stats);
    case 3: return shard_solve_k<3, ST>(sh, n, iters, r, l, v, stats);
    case 4: return shard_solve_k<4, ST>(sh, n, iters, r, l, v, stats);
    case 5: return shard_solve_k<5, ST>(sh, n, iters, r, l, v, stats);
    case 6: return shard_solve_k<6, ST>(sh, n, iters, r, l, v, stats);
    }
    return fail(POTTS_EINVAL, "K must be in [2, 6]");
}

// The shards of one call: this process's, all on one context, with the same
// parameters; either every rank's shard linked in order (shards of one
// process), or one shard on an NCCL communicator, or a single shard.
int shard_check(potts_shard *const *sh, int n, int iters)
{
    if (!sh || n < 1) return fail(POTTS_EINVAL, "no shards");
    if (iters < 0) return fail(POTTS_EINVAL, "iters must be >= 0");
    for (int i = 0; i < n; ++i) {
        if (!sh[i]) return fail(POTTS_EINVAL, "shard is NULL");
        const potts_shard *a = sh[0], *b = sh[i];
        if (b->ctx != a->ctx) return fail(POTTS_EINVAL, "the shards of one call share one context");
        if (b->K != a->K || b->opts.storage != a->opts.storage || b->opts.arith != a->opts.arith ||
            b->opts.gap_every != a->opts.gap_every || b->world != a->world || b->mc.m.n_images != a->mc.m.n_images)
            return fail(POTTS_EINVAL, "the shards of one call need the same K, storage, arith, gap_every and volume");
    }
    if (sh[0]->nccl) {
        if (n != 1) return fail(POTTS_EINVAL, "a process runs one NCCL shard per call");
        return POTTS_OK;
    }
    if (n != sh[0]->world) return fail(POTTS_EINVAL, "without NCCL a call runs every shard of the volume");
    for (int i = 0; i < n; ++i) {
        if (sh[i]->rank != i) return fail(POTTS_EINVAL, "shards must be passed in rank order");
        if (i + 1 < n && sh[i]->right != sh[i + 1]) return fail(POTTS_EINVAL, "neighbouring shards are not linked");
    }
    return POTTS_OK;
}
