// Host side of the field archive, the input normalisation and the output writers
// (kernels_fieldio.cuh).  Included by potts_b200.cu inside its internal namespace.
//
// Archive format (no archive header, no class information: io::BinOArchive writes
// nothing for Boost's version/class records, include/io/binoarchive.h:27-35):
//   mapping_storage::save (include/layout_cylinder.h:233-257), Exp-Golomb codes
//     ue n_images, ue rows, ue cols, ue nstride, ue col_begin, ue col_end,
//     ue cols, ue start_row[0], se start_row[i] - start_row[i-1] (i = 1 .. cols-1),
//     ue cols + 1, ue base[0], se base[i] - base[i-1] (i = 1 .. cols)
//   Field<float> only (include/field.h:98-104): the FP32 bit patterns of lo and hi, 32 bits each
//   voxels (include/field.h:105-118): columns col_begin .. col_end-1, their rows, n = 0 .. n_images-1,
//     32 bits (FP32 bit pattern) or 16 bits (uint16) each
// all as one MSB-first bit stream (include/io/outbitstream.h:17-50); the last byte is padded with 0.
#pragma once

// MSB-first bit writer: bits fill each byte from its most significant bit down.
struct BitWriter {
    std::vector<uint8_t> bytes;
    uint64_t bits = 0;

    void put(uint64_t v, int n)  // the low n bits of v, most significant first
    {
        for (int k = n - 1; k >= 0; --k) {
            if ((bits & 7u) == 0) bytes.push_back(0);
            if ((v >> k) & 1u) bytes.back() |= (uint8_t)(0x80u >> (bits & 7u));
            ++bits;
        }
    }
    // Exp-Golomb (include/io/writeprimitives.h:55-60): m = v + 1 of b bits is sent as b - 1 zeros, then m.
    void ue(uint64_t v)
    {
        const uint64_t m = v + 1;
        const int b = 64 - __builtin_clzll(m);
        put(0, b - 1);
        put(m, b);
    }
    // Signed form (writeprimitives.h:62-66): v > 0 as 2v - 1, v <= 0 as -2v.
    void se(int64_t v) { ue(v > 0 ? 2 * (uint64_t)v - 1 : 2 * (uint64_t)(-v)); }
};

// MSB-first bit reader over a byte range; reading past the end sets `overrun`.
struct BitReader {
    const uint8_t *p = nullptr;
    uint64_t n_bits = 0, pos = 0;
    bool overrun = false;

    uint64_t get(int n)
    {
        uint64_t v = 0;
        for (int k = 0; k < n; ++k) {
            if (pos >= n_bits) {
                overrun = true;
                return 0;
            }
            v = (v << 1) | ((p[pos >> 3] >> (7 - (pos & 7u))) & 1u);
            ++pos;
        }
        return v;
    }
    // include/io/readprimitives.h:54-64
    bool ue(uint64_t &v)
    {
        int zeros = 0;
        while (get(1) == 0) {
            if (overrun || ++zeros > 63) return false;
        }
        v = zeros == 0 ? 0 : (uint64_t{1} << zeros) + get(zeros) - 1;
        return !overrun;
    }
    // readprimitives.h:66-76: even codes are -(c / 2), odd ones (c + 1) / 2
    bool se(int64_t &v)
    {
        uint64_t c = 0;
        if (!ue(c)) return false;
        v = (c & 1u) ? (int64_t)((c + 1) >> 1) : -(int64_t)(c >> 1);
        return true;
    }
};

int elem_bits_of(int elem)
{
    if (elem == POTTS_ELEM_F32) return 32;
    if (elem == POTTS_ELEM_U16) return 16;
    return 0;
}

// The archive's header bits (mapping, then lo/hi for FP32 fields).
void encode_header(const potts_mapping &m, int bits, float lo, float hi, BitWriter &w)
{
    w.ue(m.n_images);
    w.ue(m.rows);
    w.ue(m.cols);
    w.ue(m.nstride);
    w.ue(m.col_begin);
    w.ue(m.col_end);
    w.ue(m.cols);
    if (m.cols > 0) {
        w.ue(m.start_row[0]);
        for (uint32_t i = 1; i < m.cols; ++i) w.se((int64_t)m.start_row[i] - (int64_t)m.start_row[i - 1]);
    }
    w.ue((uint64_t)m.cols + 1);
    w.ue(m.base[0]);
    for (uint32_t i = 1; i <= m.cols; ++i) w.se((int64_t)m.base[i] - (int64_t)m.base[i - 1]);
    if (bits == 32) {
        uint32_t b;
        std::memcpy(&b, &lo, 4);
        w.put(b, 32);
        std::memcpy(&b, &hi, 4);
        w.put(b, 32);
    }
}

// A parsed header: the mapping (tables owned here) and where the voxels start.
struct ArchiveHeader {
    MappingCopy mc;
    float lo = 0.0f, hi = 0.0f;
    uint64_t header_bits = 0, voxels = 0, total_bytes = 0;
};

bool get_u32(BitReader &r, uint32_t &out)
{
    uint64_t v = 0;
    if (!r.ue(v) || v > 0xffffffffull) return false;
    out = (uint32_t)v;
    return true;
}

// mapping_storage::load (include/layout_cylinder.h:259-312) and Field<float>::load's lo/hi
// (include/field.h:121-131); the tables must have cols and cols + 1 entries, every value must fit
// 32 bits and the mapping must be one the library accepts.
int decode_header(const uint8_t *bytes, uint64_t n_bytes, int bits, ArchiveHeader &h)
{
    if (!bytes) return fail(POTTS_EINVAL, "archive bytes are NULL");
    if (n_bytes > (UINT64_MAX >> 3)) return fail(POTTS_EINVAL, "archive too large");
    BitReader r{bytes, n_bytes * 8};
    potts_mapping &m = h.mc.m;
    m = potts_mapping{};
    uint32_t n_start = 0;
    if (!get_u32(r, m.n_images) || !get_u32(r, m.rows) || !get_u32(r, m.cols) || !get_u32(r, m.nstride) ||
        !get_u32(r, m.col_begin) || !get_u32(r, m.col_end) || !get_u32(r, n_start))
        return fail(POTTS_EINVAL, "archive header is truncated or holds a value beyond 32 bits");
    if (n_start != m.cols) return fail(POTTS_EINVAL, "archive's start_row table does not have cols entries");
    h.mc.start_row.assign(m.cols, 0u);
    for (uint32_t i = 0; i < m.cols; ++i) {
        int64_t v = 0;
        if (i == 0) {
            uint64_t u = 0;
            if (!r.ue(u)) return fail(POTTS_EINVAL, "archive header is truncated");
            v = (int64_t)u;
        } else {
            int64_t d = 0;
            if (!r.se(d)) return fail(POTTS_EINVAL, "archive header is truncated");
            v = (int64_t)h.mc.start_row[i - 1] + d;
        }
        if (v < 0 || v > 0xffffffffll) return fail(POTTS_EINVAL, "archive start_row value beyond 32 bits");
        h.mc.start_row[i] = (uint32_t)v;
    }
    uint64_t n_base = 0;
    if (!r.ue(n_base)) return fail(POTTS_EINVAL, "archive header is truncated");
    if (n_base != (uint64_t)m.cols + 1) return fail(POTTS_EINVAL, "archive's base table does not have cols + 1 entries");
    h.mc.base.assign((size_t)m.cols + 1, 0u);
    for (uint64_t i = 0; i < n_base; ++i) {
        int64_t v = 0;
        if (i == 0) {
            uint64_t u = 0;
            if (!r.ue(u)) return fail(POTTS_EINVAL, "archive header is truncated");
            v = (int64_t)u;
        } else {
            int64_t d = 0;
            if (!r.se(d)) return fail(POTTS_EINVAL, "archive header is truncated");
            v = (int64_t)h.mc.base[i - 1] + d;
        }
        if (v < 0 || v > 0xffffffffll) return fail(POTTS_EINVAL, "archive base value beyond 32 bits");
        h.mc.base[(size_t)i] = (uint32_t)v;
    }
    if (bits == 32) {
        const uint32_t lo = (uint32_t)r.get(32), hi = (uint32_t)r.get(32);
        if (r.overrun) return fail(POTTS_EINVAL, "archive header is truncated");
        std::memcpy(&h.lo, &lo, 4);
        std::memcpy(&h.hi, &hi, 4);
    }
    h.mc.rebind();
    POTTS_TRY(validate_mapping(&h.mc.m));
    h.mc.span = m.base[m.cols];
    h.mc.n_lines = (int64_t)(h.mc.span / m.nstride);
    h.header_bits = r.pos;
    h.voxels = (uint64_t)h.mc.n_lines * m.n_images;
    h.total_bytes = (h.header_bits + h.voxels * (uint64_t)bits + 7) / 8;
    return POTTS_OK;
}

void fill_info(const ArchiveHeader &h, potts_archive_info *info)
{
    if (!info) return;
    const potts_mapping &m = h.mc.m;
    info->n_images = m.n_images;
    info->rows = m.rows;
    info->cols = m.cols;
    info->nstride = m.nstride;
    info->col_begin = m.col_begin;
    info->col_end = m.col_end;
    info->span = h.mc.span;
    info->lo = h.lo;
    info->hi = h.hi;
    info->header_bits = h.header_bits;
    info->voxels = h.voxels;
    info->total_bytes = h.total_bytes;
}

potts::IoLines io_lines(const potts_mapping &m)
{
    potts::IoLines g;
    g.n_lines = (int64_t)(m.base[m.cols] / m.nstride);
    g.ns = (int)m.n_images;
    g.nstride = (int)m.nstride;
    return g;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

// Lines of `per` voxels' worth of 16 bytes each (voxel count and stride multiples of `per`).
bool lines_vec(const potts::IoLines &g, int per) { return g.ns % per == 0 && g.nstride % per == 0; }

unsigned io_blocks(const potts_context *ctx, int64_t n_lines)
{
    const int64_t want = (int64_t)std::max(ctx->n_sm, 1) * 8;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(n_lines, want));
}

void io_stats_reset(potts_io_stats *st)
{
    if (st) *st = potts_io_stats{};
}

// Device time between the context's two events (after the stream has passed the second).
int io_stats_kernel(potts_context *ctx, potts_io_stats *st, int launches)
{
    if (!st) return POTTS_OK;
    float ms = 0.0f;
    POTTS_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    st->kernel_ms = ms;
    st->launches = launches;
    return POTTS_OK;
}

// Field<T>::load: the payload from host bytes into a device field of the archive's mapping.
int archive_load_run(potts_context *ctx, const uint8_t *bytes, uint64_t n_bytes, int bits, void *d_field,
                     uint64_t capacity, potts_archive_info *info, potts_io_stats *st)
{
    ArchiveHeader h;
    POTTS_TRY(decode_header(bytes, n_bytes, bits, h));
    fill_info(h, info);
    if (n_bytes < h.total_bytes) return fail(POTTS_EINVAL, "archive ends inside the voxel payload");
    if (capacity < h.mc.span) return fail(POTTS_EINVAL, "device field is smaller than the archive's span");
    if (h.voxels == 0) return POTTS_OK;
    const uint64_t first = h.header_bits / 8, shift = h.header_bits % 8;
    const uint64_t payload = h.total_bytes - first;
    const uint64_t staged = (payload + 15) / 16 * 16 + 16;  // whole words plus the word after the last
    POTTS_TRY(ensure(ctx, ctx->io, staged));
    uint8_t *d_words = static_cast<uint8_t *>(ctx->io.p);
    const uint64_t tail = payload & ~uint64_t{3};  // the last partial word and the words after it read as 0
    POTTS_CUDA(cudaMemsetAsync(d_words + tail, 0, staged - tail, ctx->stream));
    POTTS_CUDA(cudaMemcpyAsync(d_words, bytes + first, payload, cudaMemcpyHostToDevice, ctx->stream));
    const potts::IoLines g = io_lines(h.mc.m);
    POTTS_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    const unsigned nb = io_blocks(ctx, g.n_lines);
    const uint32_t *w = reinterpret_cast<const uint32_t *>(d_words);
    const bool vec = aligned16(d_field) && lines_vec(g, 128 / bits);
    if (bits == 32) {
        uint32_t *o = static_cast<uint32_t *>(d_field);
        if (vec)
            potts::archive_unpack_kernel<32, true><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, w, (int)shift, o);
        else
            potts::archive_unpack_kernel<32, false><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, w, (int)shift, o);
    } else {
        uint16_t *o = static_cast<uint16_t *>(d_field);
        if (vec)
            potts::archive_unpack_kernel<16, true><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, w, (int)shift, o);
        else
            potts::archive_unpack_kernel<16, false><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, w, (int)shift, o);
    }
    POTTS_CUDA(cudaGetLastError());
    POTTS_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->total_launches += 1;
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return io_stats_kernel(ctx, st, 1);
}

// Field<T>::save: the whole archive of a device field into host memory.
int archive_save_run(potts_context *ctx, const potts_mapping *map, int bits, const void *d_field, float lo, float hi,
                     uint8_t *out, uint64_t capacity, uint64_t *out_bytes, potts_io_stats *st)
{
    BitWriter w;
    encode_header(*map, bits, lo, hi, w);
    const potts::IoLines g = io_lines(*map);
    const uint64_t voxels = (uint64_t)g.n_lines * (uint64_t)g.ns;
    const uint64_t total = (w.bits + voxels * (uint64_t)bits + 7) / 8;
    if (out_bytes) *out_bytes = total;
    if (!out) return POTTS_OK;
    if (capacity < total) return fail(POTTS_EINVAL, "output buffer is smaller than the archive");
    const uint64_t first = w.bits / 8, shift = w.bits % 8;
    std::memcpy(out, w.bytes.data(), first);
    if (voxels == 0) {
        if (shift) out[first] = w.bytes[first];
        return POTTS_OK;
    }
    if (!d_field) return fail(POTTS_EINVAL, "field is NULL");
    const uint64_t payload = total - first;
    POTTS_TRY(ensure(ctx, ctx->io, (payload + 15) / 16 * 16 + 16));
    uint8_t *d_words = static_cast<uint8_t *>(ctx->io.p);
    POTTS_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    const unsigned nb = io_blocks(ctx, g.n_lines);
    if (bits == 32) {
        const uint32_t *in = static_cast<const uint32_t *>(d_field);
        uint32_t *o = reinterpret_cast<uint32_t *>(d_words);
        if (aligned16(d_field) && lines_vec(g, 4))
            potts::archive_pack_kernel<32, true><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, in, (int)shift, o);
        else
            potts::archive_pack_kernel<32, false><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, in, (int)shift, o);
    } else {
        potts::archive_pack_kernel<16, false><<<nb, potts::kIoThreads, 0, ctx->stream>>>(
            g, static_cast<const uint16_t *>(d_field), (int)shift, reinterpret_cast<uint16_t *>(d_words));
    }
    POTTS_CUDA(cudaGetLastError());
    POTTS_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->total_launches += 1;
    POTTS_CUDA(cudaMemcpyAsync(out + first, d_words, payload, cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (shift) out[first] |= w.bytes[first];  // the header's last bits share the payload's first byte
    return io_stats_kernel(ctx, st, 1);
}

int convert_to_fp_run(potts_context *ctx, const potts_mapping *map, int bits, const void *d_in, float lo, float hi,
                      float *d_out)
{
    const potts::IoLines g = io_lines(*map);
    if (g.n_lines == 0) return POTTS_OK;
    const unsigned nb = io_blocks(ctx, g.n_lines);
    const bool vec = aligned16(d_in) && aligned16(d_out) && lines_vec(g, 4);
    if (bits == 32) {
        const float *in = static_cast<const float *>(d_in);
        if (vec)
            potts::convert_to_fp_kernel<float, true><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, in, lo, hi, d_out);
        else
            potts::convert_to_fp_kernel<float, false><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, in, lo, hi, d_out);
    } else {
        const uint16_t *in = static_cast<const uint16_t *>(d_in);
        if (vec)
            potts::convert_to_fp_kernel<uint16_t, true><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, in, lo, hi, d_out);
        else
            potts::convert_to_fp_kernel<uint16_t, false><<<nb, potts::kIoThreads, 0, ctx->stream>>>(g, in, lo, hi,
                                                                                                  d_out);
    }
    ctx->total_launches += 1;
    POTTS_CUDA(cudaGetLastError());
    return POTTS_OK;
}

constexpr int kU16Bins = 65536;

// find_intensity_range (transpose/find_intensity_range.cpp:64-110): the histogram, then the first
// bin whose cumulative count reaches (1 - tail) of the total and the last one whose cumulative
// count stays at or below tail of it.
int intensity_range_run(potts_context *ctx, const potts_mapping *map, const uint16_t *d_f, double tail,
                        uint16_t *out_lo, uint16_t *out_hi, uint64_t *out_hist)
{
    const potts::IoLines g = io_lines(*map);
    POTTS_TRY(ensure(ctx, ctx->hist, sizeof(unsigned long long) * kU16Bins));
    unsigned long long *d_hist = static_cast<unsigned long long *>(ctx->hist.p);
    POTTS_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(unsigned long long) * kU16Bins, ctx->stream));
    if (g.n_lines > 0) {
        const int smem = (int)sizeof(uint32_t) * potts::kU16Slice;
        const bool vec = aligned16(d_f) && lines_vec(g, 8);
        void *kfn = vec ? (void *)potts::u16_hist_cluster_kernel<true> : (void *)potts::u16_hist_cluster_kernel<false>;
        POTTS_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)std::max(potts::kU16Cluster,
                                              std::max(ctx->n_sm, 1) / potts::kU16Cluster * potts::kU16Cluster));
        cfg.blockDim = dim3(potts::kU16Threads);
        cfg.dynamicSmemBytes = (size_t)smem;
        cfg.stream = ctx->stream;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, kfn, &cfg) != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            clusters = 1;
        }
        const int64_t want = (g.n_lines + 31) / 32;  // a warp per line in each block of a cluster
        clusters = (int)std::max<int64_t>(1, std::min<int64_t>(clusters, want));
        const unsigned blocks = (unsigned)(clusters * potts::kU16Cluster);
        if (vec)
            potts::u16_hist_cluster_kernel<true><<<blocks, potts::kU16Threads, smem, ctx->stream>>>(g, d_f, d_hist);
        else
            potts::u16_hist_cluster_kernel<false><<<blocks, potts::kU16Threads, smem, ctx->stream>>>(g, d_f, d_hist);
        ctx->total_launches += 1;
        POTTS_CUDA(cudaGetLastError());
    }
    std::vector<uint64_t> hist(kU16Bins);
    POTTS_CUDA(cudaMemcpyAsync(hist.data(), d_hist, sizeof(uint64_t) * kU16Bins, cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    uint64_t total = 0;
    for (uint64_t c : hist) total += c;
    const double pct_lo = tail * (double)total, pct_hi = (1.0 - tail) * (double)total;
    size_t lo = 0, hi = hist.size();
    uint64_t cum = 0;
    for (size_t i = 0; i < hist.size(); ++i) {
        cum += hist[i];
        if (pct_lo >= (double)cum) lo = i;
        if (pct_hi <= (double)cum) {
            hi = i;
            break;
        }
    }
    *out_lo = (uint16_t)lo;  // the reference narrows both to uint16_t
    *out_hi = (uint16_t)hi;
    if (out_hist) std::memcpy(out_hist, hist.data(), sizeof(uint64_t) * kU16Bins);
    return POTTS_OK;
}

// Extent of the raw label box (potts-model.cpp:186-196): rows from the smallest first row to the
// largest end row over the columns that hold rows, columns col_begin .. col_end-1.
int raw_box_dims(const potts_mapping &m, uint32_t *row_begin, uint32_t *rows, uint32_t *cols)
{
    if (m.col_end <= m.col_begin) return fail(POTTS_EINVAL, "the mapping holds no voxels");
    int64_t rb = INT64_MAX, re = INT64_MIN;
    for (uint32_t c = m.col_begin; c < m.col_end; ++c) {
        const int64_t cnt = (int64_t)(m.base[c + 1] - m.base[c]) / m.nstride;
        if (cnt == 0) continue;
        rb = std::min<int64_t>(rb, m.start_row[c]);
        re = std::max<int64_t>(re, (int64_t)m.start_row[c] + cnt);
    }
    if (re <= rb) return fail(POTTS_EINVAL, "the mapping holds no voxels");
    *row_begin = (uint32_t)rb;
    *rows = (uint32_t)(re - rb);
    *cols = m.col_end - m.col_begin;
    return POTTS_OK;
}

int raw_box_run(potts_context *ctx, const potts_mapping *map, const float *d_f, uint8_t *d_box)
{
    uint32_t rb = 0, rows = 0, cols = 0;
    POTTS_TRY(raw_box_dims(*map, &rb, &rows, &cols));
    const size_t tb = sizeof(uint32_t) * (2 * (size_t)map->cols + 1);
    POTTS_TRY(ensure(ctx, ctx->io_tables, tb));
    uint32_t *d_sr = static_cast<uint32_t *>(ctx->io_tables.p);
    POTTS_CUDA(cudaMemcpyAsync(d_sr, map->start_row, sizeof(uint32_t) * map->cols, cudaMemcpyHostToDevice,
                               ctx->stream));
    POTTS_CUDA(cudaMemcpyAsync(d_sr + map->cols, map->base, sizeof(uint32_t) * ((size_t)map->cols + 1),
                               cudaMemcpyHostToDevice, ctx->stream));
    potts::BoxGeom g;
    g.start_row = d_sr;
    g.base = d_sr + map->cols;
    g.col_begin = map->col_begin;
    g.row_begin = rb;
    g.row_size = (int)rows;
    g.box_lines = (int64_t)rows * cols;
    g.ns = (int)map->n_images;
    g.nstride = (int)map->nstride;
    POTTS_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    if (aligned16(d_f) && ((uintptr_t)d_box & 3u) == 0 && g.ns % 4 == 0)
        potts::raw_box_kernel<true><<<io_blocks(ctx, g.box_lines), potts::kIoThreads, 0, ctx->stream>>>(g, d_f, d_box);
    else
        potts::raw_box_kernel<false><<<io_blocks(ctx, g.box_lines), potts::kIoThreads, 0, ctx->stream>>>(g, d_f, d_box);
    POTTS_CUDA(cudaGetLastError());
    POTTS_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->total_launches += 1;
    return POTTS_OK;
}

// The XML around the raw box (potts-model.cpp:218-240): header, 4-byte little-endian size, bytes, footer.
std::string vtk_header(uint32_t slices, uint32_t rows, uint32_t cols)
{
    char buf[1024];
    const unsigned a = slices - 1, b = rows - 1, c = cols - 1;
    std::snprintf(buf, sizeof buf,
                  "<?xml version=\"1.0\"?>\n"
                  "<VTKFile type=\"ImageData\" byte_order=\"LittleEndian\">\n"
                  "  <ImageData WholeExtent=\"0 %u 0 %u 0 %u\">\n"
                  "    <Piece Extent=\"0 %u 0 %u 0 %u\">\n"
                  "      <PointData Scalars=\"labels\">\n"
                  "        <DataArray type=\"UInt8\" Name=\"labels\" format=\"appended\" offset=\"0\"/>\n"
                  "      </PointData>\n"
                  "    </Piece>\n"
                  "  </ImageData>\n"
                  "  <AppendedData encoding=\"raw\">\n_",
                  a, b, c, a, b, c);
    return std::string(buf);
}
const char kVtkFooter[] = "\n  </AppendedData>\n</VTKFile>\n";

int vtk_labels_run(potts_context *ctx, const potts_mapping *map, const float *d_f, uint8_t *out, uint64_t capacity,
                   uint64_t *out_bytes, potts_io_stats *st)
{
    uint32_t rb = 0, rows = 0, cols = 0;
    POTTS_TRY(raw_box_dims(*map, &rb, &rows, &cols));
    const std::string head = vtk_header(map->n_images, rows, cols);
    const uint64_t box = (uint64_t)map->n_images * rows * cols;
    const uint64_t total = head.size() + 4 + box + (sizeof(kVtkFooter) - 1);
    if (out_bytes) *out_bytes = total;
    if (!out) return POTTS_OK;
    if (capacity < total) return fail(POTTS_EINVAL, "output buffer is smaller than the VTK file");
    if (!d_f) return fail(POTTS_EINVAL, "field is NULL");
    POTTS_TRY(ensure(ctx, ctx->io, box));
    POTTS_TRY(raw_box_run(ctx, map, d_f, static_cast<uint8_t *>(ctx->io.p)));
    uint8_t *p = out;
    std::memcpy(p, head.data(), head.size());
    p += head.size();
    const uint32_t nbytes = (uint32_t)box;  // a 32-bit size, as the reference writes it
    std::memcpy(p, &nbytes, 4);
    p += 4;
    POTTS_CUDA(cudaMemcpyAsync(p, ctx->io.p, box, cudaMemcpyDeviceToHost, ctx->stream));
    std::memcpy(p + box, kVtkFooter, sizeof(kVtkFooter) - 1);
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    return io_stats_kernel(ctx, st, 1);
}

// ---- PNG slice (potts-model.cpp:34-49): the lines of one column as an 8-bit grey image, rows
// down, slices across, gray = saturate(round-half-even(255 |x|^(1/2.2))) computed in double.  The
// image is written as a PNG with stored (uncompressed) deflate blocks.
// CRC-32 of PNG chunks (reflected polynomial 0xedb88320); the table is built once, thread-safely.
struct Crc32Table {
    uint32_t t[256];
    Crc32Table()
    {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xedb88320u ^ (c >> 1) : c >> 1;
            t[i] = c;
        }
    }
};

uint32_t crc32_update(uint32_t crc, const uint8_t *p, size_t n)
{
    static const Crc32Table table;
    for (size_t i = 0; i < n; ++i) crc = table.t[(crc ^ p[i]) & 0xffu] ^ (crc >> 8);
    return crc;
}

void put_be32(std::vector<uint8_t> &v, uint32_t x)
{
    for (int s = 24; s >= 0; s -= 8) v.push_back((uint8_t)(x >> s));
}

void png_chunk(std::vector<uint8_t> &out, const char type[4], const uint8_t *data, size_t n)
{
    put_be32(out, (uint32_t)n);
    const size_t at = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data, data + n);
    const uint32_t crc = crc32_update(0xffffffffu, out.data() + at, n + 4) ^ 0xffffffffu;
    put_be32(out, crc);
}

// cv::pow raises |x| for a non-integer exponent; NaN and 0 give 0.
uint8_t gamma_gray(float x)
{
    const double a = std::fabs((double)x);
    if (!(a > 0.0)) return 0;
    const double v = std::nearbyint(std::pow(a, 1.0 / 2.2) * 255.0);  // ties to even
    return (uint8_t)(v >= 255.0 ? 255 : v);
}

// PNG bytes of a width x height grey image (rows top to bottom, filter 0 per row).
std::vector<uint8_t> encode_png_gray(const uint8_t *pix, uint32_t width, uint32_t height)
{
    std::vector<uint8_t> raw;
    raw.reserve((size_t)(width + 1) * height);
    for (uint32_t r = 0; r < height; ++r) {
        raw.push_back(0);
        raw.insert(raw.end(), pix + (size_t)r * width, pix + (size_t)(r + 1) * width);
    }
    std::vector<uint8_t> z = {0x78, 0x01};  // zlib stream, deflate with stored blocks
    size_t off = 0;
    do {
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        z.push_back(off + len == raw.size() ? 1 : 0);
        z.push_back((uint8_t)len);
        z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)~len);
        z.push_back((uint8_t)(~len >> 8));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
        off += len;
    } while (off < raw.size());
    uint32_t a = 1, b = 0;  // Adler-32 of the uncompressed bytes
    for (uint8_t c : raw) {
        a = (a + c) % 65521u;
        b = (b + a) % 65521u;
    }
    put_be32(z, (b << 16) | a);
    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    uint8_t ihdr[13];
    for (int i = 0; i < 4; ++i) {
        ihdr[i] = (uint8_t)(width >> (24 - 8 * i));
        ihdr[4 + i] = (uint8_t)(height >> (24 - 8 * i));
    }
    ihdr[8] = 8;   // bit depth
    ihdr[9] = 0;   // greyscale
    ihdr[10] = 0;  // deflate
    ihdr[11] = 0;  // adaptive filtering (every row uses filter 0)
    ihdr[12] = 0;  // no interlace
    png_chunk(png, "IHDR", ihdr, sizeof ihdr);
    png_chunk(png, "IDAT", z.data(), z.size());
    png_chunk(png, "IEND", nullptr, 0);
    return png;
}

int png_slice_run(potts_context *ctx, const potts_mapping *map, const float *d_f, uint32_t col, uint8_t *out,
                  uint64_t capacity, uint64_t *out_bytes)
{
    if (col < map->col_begin || col >= map->col_end) return fail(POTTS_EINVAL, "column holds no rows");
    const uint32_t height = (map->base[col + 1] - map->base[col]) / map->nstride;
    if (height == 0) return fail(POTTS_EINVAL, "column holds no rows");
    const uint32_t width = map->n_images;
    // stored-block PNG: fixed size for given dimensions
    const uint64_t raw = (uint64_t)(width + 1) * height;
    const uint64_t blocks = (raw + 65534) / 65535;
    const uint64_t total = 8 + (12 + 13) + (12 + 2 + raw + 5 * blocks + 4) + 12;
    if (out_bytes) *out_bytes = total;
    if (!out) return POTTS_OK;
    if (capacity < total) return fail(POTTS_EINVAL, "output buffer is smaller than the PNG");
    if (!d_f) return fail(POTTS_EINVAL, "field is NULL");
    std::vector<float> lines((size_t)width * height);
    POTTS_CUDA(cudaMemcpy2DAsync(lines.data(), sizeof(float) * width, d_f + map->base[col], sizeof(float) * map->nstride,
                                 sizeof(float) * width, height, cudaMemcpyDeviceToHost, ctx->stream));
    POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<uint8_t> pix(lines.size());
    for (size_t i = 0; i < lines.size(); ++i) pix[i] = gamma_gray(lines[i]);
    const std::vector<uint8_t> png = encode_png_gray(pix.data(), width, height);
    if (png.size() != total) return fail(POTTS_ECUDA, "internal PNG size mismatch");
    std::memcpy(out, png.data(), png.size());
    return POTTS_OK;
}
