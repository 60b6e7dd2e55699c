// Compiles the C++ drop-in layers (potts_min_partition.hpp, field_io.hpp) against
// the C ABI and checks the parts that need no GPU: the mapping adapter, the
// archive size and the reference-style error behaviour; with a GPU, a small
// solve and an archive round trip.
#include <array>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "field_io.hpp"
#include "potts_min_partition.hpp"

// Stand-in with the interface of layout_cylinder::mapping (include/layout_cylinder.h:30-112).
struct FakeExtents {
    uint32_t e[3];
    uint32_t extent(int i) const { return e[i]; }
};
struct FakeMapping {
    FakeExtents ext;
    uint32_t ns, cb, ce;
    struct {
        const uint32_t *start_row_;
        const uint32_t *base_;
    } csc;
    const FakeExtents &extents() const { return ext; }
    uint32_t nstride() const { return ns; }
    uint32_t col_begin() const { return cb; }
    uint32_t col_end() const { return ce; }
};

int main()
{
    const uint32_t rows = 20, cols = 18, n = 40;
    std::vector<uint32_t> start_row(cols), base(cols + 1);
    uint32_t cb = 0, ce = 0;
    const uint64_t span = potts_cylinder_mapping(rows, cols, (cols - 1) / 2.0, (rows - 1) / 2.0, 8.5,
                                                 potts_get_stride(n), start_row.data(), base.data(), &cb, &ce);
    FakeMapping fm{{{n, rows, cols}}, potts_get_stride(n), cb, ce, {start_row.data(), base.data()}};
    const potts_mapping m = potts_b200::to_potts_mapping(fm);
    if (m.n_images != n || m.rows != rows || m.cols != cols || m.nstride != 64 || m.base[cols] != span ||
        m.start_row != start_row.data()) {
        std::printf("adapter mismatch\n");
        return 1;
    }
    uint64_t arch_bytes = 0, header_bits = 0;
    if (potts_archive_size(&m, POTTS_ELEM_F32, &arch_bytes, &header_bits) != POTTS_OK || header_bits % 2 != 1 ||
        arch_bytes != (header_bits + 32ull * (span / m.nstride) * n + 7) / 8) {
        std::printf("archive size mismatch\n");
        return 1;
    }
    try {
        auto ctx = potts_b200::make_context(0);
        // a GPU is present: one small solve through the drop-in entry point
        std::vector<float> u(span, 0.5f);
        auto g = potts_b200::upload(*ctx, m, u.data());
        auto res = potts_b200::potts_min_partition<3>(*ctx, *g, m, std::array<float, 3>{0.2f, 0.5f, 0.8f}, 30.0f,
                                                      0.28f, 0.28f, 5);
        std::vector<float> out(span);
        potts_b200::download(*ctx, *res, out.data(), span);
        // the .bin archive of the result, loaded back through the reference-named layer
        const std::vector<uint8_t> bytes = potts_b200::save_field(*ctx, m, res->data(), 0.25f, 0.75f);
        if (bytes.size() != arch_bytes) throw std::runtime_error("archive size differs from potts_archive_size");
        potts_b200::LoadedField back = potts_b200::load_field(*ctx, bytes.data(), bytes.size());
        std::vector<float> again(span);
        potts_b200::download(*ctx, *back.field, again.data(), span);
        for (uint64_t i = 0; i < span; ++i)
            if ((i % m.nstride) < n && again[i] != out[i]) throw std::runtime_error("archive round trip differs");
        if (back.lo != 0.25f || back.hi != 0.75f) throw std::runtime_error("lo/hi not kept");
        std::printf("solved %.3f\n", out[0]);
    } catch (const std::runtime_error &e) {
        std::printf("error: %s\n", e.what());
        return 2;
    }
    return 0;
}
