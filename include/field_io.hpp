// field_io.hpp — header-only C++ layer over the C ABI (potts_b200.h) for the
// steps around the solve, with the reference's names:
//
//   reference                                               here
//   ia >> img  (Field<T>::load, include/field.h:121-147)    potts_b200::load_field(ctx, bytes, n)
//   oa << img  (Field<T>::save, include/field.h:92-119)     potts_b200::save_field(ctx, map, d_field, lo, hi)
//   convert_to_fp(ctx, in, lo, hi)                          potts_b200::convert_to_fp(ctx, map, d_in, lo, hi)
//     (transpose/convert_to_fp.h:8-10)
//   find_intensity_range(ctx, field, tail_thr)             potts_b200::find_intensity_range(ctx, map, d_u16, tail)
//     (transpose/find_intensity_range.h)
//   write_png(img, col, lambda) (potts-model.cpp:34-49)     potts_b200::write_png(ctx, map, d_field, col, lambda)
//   --rawout VTK file (potts-model.cpp:184-243)             potts_b200::write_vtk_labels(ctx, map, d_field, path)
//
// Where the reference keeps the volume in a host Field<T> and uploads it, the
// archive calls here move the voxels straight between the archive bytes and
// device memory.  Failures throw std::runtime_error, like the reference's
// cuda::cuda_error and std::system_error.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <tuple>
#include <vector>

#include "potts_min_partition.hpp"

namespace potts_b200 {

// A mapping that owns its tables (layout_cylinder::mapping_storage, include/layout_cylinder.h:114-322).
struct MappingStorage {
    potts_mapping map{};
    std::vector<uint32_t> start_row, base;
    const potts_mapping &mapping()
    {
        map.start_row = start_row.data();
        map.base = base.data();
        return map;
    }
};

// A Field<float> loaded from an archive: its mapping, lo/hi (include/field.h:79-80) and the device voxels.
struct LoadedField {
    MappingStorage storage;
    float lo = 0.0f, hi = 0.0f;
    device_field_ptr field;
};

// ia >> img for a Field<float> archive in host memory, straight into device memory.
inline LoadedField load_field(CudaContext &ctx, const uint8_t *bytes, uint64_t n_bytes)
{
    potts_archive_info info{};
    check(potts_archive_read_header(bytes, n_bytes, POTTS_ELEM_F32, &info, nullptr, nullptr));
    LoadedField out;
    out.storage.start_row.resize(info.cols);
    out.storage.base.resize((size_t)info.cols + 1);
    check(potts_archive_read_header(bytes, n_bytes, POTTS_ELEM_F32, &info, out.storage.start_row.data(),
                                    out.storage.base.data()));
    out.storage.map = potts_mapping{info.n_images, info.rows, info.cols, info.nstride, info.col_begin, info.col_end,
                                    nullptr, nullptr};
    const potts_mapping &m = out.storage.mapping();
    potts_field *f = nullptr;
    check(potts_field_create(ctx.get(), &m, &f));
    out.field = std::make_unique<DeviceField>(f);
    check(potts_archive_load(ctx.get(), bytes, n_bytes, POTTS_ELEM_F32, out.field->data(), info.span, &info, nullptr));
    out.lo = info.lo;
    out.hi = info.hi;
    return out;
}

// oa << img for a device field (float: elem POTTS_ELEM_F32 with lo/hi; uint16: POTTS_ELEM_U16).
inline std::vector<uint8_t> save_field(CudaContext &ctx, const potts_mapping &map, const void *d_field, float lo,
                                       float hi, int elem = POTTS_ELEM_F32)
{
    uint64_t n = 0;
    check(potts_archive_save(ctx.get(), &map, elem, d_field, lo, hi, nullptr, 0, &n, nullptr));
    std::vector<uint8_t> out(n);
    check(potts_archive_save(ctx.get(), &map, elem, d_field, lo, hi, out.data(), n, &n, nullptr));
    return out;
}

// convert_to_fp(ctx, in, lo, hi) of a uint16 (POTTS_ELEM_U16) or float device field: a new float field.
inline device_field_ptr convert_to_fp(CudaContext &ctx, const potts_mapping &map, const void *d_in, float lo,
                                      float hi, int elem = POTTS_ELEM_U16)
{
    potts_field *f = nullptr;
    check(potts_field_create(ctx.get(), &map, &f));
    auto out = std::make_unique<DeviceField>(f);
    check(potts_convert_to_fp(ctx.get(), &map, elem, d_in, lo, hi, out->data()));
    return out;
}

// find_intensity_range(ctx, field, tail_thr) of a uint16 device field.
inline std::tuple<uint16_t, uint16_t> find_intensity_range(CudaContext &ctx, const potts_mapping &map,
                                                           const uint16_t *d_field, double tail_thr)
{
    uint16_t lo = 0, hi = 0;
    check(potts_find_intensity_range(ctx.get(), &map, d_field, tail_thr, &lo, &hi, nullptr));
    return {lo, hi};
}

inline void write_file(const std::string &path, const std::vector<uint8_t> &bytes)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + path);
    const size_t w = std::fwrite(bytes.data(), 1, bytes.size(), f);
    std::fclose(f);
    if (w != bytes.size()) throw std::runtime_error("short write to " + path);
}

// write_png(img, col, lambda): "slice-{col} (𝜆 = {lambda:07.3f}).png" in the working directory; returns the name.
inline std::string write_png(CudaContext &ctx, const potts_mapping &map, const float *d_field, uint32_t col,
                             float lambda)
{
    uint64_t n = 0;
    check(potts_png_slice(ctx.get(), &map, d_field, col, nullptr, 0, &n));
    std::vector<uint8_t> png(n);
    check(potts_png_slice(ctx.get(), &map, d_field, col, png.data(), n, &n));
    char name[96];
    std::snprintf(name, sizeof name, "slice-%u (\xf0\x9d\x9c\x86 = %07.3f).png", col, (double)lambda);
    write_file(name, png);
    return name;
}

// The --rawout file of potts-model for a device field of c[argmax] values.
inline void write_vtk_labels(CudaContext &ctx, const potts_mapping &map, const float *d_field, const std::string &path)
{
    uint64_t n = 0;
    check(potts_vtk_labels(ctx.get(), &map, d_field, nullptr, 0, &n, nullptr));
    std::vector<uint8_t> vtk(n);
    check(potts_vtk_labels(ctx.get(), &map, d_field, vtk.data(), n, &n, nullptr));
    write_file(path, vtk);
}

}  // namespace potts_b200
