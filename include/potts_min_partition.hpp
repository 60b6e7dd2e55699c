// potts_min_partition.hpp — header-only C++ layer over the C ABI (potts_b200.h)
// with the reference's entry points, so that potts-model/potts-model.cpp can
// switch to the B200 library by changing includes and a namespace:
//
//   reference                                        here
//   make_context()          cuda-context.cpp:18-20   potts_b200::make_context()
//   upload(ctx, span)       cuda-context.cpp:49-57   potts_b200::upload(ctx, mapping, host_ptr)
//   download(ctx, f, span)  cuda-context.cpp:59-77   potts_b200::download(ctx, f, host_ptr, span)
//   device_memory(ctx)      cuda-context.cpp:22-42   potts_b200::device_memory(ctx)
//   potts_min_partition<K>  potts-min-partition.h:8-16
//                                                    potts_b200::potts_min_partition<K>(ctx, g, cpu_map, ci,
//                                                                                       lambda, tau1, tau2, iters)
//
// Error behaviour follows the reference: a slab plan that does not fit in
// device memory returns an empty pointer (potts-min-partition.cpp:571-577);
// other failures throw std::runtime_error (the reference throws
// cuda::cuda_error).  to_potts_mapping() adapts any mapping with the
// layout_cylinder::mapping interface (include/layout_cylinder.h:30-112).
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>

#include "potts_b200.h"

namespace potts_b200 {

inline void check(int status)
{
    if (status != POTTS_OK)
        throw std::runtime_error(std::string(potts_status_string(status)) + ": " + potts_last_error());
}

// A potts_mapping viewing the tables of a layout_cylinder::mapping-like object
// (extents(), nstride(), col_begin(), col_end(), csc.start_row_, csc.base_).
// The tables are borrowed: keep `m` alive while the result is used.
template <class Mapping>
potts_mapping to_potts_mapping(const Mapping &m)
{
    potts_mapping p;
    p.n_images = static_cast<uint32_t>(m.extents().extent(0));
    p.rows = static_cast<uint32_t>(m.extents().extent(1));
    p.cols = static_cast<uint32_t>(m.extents().extent(2));
    p.nstride = static_cast<uint32_t>(m.nstride());
    p.col_begin = static_cast<uint32_t>(m.col_begin());
    p.col_end = static_cast<uint32_t>(m.col_end());
    p.start_row = reinterpret_cast<const uint32_t *>(m.csc.start_row_);
    p.base = reinterpret_cast<const uint32_t *>(m.csc.base_);
    return p;
}

class CudaContext {
public:
    explicit CudaContext(int device = 0) { check(potts_context_create(device, &ctx_)); }
    CudaContext(int device, void *stream) { check(potts_context_create_on_stream(device, stream, &ctx_)); }
    ~CudaContext() { potts_context_destroy(ctx_); }
    CudaContext(const CudaContext &) = delete;
    CudaContext &operator=(const CudaContext &) = delete;
    potts_context *get() const { return ctx_; }
    void synchronize() { check(potts_context_synchronize(ctx_)); }

private:
    potts_context *ctx_ = nullptr;
};
using cuda_context_ptr = std::unique_ptr<CudaContext>;

inline cuda_context_ptr make_context(int device = 0) { return std::make_unique<CudaContext>(device); }

struct device_memory_info {
    std::size_t available;
    std::size_t total;
};

inline device_memory_info device_memory(const CudaContext &ctx)
{
    device_memory_info d{};
    check(potts_device_memory(ctx.get(), &d.available, &d.total));
    return d;
}

// DeviceField<float>: device voxels with the mapping of the host field.
class DeviceField {
public:
    explicit DeviceField(potts_field *f) : f_(f) {}
    ~DeviceField() { potts_field_destroy(f_); }
    DeviceField(const DeviceField &) = delete;
    DeviceField &operator=(const DeviceField &) = delete;
    float *data() { return potts_field_data(f_); }
    uint64_t span() const { return potts_field_span(f_); }
    potts_field *get() const { return f_; }

private:
    potts_field *f_ = nullptr;
};
using device_field_ptr = std::unique_ptr<DeviceField>;

inline device_field_ptr upload(CudaContext &ctx, const potts_mapping &map, const float *host)
{
    potts_field *f = nullptr;
    check(potts_field_upload(ctx.get(), &map, host, &f));
    return std::make_unique<DeviceField>(f);
}

inline void download(CudaContext &ctx, const DeviceField &f, float *host, uint64_t span)
{
    check(potts_field_download(ctx.get(), f.get(), host, span));
}

// potts_min_partition<K>: ci[argmax_i V_i] for every voxel of g, as a new field.
template <std::size_t K>
device_field_ptr potts_min_partition(CudaContext &ctx, DeviceField &g, const potts_mapping &cpu_map,
                                     std::array<float, K> ci, float lambda, float tau1, float tau2, int iters,
                                     const potts_options *opts = nullptr, potts_stats *stats = nullptr)
{
    static_assert(K >= 2 && K <= POTTS_MAX_PHASES, "2 to POTTS_MAX_PHASES labels");
    potts_field *res = nullptr;
    const int s = ::potts_min_partition(ctx.get(), g.get(), &cpu_map, static_cast<int>(K), ci.data(), lambda, tau1,
                                        tau2, iters, opts, &res, stats);
    if (s == POTTS_ENOMEM) return {};  // the reference prints a message and returns an empty pointer
    check(s);
    return std::make_unique<DeviceField>(res);
}

}  // namespace potts_b200
