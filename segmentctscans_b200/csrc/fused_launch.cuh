// Definition of potts::launch_fused (declared in kernels_tiled.cuh) and the
// helper that instantiates it for every compiled tile shape of one (K,
// storage, arithmetic).  Included only by the fused_*.cu translation units,
// which the build compiles in parallel.
#pragma once

#include <cuda_runtime.h>

#include <utility>

#include "kernels_tiled.cuh"
#include "tile_shapes.cuh"

namespace potts {

template <int K, int R, int NT, int VPT, typename ST, bool FAST>
cudaError_t launch_fused(cudaStream_t stream, const FusedVolume<K, ST> *vols, const int4 *work, const int *work_vol,
                         int n_work, int in, int it, float tau2, DykstraThresholds thr, int *err)
{
    using S = TileShape<K, R, NT, VPT, ST>;
    constexpr int kMaxDevices = 64;
    static bool attr_set[kMaxDevices] = {};  // the shared-memory opt-in is per device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kMaxDevices && !attr_set[dev]) {
        e = cudaFuncSetAttribute(fused_tiled_kernel<K, R, NT, VPT, ST, FAST>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM_ALLOC);
        if (e != cudaSuccess) return e;
        attr_set[dev] = true;
    }
    if (n_work == 0) return cudaSuccess;
    fused_tiled_kernel<K, R, NT, VPT, ST, FAST><<<n_work, S::THREADS, S::SMEM_ALLOC, stream>>>(
        vols, work, work_vol, in, it, tau2, thr, err);
    return cudaGetLastError();
}

template <int K, int R, int NT, int VPT, typename ST, bool FAST>
cudaError_t launch_fused_persistent(cudaStream_t stream, const FusedVolume<K, ST> *vols, const int4 *work,
                                    const int *work_vol, int n_work, int in0, int it0, int n_iters, float tau2,
                                    DykstraThresholds thr, int *err, uint32_t *ctl)
{
    using S = TileShape<K, R, NT, VPT, ST>;
    constexpr int kMaxDevices = 64;
    static bool attr_set[kMaxDevices] = {};
    static int grid_of[kMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    auto kern = fused_persistent_kernel<K, R, NT, VPT, ST, FAST>;
    if (!attr_set[dev]) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM_ALLOC);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, S::THREADS, S::SMEM_ALLOC);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
        grid_of[dev] = per_sm * sms;
        attr_set[dev] = true;
    }
    if (n_work == 0 || n_iters <= 0) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(n_work < grid_of[dev] ? n_work : grid_of[dev]));
    cfg.blockDim = dim3(S::THREADS);
    cfg.dynamicSmemBytes = S::SMEM_ALLOC;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, vols, work, work_vol, n_work, in0, it0, n_iters, tau2, thr, err, ctl);
}

// Instantiates launch_fused and launch_fused_persistent for every tile shape
// of ShapesOf<K, ST>.
template <int K, typename ST, bool FAST, size_t... I>
const void *const *fused_instances(std::index_sequence<I...>)
{
    using TS = ShapesOf<K, ST>;
    static const void *const table[] = {
        reinterpret_cast<const void *>(&launch_fused<K, TS::r[I], TS::t[I], TS::v[I], ST, FAST>)...,
        reinterpret_cast<const void *>(&launch_fused_persistent<K, TS::r[I], TS::t[I], TS::v[I], ST, FAST>)...};
    return table;
}

}  // namespace potts

// Explicit instantiation of every shape of (K, ST, FAST) in this translation unit.
#define POTTS_FUSED_INSTANCES(K, ST, FAST)                                                                    \
    template const void *const *potts::fused_instances<K, ST, FAST>(                                          \
        std::make_index_sequence<(size_t)potts::ShapesOf<K, ST>::n>)
