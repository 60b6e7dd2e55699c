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

// Instantiates launch_fused for every tile shape of ShapesOf<K, ST>.
template <int K, typename ST, bool FAST, size_t... I>
const void *const *fused_instances(std::index_sequence<I...>)
{
    using TS = ShapesOf<K, ST>;
    static const void *const table[] = {
        reinterpret_cast<const void *>(&launch_fused<K, TS::r[I], TS::t[I], TS::v[I], ST, FAST>)...};
    return table;
}

}  // namespace potts

// Explicit instantiation of every shape of (K, ST, FAST) in this translation unit.
#define POTTS_FUSED_INSTANCES(K, ST, FAST)                                                                    \
    template const void *const *potts::fused_instances<K, ST, FAST>(                                          \
        std::make_index_sequence<(size_t)potts::ShapesOf<K, ST>::n>)
