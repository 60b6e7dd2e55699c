// Tiled fused iteration (the hot path).  The reference runs the dual step
// (grad_kernel) and the primal step (div_kernel) as two launches and keeps
// Vbar in memory.  Here one launch runs the primal step of iteration m and the
// dual step of iteration m+1:
//   V^m      = Pi_S(V^{m-1} + tau1 (div- Xi^m - G))
//   Vbar^m   = 2 V^m - V^{m-1}                       (shared memory only)
//   Xi^{m+1} = Pi_K(Xi^m + tau2 grad+ Vbar^m)
// so (Xi^m, V^{m-1}) become (Xi^{m+1}, V^m).  The dual step at x needs Vbar^m
// at x + e_n, x + e_row, x + e_col, so each tile also runs the primal step on
// a one-voxel high halo.  The host runs a plain dual step first (Xi^1 from
// V^0) and a plain primal step last (V^iters from Xi^iters).
//
// Work item = a tile of R rows x NT slices (n) that marches along the columns
// c in [ca, cb).  Planes (columns) pass through a ring of D = 3 shared-memory
// slots; slot p % D holds, for ring position p = c - ca + 1 (plane ca-1 is
// p = 0): Xi^m on rows r0-1 .. r0+R and slices n0-4 .. n0+NT+3 (one 3-D TMA
// box for all components), V^{m-1} and u on rows r0 .. r0+R and slices
// n0 .. n0+NT+3, and the Vbar^m the block computes for that plane.
// The block is warp-specialised and has no block-wide barrier in the loop:
//   producer warp   for every plane: wait until the slot is released, then
//                   issue its TMA loads (mbarrier `full` counts the bytes);
//   row warps       warp w owns tile row w: stage A (primal step at plane c,
//                   Vbar to shared memory, V^m to global), then stage B (dual
//                   step at plane c-1, Xi^{m+1} to global);
//   halo warp       stage A on the high halo (row r0+R, slice n0+NT).
// Per plane two more mbarriers order the warps: `ready` (every warp's stage A
// is done, so stage B may read its neighbours' Vbar rows) and `empty` (every
// warp is done reading the slot, so the producer may refill it).  Warps can
// therefore run up to two planes apart instead of waiting for the slowest one
// at every plane.
//
// Dykstra's full loop is needed only where some pair |q_i - q_j| exceeds 1;
// elsewhere its first sweep is the identity.  Stage B tests this per voxel,
// gathers the warp's voxels that need the loop into a shared-memory queue and
// runs the loop on them with all 32 lanes busy, so the common voxels do not
// wait for the warp's slowest lane.
//
// HBM traffic per voxel and iteration: Xi and V read and written once, u read
// once (8(K-1)+1 floats: 68 bytes at K = 3); halo rows/slices and the
// neighbouring plane come from L2.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "geometry.cuh"
#include "kernels_plain.cuh"
#include "tma.cuh"
#include "voxel.cuh"

namespace potts {

// Per column: x = line of row start_row[col], y = first row, z = one past the
// last row (y = z = 0 for an empty column).
// Per work item: x = r0 (first row of the tile), y = n0, z = ca, w = cb.
struct TiledParams {
    const int4 *cols;
    const int4 *work;
    int col_begin, col_end;
    int ns;         // slab extent along n
    int nstride_w;  // stride of the state arrays
    int64_t plane_w;
    int u_x0;       // n offset of the slab in the u tensor map
};

template <int K, int R, int NT>
struct TileShape {
    static constexpr int D = 3;  // ring depth (planes)
    static constexpr int C3 = 3 * (K - 1), C1 = K - 1, Q = NT / 4;
    static constexpr int NX = NT + 8;  // Xi box: slices n0-4 .. n0+NT+3
    static constexpr int NV = NT + 4;  // V/u/Vbar box: slices n0 .. n0+NT+3
    static constexpr int MAIN = R * Q;
    static constexpr int MAIN_WARPS = MAIN / 32;
    static constexpr int HALO_WARP = MAIN_WARPS, PRODUCER_WARP = MAIN_WARPS + 1;
    static constexpr int THREADS = MAIN + 64;
    static constexpr int QSTRIDE = (3 * K) | 1;  // queue entry stride (odd: no bank conflicts)
    static constexpr int QCAP = 4 * 32;           // a warp's voxels per plane
    static constexpr int XI_BYTES = C3 * (R + 2) * NX * 4;
    static constexpr int V_BYTES = C1 * (R + 1) * NV * 4;
    static constexpr int U_BYTES = (R + 1) * NV * 4;
    static constexpr int al(int b) { return (b + 127) / 128 * 128; }
    static constexpr int XI_SLOT = al(XI_BYTES), V_SLOT = al(V_BYTES), U_SLOT = al(U_BYTES);
    static constexpr int OFF_XI = 0;
    static constexpr int OFF_V = OFF_XI + D * XI_SLOT;
    static constexpr int OFF_U = OFF_V + D * V_SLOT;
    static constexpr int OFF_VB = OFF_U + D * U_SLOT;
    static constexpr int OFF_Q = OFF_VB + D * V_SLOT;
    static constexpr int OFF_BAR = OFF_Q + al(MAIN_WARPS * QCAP * QSTRIDE * 4);
    static constexpr int SMEM = OFF_BAR + 3 * D * 8 + 16;
    static constexpr int SMEM_ALLOC = SMEM + 128;  // room to align the base to 128 bytes
    static_assert(NT % 4 == 0 && Q <= 32 && R + 1 <= 32, "tile shape");
    static_assert(MAIN % 32 == 0, "row threads fill whole warps");
    static_assert(SMEM_ALLOC <= 227 * 1024, "shared memory of one block");
};

__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void sts4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ void f4_to(float (&a)[4], float4 v)
{
    a[0] = v.x;
    a[1] = v.y;
    a[2] = v.z;
    a[3] = v.w;
}

__device__ __forceinline__ bool row_in_col(int4 ci, int row) { return row >= ci.y && row < ci.z; }

template <int K, int R, int NT>
struct TiledSmem {
    using S = TileShape<K, R, NT>;
    uint8_t *base;

    __device__ __forceinline__ float *xi_slot(int p) const
    {
        return reinterpret_cast<float *>(base + S::OFF_XI + (p % S::D) * S::XI_SLOT);
    }
    __device__ __forceinline__ float *v_slot(int p) const
    {
        return reinterpret_cast<float *>(base + S::OFF_V + (p % S::D) * S::V_SLOT);
    }
    __device__ __forceinline__ float *u_slot(int p) const
    {
        return reinterpret_cast<float *>(base + S::OFF_U + (p % S::D) * S::U_SLOT);
    }
    __device__ __forceinline__ float *vb_plane(int p) const
    {
        return reinterpret_cast<float *>(base + S::OFF_VB + (p % S::D) * S::V_SLOT);
    }
    __device__ __forceinline__ float *queue(int warp) const
    {
        return reinterpret_cast<float *>(base + S::OFF_Q) + warp * S::QCAP * S::QSTRIDE;
    }
    __device__ __forceinline__ uint64_t *full(int p) const
    {
        return reinterpret_cast<uint64_t *>(base + S::OFF_BAR) + (p % S::D);
    }
    __device__ __forceinline__ uint64_t *ready(int p) const
    {
        return reinterpret_cast<uint64_t *>(base + S::OFF_BAR) + S::D + (p % S::D);
    }
    __device__ __forceinline__ uint64_t *empty(int p) const
    {
        return reinterpret_cast<uint64_t *>(base + S::OFF_BAR) + 2 * S::D + (p % S::D);
    }
    __device__ __forceinline__ volatile int *abort_flag() const
    {
        return reinterpret_cast<volatile int *>(base + S::OFF_BAR + 3 * S::D * 8);
    }
    // phase parity of ring position p's use of its slot's barriers
    __device__ __forceinline__ static uint32_t parity(int p) { return (uint32_t)((p / S::D) & 1); }
    // element (comp, box row, box slice) of an Xi plane / a V-shaped plane
    __device__ __forceinline__ static int xi_at(int comp, int rr, int nn) { return (comp * (R + 2) + rr) * S::NX + nn; }
    __device__ __forceinline__ static int v_at(int comp, int rr, int nn) { return (comp * (R + 1) + rr) * S::NV + nn; }
};

// Stage A for 4 consecutive slices n0+4q .. n0+4q+3 of tile row rr (row r0+rr).
// Planes are indexed by "ring position" p = c - ca + 1 (plane ca-1 is p = 0).
template <int K, int R, int NT>
__device__ __forceinline__ void stage_a_quad(const TiledSmem<K, R, NT> &sm, const TiledParams &tp,
                                             const PhaseParams<K> &pp, int p, int c, int r0, int rr, int n0, int q,
                                             bool store_v, float *__restrict__ Vout, float &dqmax)
{
    using S = TileShape<K, R, NT>;
    using T = TiledSmem<K, R, NT>;
    const int row = r0 + rr;
    float *vb = sm.vb_plane(p);
    const int4 ci = tp.cols[c];
    const int nb = n0 + 4 * q;
    if (!row_in_col(ci, row) || nb >= tp.ns) {
#pragma unroll
        for (int i = 0; i < K - 1; ++i) sts4(vb + T::v_at(i, rr, 4 * q), make_float4(0, 0, 0, 0));
        return;
    }
    const bool pr = row > ci.y, hr = row + 1 < ci.z;
    const bool pc = c - 1 >= tp.col_begin && row_in_col(tp.cols[c - 1], row);
    const bool hc = c + 1 < tp.col_end && row_in_col(tp.cols[c + 1], row);
    const float *xs = sm.xi_slot(p), *xp = sm.xi_slot(p - 1);
    const float *vs = sm.v_slot(p), *us = sm.u_slot(p);

    float x[S::C3][4], xn[K - 1][4], xr[K - 1][4], xc[K - 1][4], v[K - 1][4], u[4];
#pragma unroll
    for (int comp = 0; comp < S::C3; ++comp) f4_to(x[comp], lds4(xs + T::xi_at(comp, rr + 1, 4 * q + 4)));
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        f4_to(xn[i], lds4(xs + T::xi_at(3 * i, rr + 1, 4 * q)));  // slices nb-4 .. nb-1
        f4_to(xr[i], lds4(xs + T::xi_at(3 * i + 1, rr, 4 * q + 4)));
        f4_to(xc[i], lds4(xp + T::xi_at(3 * i + 2, rr + 1, 4 * q + 4)));
        f4_to(v[i], lds4(vs + T::v_at(i, rr, 4 * q)));
    }
    f4_to(u, lds4(us + T::v_at(0, rr, 4 * q)));

    float onew[K - 1][4], obar[K - 1][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int n = nb + j;
        float xi_j[S::C3], xin_j[K - 1], xir_j[K - 1], xic_j[K - 1], v_j[K - 1], vn[K - 1], vbar[K - 1];
#pragma unroll
        for (int comp = 0; comp < S::C3; ++comp) xi_j[comp] = x[comp][j];
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            xin_j[i] = (j == 0) ? xn[i][3] : x[3 * i][j - 1];
            xir_j[i] = xr[i][j];
            xic_j[i] = xc[i][j];
            v_j[i] = v[i][j];
        }
        float d = 0.0f;
        if (n < tp.ns) {
            d = primal_voxel<K>(vn, vbar, v_j, xi_j, xin_j, xir_j, xic_j, n > 0, n + 1 < tp.ns, pr, hr, pc, hc, u[j],
                                pp.c, pp.lam, pp.tau1);
        } else {
#pragma unroll
            for (int i = 0; i < K - 1; ++i) vn[i] = vbar[i] = 0.0f;
        }
        if (store_v) dqmax = fmaxf(dqmax, d);
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            onew[i][j] = vn[i];
            obar[i][j] = vbar[i];
        }
    }
#pragma unroll
    for (int i = 0; i < K - 1; ++i)
        sts4(vb + T::v_at(i, rr, 4 * q), make_float4(obar[i][0], obar[i][1], obar[i][2], obar[i][3]));
    if (store_v) {
        const int64_t o = (int64_t)(ci.x + row - ci.y) * tp.nstride_w + nb;
        if (nb + 4 <= tp.ns) {
#pragma unroll
            for (int i = 0; i < K - 1; ++i)
                *reinterpret_cast<float4 *>(Vout + i * tp.plane_w + o) =
                    make_float4(onew[i][0], onew[i][1], onew[i][2], onew[i][3]);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (nb + j < tp.ns)
#pragma unroll
                    for (int i = 0; i < K - 1; ++i) Vout[i * tp.plane_w + o + j] = onew[i][j];
        }
    }
}

// Stage A for the single slice n0+NT of tile row rr (the high halo along n).
template <int K, int R, int NT>
__device__ __forceinline__ void stage_a_nhalo(const TiledSmem<K, R, NT> &sm, const TiledParams &tp,
                                              const PhaseParams<K> &pp, int p, int c, int r0, int rr, int n0)
{
    using S = TileShape<K, R, NT>;
    using T = TiledSmem<K, R, NT>;
    const int row = r0 + rr, n = n0 + NT;
    float *vb = sm.vb_plane(p);
    const int4 ci = tp.cols[c];
    if (!row_in_col(ci, row) || n >= tp.ns) {
#pragma unroll
        for (int i = 0; i < K - 1; ++i) vb[T::v_at(i, rr, NT)] = 0.0f;
        return;
    }
    const bool pr = row > ci.y, hr = row + 1 < ci.z;
    const bool pc = c - 1 >= tp.col_begin && row_in_col(tp.cols[c - 1], row);
    const bool hc = c + 1 < tp.col_end && row_in_col(tp.cols[c + 1], row);
    const float *xs = sm.xi_slot(p), *xp = sm.xi_slot(p - 1);
    float xi[S::C3], xin[K - 1], xir[K - 1], xic[K - 1], v[K - 1], vn[K - 1], vbar[K - 1];
#pragma unroll
    for (int comp = 0; comp < S::C3; ++comp) xi[comp] = xs[T::xi_at(comp, rr + 1, NT + 4)];
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        xin[i] = xs[T::xi_at(3 * i, rr + 1, NT + 3)];
        xir[i] = xs[T::xi_at(3 * i + 1, rr, NT + 4)];
        xic[i] = xp[T::xi_at(3 * i + 2, rr + 1, NT + 4)];
        v[i] = sm.v_slot(p)[T::v_at(i, rr, NT)];
    }
    const float uu = sm.u_slot(p)[T::v_at(0, rr, NT)];
    primal_voxel<K>(vn, vbar, v, xi, xin, xir, xic, n > 0, n + 1 < tp.ns, pr, hr, pc, hc, uu, pp.c, pp.lam, pp.tau1);
#pragma unroll
    for (int i = 0; i < K - 1; ++i) vb[T::v_at(i, rr, NT)] = vbar[i];
}

// Stage B: dual step at plane c (ring position p) for slices n0+4q .. +3 of
// tile row rr.  Called by every lane of the main warps (warp-wide gathers).
template <int K, int R, int NT>
__device__ __forceinline__ void stage_b_quad(const TiledSmem<K, R, NT> &sm, const TiledParams &tp, int p, int c,
                                             int r0, int rr, int n0, int q, float tau2, DykstraThresholds thr,
                                             float *__restrict__ Xout)
{
    using S = TileShape<K, R, NT>;
    using T = TiledSmem<K, R, NT>;
    const int lane = threadIdx.x & 31;
    const int row = r0 + rr;
    const int4 ci = tp.cols[c];
    const int nb = n0 + 4 * q;
    const bool live = row_in_col(ci, row) && nb < tp.ns;

    float qv[4][K][3];
    unsigned need = 0;  // bit j: slot j needs the full projection loop
    if (live) {
        const bool hr = row + 1 < ci.z;
        const bool hc = c + 1 < tp.col_end && row_in_col(tp.cols[c + 1], row);
        const float *xs = sm.xi_slot(p);
        const float *vb0 = sm.vb_plane(p), *vb1 = sm.vb_plane(p + 1);
        float x[S::C3][4], b[K - 1][4], bnext[K - 1], br[K - 1][4], bc[K - 1][4];
#pragma unroll
        for (int comp = 0; comp < S::C3; ++comp) f4_to(x[comp], lds4(xs + T::xi_at(comp, rr + 1, 4 * q + 4)));
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            f4_to(b[i], lds4(vb0 + T::v_at(i, rr, 4 * q)));
            bnext[i] = vb0[T::v_at(i, rr, 4 * q + 4)];
            f4_to(br[i], lds4(vb0 + T::v_at(i, rr + 1, 4 * q)));
            f4_to(bc[i], lds4(vb1 + T::v_at(i, rr, 4 * q)));
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float xi_j[S::C3], b_j[K - 1], bn_j[K - 1], br_j[K - 1], bc_j[K - 1];
#pragma unroll
            for (int comp = 0; comp < S::C3; ++comp) xi_j[comp] = x[comp][j];
#pragma unroll
            for (int i = 0; i < K - 1; ++i) {
                b_j[i] = b[i][j];
                bn_j[i] = (j < 3) ? b[i][j + 1] : bnext[i];
                br_j[i] = br[i][j];
                bc_j[i] = bc[i][j];
            }
            dual_build_q<K>(qv[j], xi_j, b_j, bn_j, br_j, bc_j, nb + j + 1 < tp.ns, hr, hc, tau2);
            if (nb + j < tp.ns && !dual_first_sweep_is_identity<K>(qv[j], thr)) need |= 1u << j;
        }
    }

    // gather the voxels that need the loop, run it 32 at a time, scatter back
    float *qq = sm.queue(threadIdx.x >> 5);
    int pos[4];
    int count = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const bool mine = (need >> j) & 1u;
        const unsigned bal = __ballot_sync(0xffffffffu, mine);
        if (mine) {
            pos[j] = count + __popc(bal & ((1u << lane) - 1u));
            float *e = qq + pos[j] * S::QSTRIDE;
#pragma unroll
            for (int i = 0; i < K; ++i) {
                e[3 * i] = qv[j][i][0];
                e[3 * i + 1] = qv[j][i][1];
                e[3 * i + 2] = qv[j][i][2];
            }
        }
        count += __popc(bal);
    }
    if (count > 0) {
        __syncwarp();
        for (int e = lane; e < count; e += 32) {
            float *ent = qq + e * S::QSTRIDE;
            float qe[K][3];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                qe[i][0] = ent[3 * i];
                qe[i][1] = ent[3 * i + 1];
                qe[i][2] = ent[3 * i + 2];
            }
            dual_project<K>(qe, thr);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                ent[3 * i] = qe[i][0];
                ent[3 * i + 1] = qe[i][1];
                ent[3 * i + 2] = qe[i][2];
            }
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if ((need >> j) & 1u) {
                const float *e = qq + pos[j] * S::QSTRIDE;
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    qv[j][i][0] = e[3 * i];
                    qv[j][i][1] = e[3 * i + 1];
                    qv[j][i][2] = e[3 * i + 2];
                }
            }
        __syncwarp();
    }
    if (!live) return;

    const int64_t o = (int64_t)(ci.x + row - ci.y) * tp.nstride_w + nb;
    if (nb + 4 <= tp.ns) {
#pragma unroll
        for (int i = 0; i < K - 1; ++i)
#pragma unroll
            for (int a = 0; a < 3; ++a)
                *reinterpret_cast<float4 *>(Xout + (3 * i + a) * tp.plane_w + o) =
                    make_float4(qv[0][i][a], qv[1][i][a], qv[2][i][a], qv[3][i][a]);
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (nb + j < tp.ns)
#pragma unroll
                for (int i = 0; i < K - 1; ++i)
#pragma unroll
                    for (int a = 0; a < 3; ++a) Xout[(3 * i + a) * tp.plane_w + o + j] = qv[j][i][a];
    }
}

template <int K, int R, int NT>
__global__ void __launch_bounds__(TileShape<K, R, NT>::THREADS, 1)
    fused_tiled_kernel(const __grid_constant__ CUtensorMap tm_xi, const __grid_constant__ CUtensorMap tm_v,
                       const __grid_constant__ CUtensorMap tm_u, TiledParams tp, float *__restrict__ Xout,
                       float *__restrict__ Vout, PhaseParams<K> pp, float tau2, DykstraThresholds thr, float *dq,
                       int *err)
{
    using S = TileShape<K, R, NT>;
    using T = TiledSmem<K, R, NT>;
    extern __shared__ uint8_t smem_raw[];
    T sm;
    sm.base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));

    const int4 wk = tp.work[blockIdx.x];
    const int r0 = wk.x, n0 = wk.y, ca = wk.z, cb = wk.w;
    const int c_last = cb < tp.col_end - 1 ? cb : tp.col_end - 1;
    const int P = c_last - ca + 1;  // ring position of the last plane
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    volatile int *abort = sm.abort_flag();

    if (tid == 0) {
        for (int i = 0; i < S::D; ++i) {
            mbar_init(sm.full(i), 1);
            mbar_init(sm.ready(i), S::MAIN_WARPS + 1);
            mbar_init(sm.empty(i), S::MAIN_WARPS + 1);
        }
        *abort = 0;
        mbar_fence_init();
    }
    __syncthreads();

    float dqmax = 0.0f;
    if (warp == S::PRODUCER_WARP) {
        if (lane == 0) {
            tma_prefetch_desc(&tm_xi);
            tma_prefetch_desc(&tm_v);
            tma_prefetch_desc(&tm_u);
            for (int p = 0; p <= P; ++p) {
                if (p >= S::D && !mbar_wait_thread(sm.empty(p - S::D), T::parity(p - S::D), abort)) break;
                const int c = ca - 1 + p;
                if (p == 0 && c < tp.col_begin) {  // no plane before the first column
                    mbar_arrive(sm.full(0));
                    continue;
                }
                const int4 ci = tp.cols[c];
                const int line = ci.x + (r0 - 1 - ci.y);  // line of row r0-1 in column c
                const bool xi_only = p == 0;
                mbar_arrive_expect_tx(sm.full(p),
                                      S::XI_BYTES + (xi_only ? 0u : (uint32_t)(S::V_BYTES + S::U_BYTES)));
                tma_load_3d(sm.xi_slot(p), &tm_xi, sm.full(p), n0 - 4, line, 0);
                if (!xi_only) {
                    tma_load_3d(sm.v_slot(p), &tm_v, sm.full(p), n0, line + 1, 0);
                    tma_load_2d(sm.u_slot(p), &tm_u, sm.full(p), tp.u_x0 + n0, line + 1);
                }
            }
        }
    } else {
        const bool is_main = warp < S::MAIN_WARPS;
        const int rr = is_main ? tid / S::Q : R;
        const int q = is_main ? tid % S::Q : lane;
        const bool quad_a = is_main || lane < S::Q;
        const bool nhalo = !is_main && lane <= R;
        bool ok = true;
        for (int p = 0; p <= P && ok; ++p) {
            const int c = ca - 1 + p;
            if (p > 0) {
                if (p == 1) ok = mbar_wait_warp(sm.full(0), 0, abort);
                if (ok) ok = mbar_wait_warp(sm.full(p), T::parity(p), abort);
                if (!ok) break;
                if (quad_a) stage_a_quad<K, R, NT>(sm, tp, pp, p, c, r0, rr, n0, q, is_main && c < cb, Vout, dqmax);
                if (nhalo) stage_a_nhalo<K, R, NT>(sm, tp, pp, p, c, r0, lane, n0);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(sm.ready(p));
            if (p == 0) continue;
            if (is_main && p >= 2) {
                // dual step at plane c-1 once every warp's Vbar of that plane is in
                ok = mbar_wait_warp(sm.ready(p - 1), T::parity(p - 1), abort);
                if (!ok) break;
                stage_b_quad<K, R, NT>(sm, tp, p - 1, c - 1, r0, rr, n0, q, tau2, thr, Xout);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(sm.empty(p - 1));
        }
        // the last column of the volume has no plane after it
        if (ok && is_main && c_last == cb - 1 && P >= 1) {
            ok = mbar_wait_warp(sm.ready(P), T::parity(P), abort);
            if (ok) stage_b_quad<K, R, NT>(sm, tp, P, c_last, r0, rr, n0, q, tau2, thr, Xout);
        }
    }
    __syncthreads();
    if (tid == 0 && *abort) atomicExch(err, 1);
    if (dq) block_max_to(dqmax, dq);
}

// Copies the slab's part of u into a buffer with the state's stride, so that
// every TMA box of u starts on a 16-byte boundary.
__global__ void stage_u_kernel(Geometry g, const float *__restrict__ u, float *__restrict__ out)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    if (!p.valid) return;
    out[p.line * g.nstride_w + p.n] = u[p.line * g.nstride_in + g.slab_start + p.n];
}

}  // namespace potts
