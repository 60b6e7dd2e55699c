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
// Dykstra's full loop is needed only where some pair |q_i - q_j| exceeds 1
// (a few percent of the voxels); elsewhere its first sweep is the identity.
// Stage B tests this per voxel and appends the voxels that need the loop to a
// per-warp ring queue in shared memory that persists across planes; whenever
// 32 have gathered, each lane runs the loop on one of them and writes the
// result to global memory itself (nothing reads Xi^{m+1} during the launch).
// So the common voxels never wait for a partly idle warp.
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
#include "storage.cuh"
#include "tma.cuh"
#include "voxel.cuh"
#include "voxel_fast.cuh"

namespace potts {

// Per column: x = line of row start_row[col], y = first row, z = one past the
// last row (y = z = 0 for an empty column).
// Per volume (a work item is x = r0, the first row of the tile, y = n0,
// z = ca, w = cb).
struct TiledParams {
    const int4 *cols;
    int col_begin, col_end;
    int ns;         // slab extent along n
    int nstride_w;  // stride of the state arrays
    int64_t plane_w;
    int u_x0;       // n offset of the slab in the u tensor map
    int n_base;     // global slice of the slab's slice 0
    int it;         // 0-based iteration of the launch's primal step (keys stochastic rounding)
    int prefetch;   // planes ahead of the load ring prefetched into L2 (0: none)
    int stall_plane;  // testing: > 0 = the first work item never loads that ring position (0: off)
    int64_t line_base;  // line number of line 0 in the whole volume (keys stochastic rounding)
};

template <int K, int R, int NT, int VPT, typename ST>
struct TileShape {
    static constexpr int D = 3;  // ring depth (planes)
    static constexpr int C3 = 3 * (K - 1), C1 = K - 1, Q = NT / VPT;  // Q threads per tile row
    static constexpr int ES = (int)sizeof(ST);          // bytes per stored state value
    static constexpr int XH = ES == 4 ? 4 : 8;          // Xi box starts XH slices early (16-byte TMA start)
    static constexpr int NX = NT + 2 * XH;              // Xi box: slices n0-XH .. n0+NT+XH-1
    static constexpr int NVT = NT + (ES == 4 ? 4 : 8);  // V box: slices n0 .. (whole 16-byte rows)
    static constexpr int NV = NT + 4;                   // u and Vbar (FP32): slices n0 .. n0+NT+3
    static constexpr int MAIN = R * Q;
    static constexpr int MAIN_WARPS = MAIN / 32;
    // the high halo row, then (its own warp when POTTS_NHALO_WARP) the slice n0+NT
#ifdef POTTS_NHALO_WARP
    static constexpr int NHALO_OWN = 1;
#else
    static constexpr int NHALO_OWN = 0;
#endif
    static constexpr int HALO_WARPS = (Q + 31) / 32 + NHALO_OWN;
    static constexpr int PRODUCER_WARP = MAIN_WARPS + HALO_WARPS;
    // Dykstra warps run the projection loop of queued voxels; row warp r
    // queues for Dykstra warp r % NW (about 5 % of the voxels need the loop,
    // 2.5 sweeps on average; a lane runs one voxel at a time, so the loop's
    // latency is hidden by many lanes: 6 warps measured faster than 2, 3 or 8)
#ifdef POTTS_DYKSTRA_WARPS
    static constexpr int NW = MAIN_WARPS >= 2 * POTTS_DYKSTRA_WARPS ? POTTS_DYKSTRA_WARPS : (MAIN_WARPS >= 2 ? MAIN_WARPS / 2 : 1);
#else
    static constexpr int NW = MAIN_WARPS >= 12 ? 6 : (MAIN_WARPS >= 2 ? MAIN_WARPS / 2 : 1);
#endif
    static constexpr int DYKSTRA_WARP = PRODUCER_WARP + 1;  // the first one
    static constexpr int THREADS = MAIN + 32 * HALO_WARPS + 32 + 32 * NW;
    static constexpr int QSTRIDE = (3 * K + 1) | 1;  // queue entry: q (3K floats) + state offset; odd stride
    static constexpr int QN = 128;                     // entries of each Dykstra warp's queue (a power of 2)
    static constexpr int XI_BYTES = C3 * (R + 2) * NX * ES;
    static constexpr int V_BYTES = C1 * (R + 1) * NVT * ES;
    static constexpr int U_BYTES = (R + 1) * NV * 4;
    static constexpr int VB_BYTES = C1 * (R + 1) * NV * 4;
    static constexpr int al(int b) { return (b + 127) / 128 * 128; }
    static constexpr int XI_SLOT = al(XI_BYTES), V_SLOT = al(V_BYTES), U_SLOT = al(U_BYTES), VB_SLOT = al(VB_BYTES);
    static constexpr int OFF_XI = 0;
    static constexpr int OFF_V = OFF_XI + D * XI_SLOT;
    static constexpr int OFF_U = OFF_V + D * V_SLOT;
    static constexpr int OFF_VB = OFF_U + D * U_SLOT;
    static constexpr int OFF_Q = OFF_VB + D * VB_SLOT;
    static constexpr int OFF_QSEQ = OFF_Q + al(NW * QN * QSTRIDE * 4);
    static constexpr int OFF_QCTL = OFF_QSEQ + al(NW * QN * 4);  // per queue: tail, head, finished writers
    static constexpr int MAX_SEGMENT = 64;  // columns per work item
    static constexpr int OFF_COLS = OFF_QCTL + al(NW * 16);
    static constexpr int OFF_BAR = OFF_COLS + al((MAX_SEGMENT + 3) * 16);
    static constexpr int SMEM = OFF_BAR + 3 * D * 8 + 16;  // + abort flag
    static constexpr int SMEM_ALLOC = SMEM + 128;  // room to align the base to 128 bytes
    static_assert((VPT == 2 || VPT == 4) && NT % VPT == 0 && R + 1 <= 32, "tile shape");
    static_assert(MAIN % 32 == 0, "row threads fill whole warps");
    static_assert(SMEM_ALLOC <= 227 * 1024, "shared memory of one block");
};

// VPT consecutive stored values of shared or global memory, widened to FP32
// (and the reverse, rounding), as vector accesses.
template <int VPT, typename ST>
__device__ __forceinline__ void ldv(float (&a)[VPT], const ST *p)
{
    if constexpr (VPT == 4 && sizeof(ST) == 4) {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        a[0] = v.x, a[1] = v.y, a[2] = v.z, a[3] = v.w;
    } else if constexpr (VPT == 4 && sizeof(ST) == 2) {  // one 8-byte access
        const uint2 w = *reinterpret_cast<const uint2 *>(p);
        const float2 lo = Store<ST>::cvt2(w.x), hi = Store<ST>::cvt2(w.y);
        a[0] = lo.x, a[1] = lo.y, a[2] = hi.x, a[3] = hi.y;
    } else {
#pragma unroll
        for (int j = 0; j < VPT; j += 2) {
            const float2 v = Store<ST>::ld2(p + j);
            a[j] = v.x, a[j + 1] = v.y;
        }
    }
}
template <int VPT, typename ST>
__device__ __forceinline__ void stv(ST *p, const float (&a)[VPT])
{
    if constexpr (VPT == 4 && sizeof(ST) == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(a[0], a[1], a[2], a[3]);
    } else if constexpr (VPT == 4 && sizeof(ST) == 2) {
        *reinterpret_cast<uint2 *>(p) =
            make_uint2(Store<ST>::pack2(make_float2(a[0], a[1])), Store<ST>::pack2(make_float2(a[2], a[3])));
    } else {
#pragma unroll
        for (int j = 0; j < VPT; j += 2) Store<ST>::st2(p + j, make_float2(a[j], a[j + 1]));
    }
}

__device__ __forceinline__ bool row_in_col(int4 ci, int row) { return row >= ci.y && row < ci.z; }

template <int K, int R, int NT, int VPT, typename ST>
struct TiledSmem {
    using S = TileShape<K, R, NT, VPT, ST>;
    uint8_t *base;

    __device__ __forceinline__ ST *xi_slot(int slot) const
    {
        return reinterpret_cast<ST *>(base + S::OFF_XI + slot * S::XI_SLOT);
    }
    __device__ __forceinline__ ST *v_slot(int slot) const
    {
        return reinterpret_cast<ST *>(base + S::OFF_V + slot * S::V_SLOT);
    }
    __device__ __forceinline__ float *u_slot(int slot) const
    {
        return reinterpret_cast<float *>(base + S::OFF_U + slot * S::U_SLOT);
    }
    __device__ __forceinline__ float *vb_plane(int slot) const
    {
        return reinterpret_cast<float *>(base + S::OFF_VB + slot * S::VB_SLOT);
    }
    // queue w of voxels waiting for the projection loop: entry data, and per
    // entry the ticket + 1 of the last entry written there
    __device__ __forceinline__ float *queue_entry(int w, uint32_t ticket) const
    {
        return reinterpret_cast<float *>(base + S::OFF_Q) + (w * S::QN + (ticket & (S::QN - 1))) * S::QSTRIDE;
    }
    __device__ __forceinline__ volatile uint32_t *queue_seq(int w, uint32_t ticket) const
    {
        return reinterpret_cast<volatile uint32_t *>(base + S::OFF_QSEQ) + w * S::QN + (ticket & (S::QN - 1));
    }
    // counters of queue w: tickets handed out to writers, tickets taken by
    // its Dykstra warp, and row warps writing to it that have finished
    __device__ __forceinline__ uint32_t *q_tail(int w) const
    {
        return reinterpret_cast<uint32_t *>(base + S::OFF_QCTL) + 4 * w;
    }
    __device__ __forceinline__ volatile uint32_t *q_head(int w) const
    {
        return reinterpret_cast<volatile uint32_t *>(base + S::OFF_QCTL) + 4 * w + 1;
    }
    __device__ __forceinline__ uint32_t *q_done(int w) const
    {
        return reinterpret_cast<uint32_t *>(base + S::OFF_QCTL) + 4 * w + 2;
    }
    // row warps that write to queue w
    __device__ __forceinline__ static uint32_t q_writers(int w)
    {
        return (uint32_t)((S::MAIN_WARPS - 1 - w) / S::NW + 1);
    }
    __device__ __forceinline__ uint64_t *full(int slot) const
    {
        return reinterpret_cast<uint64_t *>(base + S::OFF_BAR) + slot;
    }
    __device__ __forceinline__ uint64_t *ready(int slot) const
    {
        return reinterpret_cast<uint64_t *>(base + S::OFF_BAR) + S::D + slot;
    }
    __device__ __forceinline__ uint64_t *empty(int slot) const
    {
        return reinterpret_cast<uint64_t *>(base + S::OFF_BAR) + 2 * S::D + slot;
    }
    // column table entries of planes ca-1 .. cb+1: index c - ca + 1; an entry
    // outside [col_begin, col_end) is all zeros (no rows)
    __device__ __forceinline__ int4 *cols() const { return reinterpret_cast<int4 *>(base + S::OFF_COLS); }
    __device__ __forceinline__ volatile int *abort_flag() const
    {
        return reinterpret_cast<volatile int *>(base + S::OFF_BAR + 3 * S::D * 8);
    }

    // element (comp, box row, box slice) of an Xi plane (slice 0 = n0 - XH), of
    // a stored V plane, and of a u / Vbar plane (slice 0 = n0 in both)
    __device__ __forceinline__ static int xi_at(int comp, int rr, int nn) { return (comp * (R + 2) + rr) * S::NX + nn; }
    __device__ __forceinline__ static int vt_at(int comp, int rr, int nn) { return (comp * (R + 1) + rr) * S::NVT + nn; }
    __device__ __forceinline__ static int v_at(int comp, int rr, int nn) { return (comp * (R + 1) + rr) * S::NV + nn; }
};

// Stage A for VPT consecutive slices n0+VPT*q .. of tile row rr (row r0+rr).
// Planes are indexed by "ring position" p = c - ca + 1 (plane ca-1 is p = 0);
// sc and sp are the ring slots of planes p and p-1.
template <int K, int R, int NT, int VPT, typename ST, bool FAST>
__device__ __forceinline__ void stage_a_chunk(const TiledSmem<K, R, NT, VPT, ST> &sm, const TiledParams &tp,
                                              const PhaseParams<K> &pp, int p, int sc, int sp, int r0, int rr,
                                              int n0, int q, bool store_v, ST *__restrict__ Vout, float &dqmax)
{
    using S = TileShape<K, R, NT, VPT, ST>;
    using T = TiledSmem<K, R, NT, VPT, ST>;
    const int row = r0 + rr;
    float *vb = sm.vb_plane(sc);
    const int4 ci = sm.cols()[p];
    const int off = VPT * q;  // offset of the chunk in the V-shaped boxes
    const int nb = n0 + off;
    if (!row_in_col(ci, row) || nb >= tp.ns) {
        float z[VPT];
#pragma unroll
        for (int j = 0; j < VPT; ++j) z[j] = 0.0f;
#pragma unroll
        for (int i = 0; i < K - 1; ++i) stv<VPT>(vb + T::v_at(i, rr, off), z);
        return;
    }
    const bool pr = row > ci.y, hr = row + 1 < ci.z;
    const bool pc = row_in_col(sm.cols()[p - 1], row);
    const bool hc = row_in_col(sm.cols()[p + 1], row);
    const ST *xs = sm.xi_slot(sc), *xp = sm.xi_slot(sp);
    const ST *vs = sm.v_slot(sc);
    const float *us = sm.u_slot(sc);
    constexpr int XH = S::XH;

    float onew[K - 1][VPT], obar[K - 1][VPT];
    if constexpr (FAST) {
        // fast arithmetic, two slices at a time with paired FP32 instructions;
        // the backward n and row terms read zeros where the neighbour is missing
        float x[S::C3][VPT], xn[K - 1][VPT], xr[K - 1][VPT], xc[K - 1][VPT], v[K - 1][VPT], u[VPT];
#pragma unroll
        for (int comp = 0; comp < S::C3; ++comp) ldv<VPT>(x[comp], xs + T::xi_at(comp, rr + 1, off + XH));
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            ldv<VPT>(xn[i], xs + T::xi_at(3 * i, rr + 1, off + XH - VPT));  // slices nb-VPT .. nb-1
            ldv<VPT>(xr[i], xs + T::xi_at(3 * i + 1, rr, off + XH));
            ldv<VPT>(xc[i], xp + T::xi_at(3 * i + 2, rr + 1, off + XH));
            ldv<VPT>(v[i], vs + T::vt_at(i, rr, off));
        }
        ldv<VPT>(u, us + T::v_at(0, rr, off));
        const float2 mpc = f2(pc ? -1.0f : -0.0f);
#pragma unroll
        for (int j = 0; j < VPT; j += 2) {
            float2 xj[S::C3], xinj[K - 1], xrj[K - 1], xcj[K - 1], vj[K - 1], vn[K - 1], vbar[K - 1];
#pragma unroll
            for (int comp = 0; comp < S::C3; ++comp) xj[comp] = f2(x[comp][j], x[comp][j + 1]);
#pragma unroll
            for (int i = 0; i < K - 1; ++i) {
                xinj[i] = f2(j == 0 ? xn[i][VPT - 1] : x[3 * i][j - 1], x[3 * i][j]);
                xrj[i] = f2(xr[i][j], xr[i][j + 1]);
                xcj[i] = f2(xc[i][j], xc[i][j + 1]);
                vj[i] = f2(v[i][j], v[i][j + 1]);
            }
            const float2 d = fast::primal<K, float2>(vn, vbar, vj, xj, xinj, xrj, xcj, mpc, f2(u[j], u[j + 1]), pp.c,
                                                    pp.lam, pp.tau1);
            const bool in0 = nb + j < tp.ns, in1 = nb + j + 1 < tp.ns;
            if (store_v) dqmax = fmaxf(dqmax, in0 ? (in1 ? fmaxf(d.x, d.y) : d.x) : 0.0f);
#pragma unroll
            for (int i = 0; i < K - 1; ++i) {
                onew[i][j] = in0 ? vn[i].x : 0.0f;
                obar[i][j] = in0 ? Store<ST>::round(vbar[i].x) : 0.0f;  // Vbar as if stored
                onew[i][j + 1] = in1 ? vn[i].y : 0.0f;
                obar[i][j + 1] = in1 ? Store<ST>::round(vbar[i].y) : 0.0f;
            }
        }
    } else if constexpr (VPT == 2) {
        // both slices with paired FP32 instructions
        float2 x[S::C3], xin[K - 1], xr[K - 1], xc[K - 1], v[K - 1], vn[K - 1], vbar[K - 1];
#pragma unroll
        for (int comp = 0; comp < S::C3; ++comp) x[comp] = Store<ST>::ld2(xs + T::xi_at(comp, rr + 1, off + XH));
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            const float2 before = Store<ST>::ld2(xs + T::xi_at(3 * i, rr + 1, off + XH - 2));  // slices nb-2, nb-1
            xin[i] = f2(before.y, x[3 * i].x);
            xr[i] = Store<ST>::ld2(xs + T::xi_at(3 * i + 1, rr, off + XH));
            xc[i] = Store<ST>::ld2(xp + T::xi_at(3 * i + 2, rr + 1, off + XH));
            v[i] = Store<ST>::ld2(vs + T::vt_at(i, rr, off));
        }
        const float2 u2 = reinterpret_cast<const float2 *>(us)[T::v_at(0, rr, off) / 2];
        const bool second = nb + 1 < tp.ns;
        const float fr = pr ? 1.0f : 0.0f, gr = hr ? 1.0f : 0.0f, fc = pc ? 1.0f : 0.0f, gc = hc ? 1.0f : 0.0f;
        const float2 d = primal_pair<K>(vn, vbar, v, x, xin, xr, xc, f2(nb > 0 ? 1.0f : 0.0f, 1.0f),
                                        f2(second ? 1.0f : 0.0f, nb + 2 < tp.ns ? 1.0f : 0.0f), f2(fr), f2(gr),
                                        f2(fc), f2(gc), u2, pp.c, pp.lam, pp.tau1);
        if (store_v) dqmax = fmaxf(dqmax, second ? fmaxf(d.x, d.y) : d.x);
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            onew[i][0] = vn[i].x;
            obar[i][0] = Store<ST>::round(vbar[i].x);  // Vbar as if stored
            onew[i][1] = second ? vn[i].y : 0.0f;
            obar[i][1] = second ? Store<ST>::round(vbar[i].y) : 0.0f;
        }
    } else {
        float x[S::C3][VPT], xn[K - 1][VPT], xr[K - 1][VPT], xc[K - 1][VPT], v[K - 1][VPT], u[VPT];
#pragma unroll
        for (int comp = 0; comp < S::C3; ++comp) ldv<VPT>(x[comp], xs + T::xi_at(comp, rr + 1, off + XH));
#pragma unroll
        for (int i = 0; i < K - 1; ++i) {
            ldv<VPT>(xn[i], xs + T::xi_at(3 * i, rr + 1, off + XH - VPT));  // the chunk before: slices nb-VPT .. nb-1
            ldv<VPT>(xr[i], xs + T::xi_at(3 * i + 1, rr, off + XH));
            ldv<VPT>(xc[i], xp + T::xi_at(3 * i + 2, rr + 1, off + XH));
            ldv<VPT>(v[i], vs + T::vt_at(i, rr, off));
        }
        ldv<VPT>(u, us + T::v_at(0, rr, off));
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            const int n = nb + j;
            float xi_j[S::C3], xin_j[K - 1], xir_j[K - 1], xic_j[K - 1], v_j[K - 1], vn[K - 1], vbar[K - 1];
#pragma unroll
            for (int comp = 0; comp < S::C3; ++comp) xi_j[comp] = x[comp][j];
#pragma unroll
            for (int i = 0; i < K - 1; ++i) {
                xin_j[i] = (j == 0) ? xn[i][VPT - 1] : x[3 * i][j - 1];
                xir_j[i] = xr[i][j];
                xic_j[i] = xc[i][j];
                v_j[i] = v[i][j];
            }
            float d = 0.0f;
            if (n < tp.ns) {
                d = primal_voxel<K>(vn, vbar, v_j, xi_j, xin_j, xir_j, xic_j, n > 0, n + 1 < tp.ns, pr, hr, pc, hc,
                                    u[j], pp.c, pp.lam, pp.tau1);
            } else {
#pragma unroll
                for (int i = 0; i < K - 1; ++i) vn[i] = vbar[i] = 0.0f;
            }
            if (store_v) dqmax = fmaxf(dqmax, d);
#pragma unroll
            for (int i = 0; i < K - 1; ++i) {
                onew[i][j] = vn[i];
                obar[i][j] = Store<ST>::round(vbar[i]);  // Vbar as if stored
            }
        }
    }
#pragma unroll
    for (int i = 0; i < K - 1; ++i) stv<VPT>(vb + T::v_at(i, rr, off), obar[i]);
    if (store_v) {
        const int64_t o = (int64_t)(ci.x + row - ci.y) * tp.nstride_w + nb;
        if constexpr (Store<ST>::kStochasticV) {
            const uint32_t line = (uint32_t)(tp.line_base + ci.x + row - ci.y);
            ST sv[K - 1][VPT];
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                uint32_t h[(K - 1 + 1) / 2];
#pragma unroll
                for (int k = 0; k < (K - 1 + 1) / 2; ++k)
                    h[k] = sr_hash(line, (uint32_t)(tp.n_base + nb + j), (uint32_t)tp.it, (uint32_t)k);
#pragma unroll
                for (int i = 0; i < K - 1; ++i) sv[i][j] = Store<ST>::st_v(onew[i][j], sr_bits(h[i >> 1], i));
            }
            if (nb + VPT <= tp.ns) {
#pragma unroll
                for (int i = 0; i < K - 1; ++i)
#pragma unroll
                    for (int j = 0; j < VPT; j += 2)
                        *reinterpret_cast<__nv_bfloat162 *>(Vout + i * tp.plane_w + o + j) =
                            __halves2bfloat162(sv[i][j], sv[i][j + 1]);
            } else {
#pragma unroll
                for (int j = 0; j < VPT; ++j)
                    if (nb + j < tp.ns)
#pragma unroll
                        for (int i = 0; i < K - 1; ++i) Vout[i * tp.plane_w + o + j] = sv[i][j];
            }
        } else if (nb + VPT <= tp.ns) {
#pragma unroll
            for (int i = 0; i < K - 1; ++i) stv<VPT>(Vout + i * tp.plane_w + o, onew[i]);
        } else {
#pragma unroll
            for (int j = 0; j < VPT; ++j)
                if (nb + j < tp.ns)
#pragma unroll
                    for (int i = 0; i < K - 1; ++i) Vout[i * tp.plane_w + o + j] = Store<ST>::st(onew[i][j]);
        }
    }
}

// Stage A for the single slice n0+NT of tile row rr (the high halo along n).
template <int K, int R, int NT, int VPT, typename ST, bool FAST>
__device__ __forceinline__ void stage_a_nhalo(const TiledSmem<K, R, NT, VPT, ST> &sm, const TiledParams &tp,
                                              const PhaseParams<K> &pp, int p, int sc, int sp, int r0, int rr, int n0)
{
    using S = TileShape<K, R, NT, VPT, ST>;
    using T = TiledSmem<K, R, NT, VPT, ST>;
    const int row = r0 + rr, n = n0 + NT;
    float *vb = sm.vb_plane(sc);
    const int4 ci = sm.cols()[p];
    if (!row_in_col(ci, row) || n >= tp.ns) {
#pragma unroll
        for (int i = 0; i < K - 1; ++i) vb[T::v_at(i, rr, NT)] = 0.0f;
        return;
    }
    const bool pr = row > ci.y, hr = row + 1 < ci.z;
    const bool pc = row_in_col(sm.cols()[p - 1], row);
    const bool hc = row_in_col(sm.cols()[p + 1], row);
    const ST *xs = sm.xi_slot(sc), *xp = sm.xi_slot(sp);
    constexpr int XN = NT + S::XH;  // slice n0+NT in the Xi box
    float xi[S::C3], xin[K - 1], xir[K - 1], xic[K - 1], v[K - 1], vn[K - 1], vbar[K - 1];
#pragma unroll
    for (int comp = 0; comp < S::C3; ++comp) xi[comp] = Store<ST>::ld(xs[T::xi_at(comp, rr + 1, XN)]);
#pragma unroll
    for (int i = 0; i < K - 1; ++i) {
        xin[i] = Store<ST>::ld(xs[T::xi_at(3 * i, rr + 1, XN - 1)]);
        xir[i] = Store<ST>::ld(xs[T::xi_at(3 * i + 1, rr, XN)]);
        xic[i] = Store<ST>::ld(xp[T::xi_at(3 * i + 2, rr + 1, XN)]);
        v[i] = Store<ST>::ld(sm.v_slot(sc)[T::vt_at(i, rr, NT)]);
    }
    const float uu = sm.u_slot(sc)[T::v_at(0, rr, NT)];
    if constexpr (FAST)
        fast::primal<K, float>(vn, vbar, v, xi, xin, xir, xic, pc ? -1.0f : -0.0f, uu, pp.c, pp.lam, pp.tau1);
    else
        primal_voxel<K>(vn, vbar, v, xi, xin, xir, xic, n > 0, n + 1 < tp.ns, pr, hr, pc, hc, uu, pp.c, pp.lam,
                        pp.tau1);
#pragma unroll
    for (int i = 0; i < K - 1; ++i) vb[T::v_at(i, rr, NT)] = Store<ST>::round(vbar[i]);
}

// The Dykstra warp: runs the projection loop of the voxels that the row warps
// queue.  It sleeps until kBatch voxels have gathered in its queue (or the
// row warps are done), then each lane takes one voxel, runs it a sweep at a
// time and, once it is done, stores the result and takes the next waiting
// ticket, until the queue is empty and every lane has finished.  It returns
// when every row warp has finished and the queue is empty, or when the block
// aborts.  Every wait is bounded.
constexpr int kQueueSpin = 1 << 20;   // polls of an entry's publication flag
constexpr int kIdleRounds = 1 << 23;  // idle polls (~400 ns each) while the row warps work
#ifdef POTTS_DYKSTRA_BATCH
constexpr uint32_t kBatch = POTTS_DYKSTRA_BATCH;
#else
constexpr uint32_t kBatch = 1;  // queued voxels that start a batch (larger batches measured no faster)
#endif

template <int K, int R, int NT, int VPT, typename ST, bool FAST>
__device__ __forceinline__ void dykstra_worker(const TiledSmem<K, R, NT, VPT, ST> &sm, int w, const TiledParams &tp,
                                               DykstraThresholds thr, ST *__restrict__ Xout, volatile int *abort)
{
    constexpr int kPairs = K * (K - 1) / 2;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    using T = TiledSmem<K, R, NT, VPT, ST>;
    volatile uint32_t *tail_v = sm.q_tail(w);
    volatile uint32_t *done_v = sm.q_done(w);
    float qe[K][3], P[kPairs][3];
    int64_t o = 0;
    int sweeps = 0;
    bool active = false, batch = false;
    uint32_t next = 0;  // next ticket to hand out (the same in every lane)
    int idle_rounds = 0;
    while (true) {
        if (!batch) {
            // a row warp publishes its last entries before it counts itself
            // done, so `done` is read before the tail
            const bool done = __shfl_sync(0xffffffffu, (int)(*done_v == T::q_writers(w)), 0) != 0;
            const uint32_t avail = __shfl_sync(0xffffffffu, *tail_v, 0) - next;
            if (avail >= kBatch || (done && avail > 0u)) {
                batch = true;
            } else if (done || __shfl_sync(0xffffffffu, *abort, 0)) {
                break;
            } else {
                if (++idle_rounds > kIdleRounds) {
                    *abort = 1;
                    break;
                }
                __nanosleep(400);
                continue;
            }
            idle_rounds = 0;
        }
        const uint32_t avail = __shfl_sync(0xffffffffu, *tail_v, 0) - next;
        const unsigned idle = __ballot_sync(0xffffffffu, !active);
        if (avail > 0u && idle != 0u) {
            const uint32_t take = min((uint32_t)__popc(idle), avail);
            const uint32_t rank = (uint32_t)__popc(idle & below);
            if (!active && rank < take) {
                const uint32_t ticket = next + rank;
                volatile uint32_t *seq = sm.queue_seq(w, ticket);
                int spins = 0;
                bool published = *seq == ticket + 1u;
                while (!published && spins < kQueueSpin && !*abort) {
                    ++spins;
                    published = *seq == ticket + 1u;
                }
                if (published) {
                    __threadfence_block();
                    const float *ent = sm.queue_entry(w, ticket);
#pragma unroll
                    for (int i = 0; i < K; ++i) {
                        qe[i][0] = ent[3 * i];
                        qe[i][1] = ent[3 * i + 1];
                        qe[i][2] = ent[3 * i + 2];
                    }
                    o = (int64_t)(uint32_t)__float_as_int(ent[3 * K]);
#pragma unroll
                    for (int p = 0; p < kPairs; ++p) P[p][0] = P[p][1] = P[p][2] = 0.0f;
                    sweeps = 0;
                    active = true;
                } else {
                    *abort = 1;
                }
            }
            next += take;
            __threadfence_block();
            __syncwarp();
            if (lane == 0) *sm.q_head(w) = next;  // the taken entries' slots are free again
        }
        if (!__any_sync(0xffffffffu, active)) {
            batch = false;  // the queue ran dry: wait for the next batch
            if (__shfl_sync(0xffffffffu, *abort, 0)) break;
            continue;
        }
        if (active) {
            bool exit;
            if constexpr (FAST)
                exit = fast::dykstra_sweep<K>(qe, P);
            else
                exit = dykstra_sweep<K>(qe, P, thr);
            if (exit || ++sweeps == 20) {
#pragma unroll
                for (int i = 0; i < K - 1; ++i)
#pragma unroll
                    for (int a = 0; a < 3; ++a) Xout[(3 * i + a) * tp.plane_w + o] = Store<ST>::st(qe[i][a]);
                active = false;
            }
        }
    }
}

// Stage B: dual step at ring position p (slot sc; slot sn holds plane p+1)
// for VPT slices n0+VPT*q .. of tile row rr.  Called by every lane of the row
// warps (warp-wide ballots); voxels that need the projection loop go to the
// block's queue.
template <int K, int R, int NT, int VPT, typename ST, bool FAST>
__device__ __forceinline__ void stage_b_chunk(const TiledSmem<K, R, NT, VPT, ST> &sm, const TiledParams &tp, int p,
                                              int sc, int sn, int r0, int rr, int n0, int q, float tau2,
                                              DykstraThresholds thr, ST *__restrict__ Xout)
{
    using S = TileShape<K, R, NT, VPT, ST>;
    using T = TiledSmem<K, R, NT, VPT, ST>;
    const int lane = threadIdx.x & 31;
    const int row = r0 + rr;
    const int4 ci = sm.cols()[p];
    const int off = VPT * q;
    const int nb = n0 + off;
    const bool live = row_in_col(ci, row) && nb < tp.ns;
    const int64_t o = (int64_t)(ci.x + row - ci.y) * tp.nstride_w + nb;

    float qv[VPT][K][3];
    unsigned need = 0;  // bit j: slice nb+j needs the full projection loop
    if (live) {
        const bool hr = row + 1 < ci.z;
        const bool hc = row_in_col(sm.cols()[p + 1], row);
        const ST *xs = sm.xi_slot(sc);
        const float *vb0 = sm.vb_plane(sc), *vb1 = sm.vb_plane(sn);
        constexpr int XH = S::XH;
        if constexpr (FAST) {
            float x[S::C3][VPT], b[K - 1][VPT], bnext[K - 1], br[K - 1][VPT], bc[K - 1][VPT];
#pragma unroll
            for (int comp = 0; comp < S::C3; ++comp) ldv<VPT>(x[comp], xs + T::xi_at(comp, rr + 1, off + XH));
#pragma unroll
            for (int i = 0; i < K - 1; ++i) {
                ldv<VPT>(b[i], vb0 + T::v_at(i, rr, off));
                bnext[i] = vb0[T::v_at(i, rr, off + VPT)];
                ldv<VPT>(br[i], vb0 + T::v_at(i, rr + 1, off));
                ldv<VPT>(bc[i], vb1 + T::v_at(i, rr, off));
            }
            const float2 t2r = f2(hr ? tau2 : 0.0f), t2c = f2(hc ? tau2 : 0.0f);
#pragma unroll
            for (int j = 0; j < VPT; j += 2) {
                float2 xj[S::C3], bj[K - 1], bnj[K - 1], brj[K - 1], bcj[K - 1], q2[K][3];
#pragma unroll
                for (int comp = 0; comp < S::C3; ++comp) xj[comp] = f2(x[comp][j], x[comp][j + 1]);
#pragma unroll
                for (int i = 0; i < K - 1; ++i) {
                    bj[i] = f2(b[i][j], b[i][j + 1]);
                    bnj[i] = f2(b[i][j + 1], j + 2 < VPT ? b[i][j + 2] : bnext[i]);
                    brj[i] = f2(br[i][j], br[i][j + 1]);
                    bcj[i] = f2(bc[i][j], bc[i][j + 1]);
                }
                const float2 t2n = f2(nb + j + 1 < tp.ns ? tau2 : 0.0f, nb + j + 2 < tp.ns ? tau2 : 0.0f);
                fast::dual_q<K, float2>(q2, xj, bj, bnj, brj, bcj, t2n, t2r, t2c);
                const float2 m = fast::max_pair_dist2<K, float2>(q2);
                if (m.x > 1.0f && nb + j < tp.ns) need |= 1u << j;
                if (m.y > 1.0f && nb + j + 1 < tp.ns) need |= 2u << j;
#pragma unroll
                for (int i = 0; i < K; ++i)
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        qv[j][i][a] = q2[i][a].x;
                        qv[j + 1][i][a] = q2[i][a].y;
                    }
            }
        } else if constexpr (VPT == 2) {
            float2 x[S::C3], b[K - 1], bn[K - 1], br[K - 1], bc[K - 1], q2[K][3];
#pragma unroll
            for (int comp = 0; comp < S::C3; ++comp)
                x[comp] = Store<ST>::ld2(xs + T::xi_at(comp, rr + 1, off + XH));
#pragma unroll
            for (int i = 0; i < K - 1; ++i) {
                b[i] = reinterpret_cast<const float2 *>(vb0)[T::v_at(i, rr, off) / 2];
                bn[i] = f2(b[i].y, vb0[T::v_at(i, rr, off + 2)]);
                br[i] = reinterpret_cast<const float2 *>(vb0)[T::v_at(i, rr + 1, off) / 2];
                bc[i] = reinterpret_cast<const float2 *>(vb1)[T::v_at(i, rr, off) / 2];
            }
            dual_build_q_pair<K>(q2, x, b, bn, br, bc, f2(nb + 1 < tp.ns ? 1.0f : 0.0f, nb + 2 < tp.ns ? 1.0f : 0.0f),
                                 f2(hr ? 1.0f : 0.0f), f2(hc ? 1.0f : 0.0f), tau2);
            need = dual_needs_loop_pair<K>(q2, thr) & (nb + 1 < tp.ns ? 3u : 1u);
#pragma unroll
            for (int i = 0; i < K; ++i)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    qv[0][i][a] = q2[i][a].x;
                    qv[1][i][a] = q2[i][a].y;
                }
        } else {
            float x[S::C3][VPT], b[K - 1][VPT], bnext[K - 1], br[K - 1][VPT], bc[K - 1][VPT];
#pragma unroll
            for (int comp = 0; comp < S::C3; ++comp) ldv<VPT>(x[comp], xs + T::xi_at(comp, rr + 1, off + XH));
#pragma unroll
            for (int i = 0; i < K - 1; ++i) {
                ldv<VPT>(b[i], vb0 + T::v_at(i, rr, off));
                bnext[i] = vb0[T::v_at(i, rr, off + VPT)];
                ldv<VPT>(br[i], vb0 + T::v_at(i, rr + 1, off));
                ldv<VPT>(bc[i], vb1 + T::v_at(i, rr, off));
            }
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                float xi_j[S::C3], b_j[K - 1], bn_j[K - 1], br_j[K - 1], bc_j[K - 1];
#pragma unroll
                for (int comp = 0; comp < S::C3; ++comp) xi_j[comp] = x[comp][j];
#pragma unroll
                for (int i = 0; i < K - 1; ++i) {
                    b_j[i] = b[i][j];
                    bn_j[i] = (j < VPT - 1) ? b[i][j + 1] : bnext[i];
                    br_j[i] = br[i][j];
                    bc_j[i] = bc[i][j];
                }
                dual_build_q<K>(qv[j], xi_j, b_j, bn_j, br_j, bc_j, nb + j + 1 < tp.ns, hr, hc, tau2);
                if (nb + j < tp.ns && !dual_first_sweep_is_identity<K>(qv[j], thr)) need |= 1u << j;
            }
        }
    }

    // Every voxel's q is stored at once, whole vectors in every lane (no lane
    // takes a separate path for its loop voxels).  The voxels that need the
    // projection loop are stored again, with the loop's result, by the Dykstra
    // warp that runs them (their queue entries are published behind a block
    // fence, after this store) or by the lane itself when the queue is full.
    if (live) {
        if (nb + VPT <= tp.ns) {
#pragma unroll
            for (int i = 0; i < K - 1; ++i)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    float w[VPT];
#pragma unroll
                    for (int j = 0; j < VPT; ++j) w[j] = qv[j][i][a];
                    stv<VPT>(Xout + (3 * i + a) * tp.plane_w + o, w);
                }
        } else {
#pragma unroll
            for (int j = 0; j < VPT; ++j)
                if (nb + j < tp.ns)
#pragma unroll
                    for (int i = 0; i < K - 1; ++i)
#pragma unroll
                        for (int a = 0; a < 3; ++a)
                            Xout[(3 * i + a) * tp.plane_w + o + j] = Store<ST>::st(qv[j][i][a]);
        }
    }

    // the loop voxels of the whole warp go to the block's queue in one
    // reservation (the Dykstra warp runs them); when it is full, each lane
    // runs the loop of its own voxels
    unsigned bal[VPT];
    uint32_t total = 0;
#pragma unroll
    for (int j = 0; j < VPT; ++j) {
        bal[j] = __ballot_sync(0xffffffffu, (need >> j) & 1u);
        total += (uint32_t)__popc(bal[j]);
    }
    if (total == 0u) return;
    uint32_t base = 0;
    bool queued = false;
    const int w = (threadIdx.x >> 5) % S::NW;
    if (lane == 0) {
        uint32_t *tail = sm.q_tail(w);
        uint32_t t = *reinterpret_cast<volatile uint32_t *>(tail);
        for (int tries = 0; tries < 64; ++tries) {
            if (t + total - *sm.q_head(w) > (uint32_t)S::QN) break;  // no room
            const uint32_t prev = atomicCAS(tail, t, t + total);
            if (prev == t) {
                queued = true;
                base = t;
                break;
            }
            t = prev;
        }
    }
    queued = __shfl_sync(0xffffffffu, queued, 0);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (need == 0u) return;
    const unsigned lower = (1u << lane) - 1u;
    if (queued) {
        uint32_t first = base, tickets[VPT];
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            tickets[j] = first + (uint32_t)__popc(bal[j] & lower);
            first += (uint32_t)__popc(bal[j]);
        }
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            if (!((need >> j) & 1u)) continue;
            float *e = sm.queue_entry(w, tickets[j]);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                e[3 * i] = qv[j][i][0];
                e[3 * i + 1] = qv[j][i][1];
                e[3 * i + 2] = qv[j][i][2];
            }
            e[3 * K] = __int_as_float((int)(o + j));
        }
        __threadfence_block();
#pragma unroll
        for (int j = 0; j < VPT; ++j)
            if ((need >> j) & 1u) *sm.queue_seq(w, tickets[j]) = tickets[j] + 1u;
    } else {
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            if (!((need >> j) & 1u)) continue;
            if constexpr (FAST)
                fast::dual_project<K>(qv[j]);
            else
                dual_project<K>(qv[j], thr);
#pragma unroll
            for (int i = 0; i < K - 1; ++i)
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    Xout[(3 * i + a) * tp.plane_w + o + j] = Store<ST>::st(qv[j][i][a]);
        }
    }
}

// Everything a launch needs about one volume: tensor maps of both ping-pong
// halves of Xi and V and of u, its tables, its state buffers, its phase
// parameters and its convergence trace.  Lives in device memory (one entry
// per volume of a batch); 64-byte aligned through CUtensorMap.
template <int K, typename ST>
struct FusedVolume {
    CUtensorMap xi[2], v[2], u;
    TiledParams tp;
    ST *xi_buf[2], *v_buf[2];
    PhaseParams<K> pp;
    float *dq;  // per-iteration max |dV|^2 of this volume, or null
};

// The work of one block on one work item: a tile row range x slice range
// marching over up to 64 columns of one volume (work_vol[item], or volume 0
// when work_vol is null).  It turns (Xi^m, V^{m-1}) in half `in` into
// (Xi^{m+1}, V^m) in half in ^ 1 for the item's voxels; it = m - 1.
// `reinit`: the block ran an earlier item, so its mbarriers are invalidated
// before they are initialised again.  Ends with a block-wide barrier.
template <int K, int R, int NT, int VPT, typename ST, bool FAST>
__device__ __forceinline__ void tiled_item(const TiledSmem<K, R, NT, VPT, ST> &sm,
                                           const FusedVolume<K, ST> *__restrict__ vols, const int4 *__restrict__ work,
                                           const int *__restrict__ work_vol, int item, bool reinit, int in, int it,
                                           float tau2, DykstraThresholds thr, int *err)
{
    using S = TileShape<K, R, NT, VPT, ST>;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    volatile int *abort = sm.abort_flag();
    {
        if (tid == 0) {
            for (int i = 0; i < S::D; ++i) {
                if (reinit) {
                    mbar_inval(sm.full(i));
                    mbar_inval(sm.ready(i));
                    mbar_inval(sm.empty(i));
                }
                mbar_init(sm.full(i), 1);
                mbar_init(sm.ready(i), S::MAIN_WARPS + S::HALO_WARPS);
                mbar_init(sm.empty(i), S::MAIN_WARPS + S::HALO_WARPS);
            }
            *abort = 0;
            for (int w = 0; w < S::NW; ++w) {
                *sm.q_tail(w) = 0u;
                *sm.q_head(w) = 0u;
                *sm.q_done(w) = 0u;
            }
            mbar_fence_init();
        }
        const FusedVolume<K, ST> *vol = vols + (work_vol ? work_vol[item] : 0);
        TiledParams tp = vol->tp;
        tp.it = it;
        const PhaseParams<K> pp = vol->pp;
        ST *const Xout = vol->xi_buf[in ^ 1];
        ST *const Vout = vol->v_buf[in ^ 1];
        const CUtensorMap *tm_xi = &vol->xi[in], *tm_v = &vol->v[in], *tm_u = &vol->u;

        const int4 wk = work[item];
        const int r0 = wk.x, n0 = wk.y, ca = wk.z, cb = wk.w;
        const int c_last = cb < tp.col_end - 1 ? cb : tp.col_end - 1;
        const int P = c_last - ca + 1;  // ring position of the last plane

        for (int i = tid; i <= P + 1; i += blockDim.x) {
            const int c = ca - 1 + i;
            sm.cols()[i] = (c >= tp.col_begin && c < tp.col_end) ? tp.cols[c] : make_int4(0, 0, 0, 0);
        }
        {  // Vbar planes start as zeros: a missing neighbour's value is multiplied by 0, so it must be finite
            float *vb = sm.vb_plane(0);
            for (int i = tid; i < S::D * S::VB_SLOT / 4; i += blockDim.x) vb[i] = 0.0f;
        }
        for (int i = tid; i < S::NW * S::QN; i += blockDim.x) *sm.queue_seq(i / S::QN, (uint32_t)i) = 0u;
        if (ca - 1 < tp.col_begin) {  // no plane before the first column: its Xi slot reads as zeros
            uint32_t *x0 = reinterpret_cast<uint32_t *>(sm.xi_slot(0));
            for (int i = tid; i < S::XI_SLOT / 4; i += blockDim.x) x0[i] = 0u;
        }
        __syncthreads();

        float dqmax = 0.0f;
        if (warp == S::PRODUCER_WARP) {
            if (lane == 0) {
                // the maps were written by copies before the launch
                tma_fence_acquire_desc(tm_xi);
                tma_fence_acquire_desc(tm_v);
                tma_fence_acquire_desc(tm_u);
                // the state was written through the generic proxy (an earlier
                // iteration of a persistent launch); the loads use the async proxy
                fence_proxy_async_global();
                tma_prefetch_desc(tm_xi);
                tma_prefetch_desc(tm_v);
                tma_prefetch_desc(tm_u);
                // slot and phase parity of ring position p; waits for the release
                // of the plane D positions back in the same slot
                int slot = 0;
                uint32_t ph = 0;
                int issued = 0;  // positions whose loads are in flight or done
                for (int p = 0; p <= P; ++p) {
                    if (p >= S::D && !mbar_wait_thread(sm.empty(slot), ph ^ 1u, abort)) break;
                    const int c = ca - 1 + p;
                    if (p == 0 && c < tp.col_begin) {  // no plane before the first column
                        mbar_arrive(sm.full(0));
                    } else if (tp.stall_plane > 0 && p == tp.stall_plane && item == 0) {
                        // testing: this plane never arrives, so the waits for it run out
                    } else {
                        const int4 ci = sm.cols()[p];
                        const int line = ci.x + (r0 - 1 - ci.y);  // line of row r0-1 in column c
                        const bool xi_only = p == 0;
                        mbar_arrive_expect_tx(sm.full(slot),
                                              S::XI_BYTES + (xi_only ? 0u : (uint32_t)(S::V_BYTES + S::U_BYTES)));
                        tma_load_3d(sm.xi_slot(slot), tm_xi, sm.full(slot), n0 - S::XH, line, 0);
                        if (!xi_only) {
                            tma_load_3d(sm.v_slot(slot), tm_v, sm.full(slot), n0, line + 1, 0);
                            tma_load_2d(sm.u_slot(slot), tm_u, sm.full(slot), tp.u_x0 + n0, line + 1);
                        }
                    }
                    issued = p + 1;
                    // L2 prefetch of the plane tp.prefetch positions ahead (the
                    // ring's depth bounds what is in flight into shared memory)
                    const int pf = p + tp.prefetch;
                    if (tp.prefetch > 0 && pf <= P && ca - 1 + pf >= tp.col_begin) {
                        const int4 cf = sm.cols()[pf];
                        const int lf = cf.x + (r0 - 1 - cf.y);
                        tma_prefetch_l2_3d(tm_xi, n0 - S::XH, lf, 0);
                        tma_prefetch_l2_3d(tm_v, n0, lf + 1, 0);
                        tma_prefetch_l2_2d(tm_u, tp.u_x0 + n0, lf + 1);
                    }
                    if (++slot == S::D) slot = 0, ph ^= 1u;
                }
                if (*abort) {
                    // the consumers gave up: wait (bounded) for the loads still in
                    // flight so that none lands after this block moves on
                    for (int q = issued > S::D ? issued - S::D : 0; q < issued; ++q)
                        mbar_wait_bounded(sm.full(q % S::D), (uint32_t)((q / S::D) & 1), kDrainTries);
                }
            }
        } else if (warp >= S::DYKSTRA_WARP) {
            dykstra_worker<K, R, NT, VPT, ST, FAST>(sm, warp - S::DYKSTRA_WARP, tp, thr, Xout, abort);
        } else {
            const bool is_main = warp < S::MAIN_WARPS;
            const int hq = tid - S::MAIN;  // chunk of the halo row (halo warps)
            const int rr = is_main ? tid / S::Q : R;
            const int q = is_main ? tid % S::Q : hq;
            const bool chunk_a = is_main || hq < S::Q;
            // lanes of the first halo warp, or of the last one when it has its own
            const int hn = S::NHALO_OWN ? hq - 32 * (S::HALO_WARPS - 1) : hq;
            const bool nhalo = !is_main && hn >= 0 && hn <= R;
            bool ok = true;
            // ring slots of positions p-1, p, p+1 and the barrier parities of p-1, p
            int s_prev = S::D - 1, s_cur = 0, s_next = 1;
            uint32_t ph_prev = 1, ph_cur = 0;
            for (int p = 0; p <= P && ok; ++p) {
                if (p > 0) {
                    if (p == 1) ok = mbar_wait_warp(sm.full(0), 0, abort);
                    if (ok) ok = mbar_wait_warp(sm.full(s_cur), ph_cur, abort);
                    if (!ok) break;
                    if (chunk_a)
                        stage_a_chunk<K, R, NT, VPT, ST, FAST>(sm, tp, pp, p, s_cur, s_prev, r0, rr, n0, q,
                                                         is_main && ca - 1 + p < cb, Vout, dqmax);
                    if (nhalo) stage_a_nhalo<K, R, NT, VPT, ST, FAST>(sm, tp, pp, p, s_cur, s_prev, r0, hn, n0);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(sm.ready(s_cur));
                if (p > 0) {
                    if (is_main && p >= 2) {
                        // dual step at position p-1 once every warp's Vbar of that plane is in
                        ok = mbar_wait_warp(sm.ready(s_prev), ph_prev, abort);
                        if (!ok) break;
                        stage_b_chunk<K, R, NT, VPT, ST, FAST>(sm, tp, p - 1, s_prev, s_cur, r0, rr, n0, q, tau2, thr,
                                                         Xout);
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(sm.empty(s_prev));
                }
                s_prev = s_cur;
                ph_prev = ph_cur;
                s_cur = s_next;
                if (s_cur == 0) ph_cur ^= 1u;
                s_next = (s_next + 1 == S::D) ? 0 : s_next + 1;
            }
            // the last column of the volume has no plane after it (s_prev now holds position P)
            if (ok && is_main && c_last == cb - 1) {
                ok = mbar_wait_warp(sm.ready(s_prev), ph_prev, abort);
                if (ok)
                    stage_b_chunk<K, R, NT, VPT, ST, FAST>(sm, tp, P, s_prev, s_cur, r0, rr, n0, q, tau2, thr, Xout);
            }
            if (is_main) {  // this warp queues nothing more (also after an abort)
                __syncwarp();
                if (lane == 0) {
                    __threadfence_block();
                    atomicAdd(sm.q_done(warp % S::NW), 1u);
                }
            }
        }
        // this item's stores (generic proxy) before any later TMA load of them
        // (the next iteration of a persistent launch)
        fence_proxy_async_global();
        __syncthreads();
        if (tid == 0 && *abort) atomicExch(err, 1);
        if (vol->dq) block_max_to(dqmax, vol->dq + it);
    }
}

// 128-byte aligned view of the dynamic shared memory of a fused launch.
template <int K, int R, int NT, int VPT, typename ST>
__device__ __forceinline__ TiledSmem<K, R, NT, VPT, ST> tiled_smem()
{
    extern __shared__ __align__(128) uint8_t smem_raw[];
    TiledSmem<K, R, NT, VPT, ST> sm;
    // align by pointer arithmetic on the shared array itself, so that the
    // compiler keeps every access a shared-memory access
    sm.base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
    return sm;
}

// One block per work item; the items of every volume of a batch share one
// launch, and the block scheduler hands them out as blocks finish.  The launch
// turns (Xi^m, V^{m-1}) in half `in` into (Xi^{m+1}, V^m) in half in ^ 1;
// it = m - 1.
template <int K, int R, int NT, int VPT, typename ST, bool FAST>
__global__ void __launch_bounds__(TileShape<K, R, NT, VPT, ST>::THREADS, 1)
    fused_tiled_kernel(const FusedVolume<K, ST> *__restrict__ vols, const int4 *__restrict__ work,
                       const int *__restrict__ work_vol, int in, int it, float tau2, DykstraThresholds thr, int *err)
{
    const auto sm = tiled_smem<K, R, NT, VPT, ST>();
    tiled_item<K, R, NT, VPT, ST, FAST>(sm, vols, work, work_vol, (int)blockIdx.x, false, in, it, tau2, thr, err);
}

// Control words of a persistent launch (device memory, zeroed before it):
// ctl[0] counts the blocks that finished an iteration, ctl[1] is set when a
// block gave up (every block then leaves), ctl[2 + m] hands out the work items
// of the launch's iteration m.
constexpr int kPersistentCtlHead = 2;
// Polls (each followed by a ~256 ns sleep) of the grid barrier before a block
// gives up: about 2 s.
constexpr int kGridWaitTries = 1 << 23;

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of a persistent launch, called by thread 0 of every block
// after a block-wide barrier: waits (bounded) until `target` block arrivals
// have been counted.  False when the launch is aborting or the wait ran out
// (which then aborts the launch).
__device__ __forceinline__ bool grid_barrier(uint32_t *ctl, uint32_t target)
{
    volatile int *gabort = reinterpret_cast<volatile int *>(ctl + 1);
    __threadfence();
    atomicAdd(ctl, 1u);
    for (int i = 0; i < kGridWaitTries; ++i) {
        if (ld_acquire_gpu(ctl) >= target) return true;
        if (*gabort) return false;
        __nanosleep(256);
    }
    atomicExch(reinterpret_cast<int *>(ctl + 1), 1);
    return false;
}

// The iterations it0 .. it0 + n_iters - 1 of the fused form in one launch:
// every block of the grid is resident (cooperative launch), takes the work
// items of an iteration one at a time from a counter, and waits at a grid-wide
// barrier before the next iteration (whose items read the halos that other
// blocks wrote).  Iteration m of the launch turns state half (in0 + m) & 1
// into the other half, like fused_tiled_kernel.  The result does not depend on
// the grid size or the order in which blocks take items.
template <int K, int R, int NT, int VPT, typename ST, bool FAST>
__global__ void __launch_bounds__(TileShape<K, R, NT, VPT, ST>::THREADS, 1)
    fused_persistent_kernel(const FusedVolume<K, ST> *__restrict__ vols, const int4 *__restrict__ work,
                            const int *__restrict__ work_vol, int n_work, int in0, int it0, int n_iters, float tau2,
                            DykstraThresholds thr, int *err, uint32_t *ctl)
{
    const auto sm = tiled_smem<K, R, NT, VPT, ST>();
    // The schedule lives in shared memory and only thread 0 changes it, so no
    // register carries state across an item (the item body needs them all).
    // s_m: the block's current iteration; s_item: its next item, or -1 when
    // the block is done; s_items: items the block has run.
    __shared__ int s_m, s_item, s_items;
    if (threadIdx.x == 0) s_m = 0, s_items = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            int m = s_m, item = -1;
            while (m < n_iters) {
                if (*reinterpret_cast<volatile int *>(ctl + 1)) break;  // aborting
                item = (int)atomicAdd(ctl + kPersistentCtlHead + m, 1u);
                if (item < n_work) break;
                item = -1;
                // every item of iteration m is taken: wait for the grid before
                // the next iteration reads the halos that other blocks write
                if (m + 1 == n_iters) break;
                if (!grid_barrier(ctl, (uint32_t)(m + 1) * gridDim.x)) {
                    atomicExch(err, 1);
                    break;
                }
                ++m;
            }
            s_m = m;
            s_item = item;
        }
        __syncthreads();
        const int item = s_item;
        if (item < 0) break;
        const int m = s_m;
        tiled_item<K, R, NT, VPT, ST, FAST>(sm, vols, work, work_vol, item, s_items > 0, (in0 + m) & 1, it0 + m,
                                            tau2, thr, err);
        if (threadIdx.x == 0) {
            s_items += 1;
            if (*sm.abort_flag()) atomicExch(reinterpret_cast<int *>(ctl + 1), 1);
        }
    }
}

// One launch of fused_tiled_kernel<K, R, NT, VPT, ST, FAST> over n_work
// items on `stream`.  Defined in fused_launch.cuh and instantiated for the
// compiled tile shapes in the fused_*.cu translation units.
template <int K, int R, int NT, int VPT, typename ST, bool FAST>
cudaError_t launch_fused(cudaStream_t stream, const FusedVolume<K, ST> *vols, const int4 *work, const int *work_vol,
                         int n_work, int in, int it, float tau2, DykstraThresholds thr, int *err);

// One persistent launch of fused_persistent_kernel<K, R, NT, VPT, ST, FAST>
// running n_iters iterations (state half in0, iteration it0 first) over
// n_work items, on `stream`; ctl holds 2 + n_iters zeroed words.  The grid
// is one block per SM times the blocks an SM holds (at most n_work), launched
// cooperatively so that every block is resident.
template <int K, int R, int NT, int VPT, typename ST, bool FAST>
cudaError_t launch_fused_persistent(cudaStream_t stream, const FusedVolume<K, ST> *vols, const int4 *work,
                                    const int *work_vol, int n_work, int in0, int it0, int n_iters, float tau2,
                                    DykstraThresholds thr, int *err, uint32_t *ctl);

// Copies the slab's part of u into a buffer with the state's stride, so that
// every TMA box of u starts on a 16-byte boundary.
static __global__ void stage_u_kernel(Geometry g, const float *__restrict__ u, float *__restrict__ out)
{
    const PlainIndex p = plain_index(g, 0, g.ns);
    if (!p.valid) return;
    out[p.line * g.nstride_w + p.n] = u[p.line * g.nstride_in + g.slab_start + p.n];
}

}  // namespace potts
