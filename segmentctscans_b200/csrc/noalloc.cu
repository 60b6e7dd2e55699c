// potts_energies_static: the FP64 energies of a solver state, computed without
// allocating any device memory.
//
// Some callers cannot call cudaMalloc: a host framework that owns the device
// memory pool and forbids allocations by plug-ins, a process whose device
// memory is reserved in full up front, or a real-time loop that cannot afford
// an allocation's implicit synchronisation.  This entry point serves them: the
// caller passes u, V and Xi (device) and a host array for the result; the only
// working memory is the file-scope arrays below, which every GPU that loads
// this library holds until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/potts_b200.h"

namespace {

constexpr int kBlocks = 1184;  // 8 blocks per SM of a 148-SM B200
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kTableChunk = 512;

// Working memory: per column (line of its first row, first row, end row), one
// (lagrangian, dual) partial sum per block, and the three results.
__device__ __align__(256) int4 g_static_cols[POTTS_STATIC_MAX_COLS];
__device__ __align__(256) double2 g_static_partial[kBlocks];
__device__ __align__(256) double g_static_out[3];

struct StaticAddresses {
    int4 *cols = nullptr;
    double2 *partial = nullptr;
    double *out = nullptr;
};

// Device addresses of the arrays on the current device.  In host code the
// arrays' names are host-side stand-ins, not device addresses.  The lookup
// allocates nothing and is repeated on every call, so that an address is never
// stale (a cudaDeviceReset between calls reloads the module, possibly at a new
// address); the first lookup in a process may load the library's device code.
int device_addresses(StaticAddresses *a, std::string *err)
{
    StaticAddresses s;
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&s.cols), g_static_cols);
    if (e == cudaSuccess) e = cudaGetSymbolAddress(reinterpret_cast<void **>(&s.partial), g_static_partial);
    if (e == cudaSuccess) e = cudaGetSymbolAddress(reinterpret_cast<void **>(&s.out), g_static_out);
    if (e != cudaSuccess) {
        *err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        return POTTS_ECUDA;
    }
    *a = s;
    return POTTS_OK;
}

struct StaticGeom {
    int col_begin, col_end;
    int n;          // slices per line
    int nstride;    // stride of n in u, V and Xi
    int64_t plane;  // stride between the components of V and Xi (the span)
};

struct Labels {
    double c[POTTS_MAX_PHASES];
};

// Block-strided pass over the columns; in a column, the warps take its lines
// (rows) in turn and the lanes the slices of a line.  Per voxel the solver's
// energy terms: e_i = lam (u - c_i)^2 - div Xi_i, L += sum_i V_i e_i,
// D += min_i e_i.
template <int K>
__global__ void __launch_bounds__(kThreads)
    static_energy_kernel(StaticGeom g, const int4 *__restrict__ cols, const float *__restrict__ u,
                         const float *__restrict__ V, const float *__restrict__ xi, double lam, Labels lb,
                         double2 *partial)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double lag = 0.0, dual = 0.0;
    for (int col = g.col_begin + blockIdx.x; col < g.col_end; col += gridDim.x) {
        const int4 ci = cols[col];
        const int4 cp = col > g.col_begin ? cols[col - 1] : make_int4(0, 0, 0, 0);
        const int4 cn = col + 1 < g.col_end ? cols[col + 1] : make_int4(0, 0, 0, 0);
        for (int row = ci.y + warp; row < ci.z; row += kWarps) {
            for (int n = lane; n < g.n; n += 32) {
            const int64_t o = (int64_t)(ci.x + row - ci.y) * g.nstride + n;
            const bool hn = n + 1 < g.n, pn = n > 0;
            const bool hr = row + 1 < ci.z, pr = row > ci.y;
            const bool hc = row >= cn.y && row < cn.z, pc = row >= cp.y && row < cp.z;
            const int64_t opc = pc ? (int64_t)(cp.x + row - cp.y) * g.nstride + n : o;
            const double uu = (double)u[o];
            double xk0 = 0, xk1 = 0, xk2 = 0, xkn = 0, xkr = 0, xkc = 0, vk = 1, mn = 1.0e308, l = 0;
#pragma unroll
            for (int i = 0; i < K; ++i) {
                double x0, x1, x2, wn, wr, wc, vi;
                if (i < K - 1) {
                    x0 = xi[(3 * i) * g.plane + o];
                    x1 = xi[(3 * i + 1) * g.plane + o];
                    x2 = xi[(3 * i + 2) * g.plane + o];
                    xk0 -= x0;
                    xk1 -= x1;
                    xk2 -= x2;
                    wn = pn ? (double)xi[(3 * i) * g.plane + o - 1] : 0.0;
                    wr = pr ? (double)xi[(3 * i + 1) * g.plane + o - g.nstride] : 0.0;
                    wc = pc ? (double)xi[(3 * i + 2) * g.plane + opc] : 0.0;
                    xkn -= wn;
                    xkr -= wr;
                    xkc -= wc;
                    vi = V[i * g.plane + o];
                    vk -= vi;
                } else {
                    x0 = xk0;
                    x1 = xk1;
                    x2 = xk2;
                    wn = xkn;
                    wr = xkr;
                    wc = xkc;
                    vi = vk;
                }
                double div = 0.0;
                if (pn) div -= wn;
                if (hn) div += x0;
                if (pr) div -= wr;
                if (hr) div += x1;
                if (pc) div -= wc;
                if (hc) div += x2;
                const double dl = uu - lb.c[i];
                const double e = lam * dl * dl - div;
                l += vi * e;
                mn = e < mn ? e : mn;
            }
            lag += l;
            dual += mn;
            }
        }
    }
    __shared__ double2 red[kWarps];
    for (int s = 16; s > 0; s >>= 1) {
        lag += __shfl_xor_sync(0xffffffffu, lag, s);
        dual += __shfl_xor_sync(0xffffffffu, dual, s);
    }
    if (lane == 0) red[warp] = make_double2(lag, dual);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = red[0];
        for (int w = 1; w < kWarps; ++w) t.x += red[w].x, t.y += red[w].y;
        partial[blockIdx.x] = t;
    }
}

// Adds the block partials in block order; writes (lagrangian, dual, gap).
__global__ void static_energy_finish(const double2 *__restrict__ partial, int count, double *out)
{
    double l = 0.0, d = 0.0;
    for (int i = 0; i < count; ++i) l += partial[i].x, d += partial[i].y;
    out[0] = l;
    out[1] = d;
    out[2] = l - d;
}

template <int K>
void launch_energy(const StaticGeom &g, const StaticAddresses &a, const float *u, const float *V, const float *xi,
                   double lam, const Labels &lb, cudaStream_t s)
{
    static_energy_kernel<K><<<kBlocks, kThreads, 0, s>>>(g, a.cols, u, V, xi, lam, lb, a.partial);
}

}  // namespace

// defined with the rest of the C ABI: sets what potts_last_error() returns,
// and runs the solver's host-side checks of a mapping
void potts_set_last_error(const std::string &msg);
int potts_check_mapping(const potts_mapping *map);

namespace {
int static_fail(int code, const std::string &msg)
{
    potts_set_last_error(msg);
    return code;
}
}  // namespace

extern "C" int potts_energies_static(const potts_mapping *map, const float *d_u, int K, const float *ci,
                                     float lambda, const float *d_V, const float *d_Xi, void *stream, double *h_out)
{
    if (!map || !map->start_row || !map->base || !d_u || !ci || !d_V || !d_Xi || !h_out)
        return static_fail(POTTS_EINVAL, "NULL argument");
    if (K < 2 || K > POTTS_MAX_PHASES) return static_fail(POTTS_EINVAL, "K must be in [2, 6]");
    if (map->cols > POTTS_STATIC_MAX_COLS)
        return static_fail(POTTS_EINVAL, "more columns than POTTS_STATIC_MAX_COLS (" +
                                             std::to_string(POTTS_STATIC_MAX_COLS) + ")");
    // the same checks as every solver entry point (non-decreasing base[] of
    // multiples of nstride, rows inside the row extent, ...): a bad table
    // would make the kernel read outside u, V and Xi
    if (const int st = potts_check_mapping(map); st != POTTS_OK) return st;
    Labels lb;
    for (int i = 0; i < K; ++i) {
        if (!std::isfinite(ci[i])) return static_fail(POTTS_EINVAL, "labels must be finite");
        lb.c[i] = (double)ci[i];
    }
    if (!std::isfinite(lambda)) return static_fail(POTTS_EINVAL, "lambda must be finite");
    StaticAddresses a;
    std::string err;
    if (device_addresses(&a, &err) != POTTS_OK) {
        cudaGetLastError();
        return static_fail(POTTS_ECUDA, err);
    }

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the column table, in chunks through a host array; a copy from pageable
    // memory has read its source when cudaMemcpyAsync returns
    int4 table[kTableChunk];
    for (uint32_t c0 = 0; c0 < map->cols; c0 += kTableChunk) {
        const uint32_t cnt = map->cols - c0 < kTableChunk ? map->cols - c0 : kTableChunk;
        for (uint32_t j = 0; j < cnt; ++j) {
            const uint32_t c = c0 + j;
            const uint32_t rows = (map->base[c + 1] - map->base[c]) / map->nstride;
            table[j] = make_int4((int)(map->base[c] / map->nstride), rows ? (int)map->start_row[c] : 0,
                                 rows ? (int)(map->start_row[c] + rows) : 0, 0);
        }
        cudaError_t e = cudaMemcpyAsync(a.cols + c0, table, sizeof(int4) * cnt, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return static_fail(POTTS_ECUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    }
    StaticGeom g;
    g.col_begin = (int)(map->col_begin > map->col_end ? map->col_end : map->col_begin);
    g.col_end = (int)map->col_end;
    g.n = (int)map->n_images;
    g.nstride = (int)map->nstride;
    g.plane = (int64_t)map->base[map->cols];
    switch (K) {
    case 2: launch_energy<2>(g, a, d_u, d_V, d_Xi, (double)lambda, lb, s); break;
    case 3: launch_energy<3>(g, a, d_u, d_V, d_Xi, (double)lambda, lb, s); break;
    case 4: launch_energy<4>(g, a, d_u, d_V, d_Xi, (double)lambda, lb, s); break;
    case 5: launch_energy<5>(g, a, d_u, d_V, d_Xi, (double)lambda, lb, s); break;
    case 6: launch_energy<6>(g, a, d_u, d_V, d_Xi, (double)lambda, lb, s); break;
    }
    static_energy_finish<<<1, 1, 0, s>>>(a.partial, kBlocks, a.out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_out, a.out, sizeof(double) * 3, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return static_fail(POTTS_ECUDA, cudaGetErrorString(e));
    return POTTS_OK;
}
