// vec_kernels.cu -- H and E half-steps, one vector of x cells per thread.
//
// Kernels around the per-warp bodies of vec_body.cuh for one solve: one
// single-warp CTA per warp task (grid = vector blocks of a row, rows,
// planes).  A finished warp frees its slot at once, which keeps more loads in
// flight than 8-warp CTAs whose slot waits for the slowest warp (124 us
// against 137 us per step on the 321 x 161 x 101 MMI block in fp32).  A
// persistent form in which each warp issued the loads of its next task
// before finishing the current one (two task register sets, 125-128
// registers, 16 warps per SM) took 167 us per step in fp32 (216 and 233 at 12
// and 20 CTAs per SM) and 445 us in fp64: fewer resident warps cost more
// than the overlap gained.
#include <algorithm>

#include "kernels.h"
#include "vec_body.cuh"

namespace fdtdb {

// Register bounds: float64 bodies are held to 18 resident single-warp CTAs
// per SM (94-96 registers instead of 120-122: 203 instead of 210 us per step
// on the 321 x 161 x 101 MMI block); float32 keeps its own allocation.
#define VEC_MINB(T) (sizeof(T) == 8 ? 18 : 0)

// float32 warps whose cells lie in no CPML slab and no source box run a body
// compiled without that code (vecb::plain_warp; 120.2 instead of 121.1 us per
// step on the MMI block: the bodies wait on their loads more than they issue);
// float64 keeps one body (a second one gained nothing: 199-200 us either way).
// The H kernel is bounded for 256-thread blocks (64 registers in float32).
template <typename T>
__global__ void __launch_bounds__(sizeof(T) == 8 ? 32 : 256, VEC_MINB(T))
k_update_H_vec(GridView<T> g, Fields<T> f, SourceList<T> src, const long long* step_base, int off,
               int i0) {
    const int i = i0 + (int)blockIdx.z, j = (int)blockIdx.y;
    if (sizeof(T) == 4 && vecb::plain_warp<T>(g, src, 3, i, j, blockIdx.x))
        vec_update_H<T, false>(g, f, src, step_base, off, i, j, blockIdx.x, threadIdx.x);
    else
        vec_update_H<T, true>(g, f, src, step_base, off, i, j, blockIdx.x, threadIdx.x);
}

// The E kernel is bounded by its real block size: that keeps it at 64
// registers in float32 (80 under the 256-thread bound), ~4% faster per step.
template <typename T>
__global__ void __launch_bounds__(32, VEC_MINB(T))
k_update_E_vec(GridView<T> g, Fields<T> f, SourceList<T> src, const long long* step_base, int off,
               int i0) {
    const int i = i0 + (int)blockIdx.z, j = (int)blockIdx.y;
    if (sizeof(T) == 4 && vecb::plain_warp<T>(g, src, 0, i, j, blockIdx.x))
        vec_update_E<T, false>(g, f, src, step_base, off, i, j, blockIdx.x, threadIdx.x);
    else
        vec_update_E<T, true>(g, f, src, step_base, off, i, j, blockIdx.x, threadIdx.x);
}

// ------------------------------------------------------------- interior/rim
// The same half steps split by task: the interior box (warp tasks that lie in
// no CPML slab) runs a body without CPML code, which needs 40-48 registers
// instead of 64, in multi-warp CTAs (more resident warps per SM); the rim
// (the tasks of the CPML slabs: whole z-slab planes, then the y-slab rows of
// the other planes, then the x-slab blocks of the other rows) runs the full
// body in single-warp CTAs.  Every task belongs to exactly one launch and is
// computed as by the single kernels, so the fields are the same.
struct SplitBox {
    int zi0, zi1, yj0, yj1, xb0, xb1;   // interior box: planes, rows, 64-cell blocks (half open)
    int nxb, Ny, Nz;
    long long nz_tasks, ny_tasks;        // rim tasks in the z slabs, in the y slabs
};

template <typename T>
bool split_box(const GridView<T>& g, SplitBox& b) {
    constexpr int W = 32 * vecb::V16<T>::N;   // cells per warp task
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    b.nxb = ((g.Nx + vecb::V16<T>::N - 1) / vecb::V16<T>::N + 31) / 32;
    b.Ny = g.Ny;
    b.Nz = g.Nz;
    // plane i is in no z slab when w0 <= i + off <= edge_max (slab_local, strict max)
    b.zi0 = std::max(0, PZ.w0 - PZ.off);
    b.zi1 = std::min(g.Nz, PZ.edge_max - PZ.off + 1);
    // row j is in no y slab when w0 <= j < edge_max
    b.yj0 = PY.w0;
    b.yj1 = std::min(g.Ny, PY.edge_max);
    // block xb (cells W xb .. W xb + W - 1) is in no x slab when they lie in [w0, edge_max)
    b.xb0 = (PX.w0 + W - 1) / W;
    b.xb1 = std::min(PX.edge_max, g.Nx) / W;
    if (b.zi1 <= b.zi0 || b.yj1 <= b.yj0 || b.xb1 <= b.xb0) return false;
    b.nz_tasks = (long long)(g.Nz - (b.zi1 - b.zi0)) * g.Ny * b.nxb;
    b.ny_tasks = (long long)(b.zi1 - b.zi0) * (g.Ny - (b.yj1 - b.yj0)) * b.nxb;
    return true;
}

#ifndef VEC_INT_WARPS
#define VEC_INT_WARPS 2
#endif
#ifndef VEC_INT_MINB32
#define VEC_INT_MINB32 18
#endif
#define VEC_INT_MINB(T) (sizeof(T) == 8 ? 10 : VEC_INT_MINB32)

template <typename T>
__global__ void __launch_bounds__(32 * VEC_INT_WARPS, VEC_INT_MINB(T))
k_update_H_int(GridView<T> g, Fields<T> f, SourceList<T> src, const long long* step_base, int off,
               SplitBox b) {
    const int j = b.yj0 + (int)(blockIdx.y * VEC_INT_WARPS + threadIdx.y);
    if (j >= b.yj1) return;   // the whole warp
    vec_update_H<T, false, false, true>(g, f, src, step_base, off, b.zi0 + (int)blockIdx.z, j,
                                        b.xb0 + (int)blockIdx.x, threadIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(32 * VEC_INT_WARPS, VEC_INT_MINB(T))
k_update_E_int(GridView<T> g, Fields<T> f, SourceList<T> src, const long long* step_base, int off,
               SplitBox b) {
    const int j = b.yj0 + (int)(blockIdx.y * VEC_INT_WARPS + threadIdx.y);
    if (j >= b.yj1) return;
    vec_update_E<T, false, false, true>(g, f, src, step_base, off, b.zi0 + (int)blockIdx.z, j,
                                        b.xb0 + (int)blockIdx.x, threadIdx.x);
}

// Rim task t -> (plane, row, block), in 32-bit arithmetic: the split pair
// runs only on grids of fewer than 2^31 cells, so task counts fit.
__device__ __forceinline__ void rim_task(const SplitBox& b, int t, int& i, int& j, int& xb) {
    const int nz = (int)b.nz_tasks, ny = (int)b.ny_tasks;
    if (t < nz) {
        const int per = b.Ny * b.nxb;
        const int p = t / per;
        const int r = t - p * per;
        i = p < b.zi0 ? p : b.zi1 + (p - b.zi0);
        j = r / b.nxb;
        xb = r - j * b.nxb;
        return;
    }
    t -= nz;
    if (t < ny) {
        const int rows = b.Ny - (b.yj1 - b.yj0);
        const int per = rows * b.nxb;
        const int p = t / per;
        const int r = t - p * per;
        const int q = r / b.nxb;
        i = b.zi0 + p;
        j = q < b.yj0 ? q : b.yj1 + (q - b.yj0);
        xb = r - q * b.nxb;
        return;
    }
    t -= ny;
    const int blocks = b.nxb - (b.xb1 - b.xb0);
    const int per = (b.yj1 - b.yj0) * blocks;
    const int p = t / per;
    const int r = t - p * per;
    const int q = r / blocks;
    const int c = r - q * blocks;
    i = b.zi0 + p;
    j = b.yj0 + q;
    xb = c < b.xb0 ? c : b.xb1 + (c - b.xb0);
}

template <typename T>
__global__ void __launch_bounds__(sizeof(T) == 8 ? 32 : 256, VEC_MINB(T))
k_update_H_rim(GridView<T> g, Fields<T> f, SourceList<T> src, const long long* step_base, int off,
               SplitBox b) {
    int i, j, xb;
    rim_task(b, (int)blockIdx.x, i, j, xb);
    vec_update_H<T, true>(g, f, src, step_base, off, i, j, xb, threadIdx.x);
}

// bounded to 32 resident CTAs in float32 (64 registers; the task decode
// would take it to 72)
template <typename T>
__global__ void __launch_bounds__(32, sizeof(T) == 8 ? 18 : 32)
k_update_E_rim(GridView<T> g, Fields<T> f, SourceList<T> src, const long long* step_base, int off,
               SplitBox b) {
    int i, j, xb;
    rim_task(b, (int)blockIdx.x, i, j, xb);
    vec_update_E<T, true>(g, f, src, step_base, off, i, j, xb, threadIdx.x);
}

template <typename T>
double split_interior_fraction(const GridView<T>& g) {
    SplitBox b;
    if (!split_box(g, b)) return 0.0;
    return (double)(b.zi1 - b.zi0) * (b.yj1 - b.yj0) * (b.xb1 - b.xb0) / ((double)b.Nz * b.Ny * b.nxb);
}

template <typename T>
cudaError_t launch_step_split(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                              const long long* step_base, int off, cudaStream_t st) {
    SplitBox b;
    if (!split_box(g, b)) return launch_step_vec<T>(g, fields, src, step_base, off, st);
    Fields<T> f;
    for (int c = 0; c < 6; c++) f.c[c] = fields[c];
    const long long rim = (long long)b.Nz * b.Ny * b.nxb -
                          (long long)(b.zi1 - b.zi0) * (b.yj1 - b.yj0) * (b.xb1 - b.xb0);
    dim3 iblock(32, VEC_INT_WARPS);
    dim3 igrid(b.xb1 - b.xb0, (b.yj1 - b.yj0 + VEC_INT_WARPS - 1) / VEC_INT_WARPS, b.zi1 - b.zi0);
    k_update_H_int<T><<<igrid, iblock, 0, st>>>(g, f, src, step_base, off, b);
    if (rim > 0) k_update_H_rim<T><<<(unsigned)rim, 32, 0, st>>>(g, f, src, step_base, off, b);
    k_update_E_int<T><<<igrid, iblock, 0, st>>>(g, f, src, step_base, off, b);
    if (rim > 0) k_update_E_rim<T><<<(unsigned)rim, 32, 0, st>>>(g, f, src, step_base, off, b);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ grid
template <typename T>
cudaError_t launch_step_vec(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                            const long long* step_base, int off, cudaStream_t st) {
    constexpr int V = vecb::V16<T>::N;
    Fields<T> f;
    for (int c = 0; c < 6; c++) f.c[c] = fields[c];
    const int nvec = (g.Nx + V - 1) / V;
    dim3 grid((nvec + 31) / 32, g.Ny, g.Nz);
    k_update_H_vec<T><<<grid, 32, 0, st>>>(g, f, src, step_base, off, 0);
    k_update_E_vec<T><<<grid, 32, 0, st>>>(g, f, src, step_base, off, 0);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_half_vec(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                            const long long* step_base, int off, int half, int i0, int ni,
                            cudaStream_t st) {
    constexpr int V = vecb::V16<T>::N;
    if (ni <= 0) return cudaSuccess;
    Fields<T> f;
    for (int c = 0; c < 6; c++) f.c[c] = fields[c];
    const int nvec = (g.Nx + V - 1) / V;
    dim3 grid((nvec + 31) / 32, g.Ny, ni);
    if (half == 0) k_update_H_vec<T><<<grid, 32, 0, st>>>(g, f, src, step_base, off, i0);
    else k_update_E_vec<T><<<grid, 32, 0, st>>>(g, f, src, step_base, off, i0);
    return cudaGetLastError();
}

template cudaError_t launch_half_vec<float>(const GridView<float>&, float* const*,
                                            const SourceList<float>&, const long long*, int, int,
                                            int, int, cudaStream_t);
template cudaError_t launch_half_vec<double>(const GridView<double>&, double* const*,
                                             const SourceList<double>&, const long long*, int, int,
                                             int, int, cudaStream_t);
template cudaError_t launch_step_vec<float>(const GridView<float>&, float* const*,
                                            const SourceList<float>&, const long long*, int,
                                            cudaStream_t);
template cudaError_t launch_step_vec<double>(const GridView<double>&, double* const*,
                                             const SourceList<double>&, const long long*, int,
                                             cudaStream_t);
template double split_interior_fraction<float>(const GridView<float>&);
template double split_interior_fraction<double>(const GridView<double>&);
template cudaError_t launch_step_split<float>(const GridView<float>&, float* const*,
                                              const SourceList<float>&, const long long*, int,
                                              cudaStream_t);
template cudaError_t launch_step_split<double>(const GridView<double>&, double* const*,
                                               const SourceList<double>&, const long long*, int,
                                               cudaStream_t);

}  // namespace fdtdb
