// vec_kernels.cu -- H and E half-steps, one vector of x cells per thread.
//
// Kernels around the per-warp bodies of vec_body.cuh for one solve: block =
// (32, VEC_BLOCK_ROWS) threads, one warp per row; grid = (vector blocks of a
// row, row blocks, planes).  Single-warp blocks (VEC_BLOCK_ROWS = 1) free
// their slot as soon as the warp finishes, which keeps more loads in flight
// than 8-warp blocks whose slot waits for the slowest warp (124 us against
// 137 us per step on the 321 x 161 x 101 MMI block in fp32).
#include "kernels.h"
#include "vec_body.cuh"

// Warps per block (blockDim.y), and rows of a plane per warp (vec_body.cuh).
#ifndef VEC_BLOCK_ROWS
#define VEC_BLOCK_ROWS 1
#endif
#ifndef VEC_WARP_ROWS32
#define VEC_WARP_ROWS32 1
#endif
// float64 keeps one row per warp: two rows do not fit its register budget
#define VEC_WARP_ROWS(T) (sizeof(T) == 4 ? VEC_WARP_ROWS32 : 1)

namespace fdtdb {

// First row of the warp.  With single-warp blocks it is derived from
// blockIdx.y alone, which the compiler knows to be the same for all lanes: the
// slab tests derived from it become uniform branches instead of predicated
// code.
template <typename T>
__device__ __forceinline__ int vec_row() {
    return VEC_WARP_ROWS(T) * (VEC_BLOCK_ROWS == 1 ? (int)blockIdx.y
                                                   : (int)(blockIdx.y * VEC_BLOCK_ROWS + threadIdx.y));
}

// Register bounds: float64 bodies are held to 18 resident single-warp CTAs
// per SM (94-96 registers instead of 120-122: 203 instead of 210 us per step
// on the 321 x 161 x 101 MMI block); float32 keeps its own allocation.
#ifndef VEC_MINB32
#define VEC_MINB32 0
#endif
#define VEC_MINB(T) (sizeof(T) == 8 ? 18 : VEC_MINB32)

// float32 warps whose cells lie in no CPML slab and no source box run a body
// compiled without that code (vecb::plain_warp; 120.2 instead of 121.1 us per
// step on the MMI block: the bodies wait on their loads more than they issue);
// float64 keeps one body (a second one gained nothing: 199-200 us either way).
template <typename T>
__global__ void __launch_bounds__(sizeof(T) == 8 || VEC_MINB32 ? 32 * VEC_BLOCK_ROWS : 256, VEC_MINB(T))
k_update_H_vec(GridView<T> g, Fields<T> f, SourceList<T> src, const long long* step_base, int off,
               int i0) {
    constexpr int NR = VEC_WARP_ROWS(T);
    const int i = i0 + (int)blockIdx.z, j0 = vec_row<T>();
    if (sizeof(T) == 4 && vecb::plain_warp<T, NR>(g, src, 3, i, j0, blockIdx.x))
        vec_update_H<T, NR, false>(g, f, src, step_base, off, i, j0, blockIdx.x, threadIdx.x);
    else
        vec_update_H<T, NR, true>(g, f, src, step_base, off, i, j0, blockIdx.x, threadIdx.x);
}

// The E kernel is bounded by its real block size: that keeps it at 64
// registers in float32 (80 under the 256-thread bound), ~4% faster per step.
template <typename T>
__global__ void __launch_bounds__(32 * VEC_BLOCK_ROWS, VEC_MINB(T))
k_update_E_vec(GridView<T> g, Fields<T> f, SourceList<T> src, const long long* step_base, int off,
               int i0) {
    constexpr int NR = VEC_WARP_ROWS(T);
    const int i = i0 + (int)blockIdx.z, j0 = vec_row<T>();
    if (sizeof(T) == 4 && vecb::plain_warp<T, NR>(g, src, 0, i, j0, blockIdx.x))
        vec_update_E<T, NR, false>(g, f, src, step_base, off, i, j0, blockIdx.x, threadIdx.x);
    else
        vec_update_E<T, NR, true>(g, f, src, step_base, off, i, j0, blockIdx.x, threadIdx.x);
}

template <typename T>
cudaError_t launch_step_vec(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                            const long long* step_base, int off, cudaStream_t st) {
    constexpr int V = vecb::V16<T>::N;
    Fields<T> f;
    for (int c = 0; c < 6; c++) f.c[c] = fields[c];
    const int nvec = (g.Nx + V - 1) / V;
    dim3 block(32, VEC_BLOCK_ROWS);
    const int rows = VEC_BLOCK_ROWS * VEC_WARP_ROWS(T);
    dim3 grid((nvec + 31) / 32, (g.Ny + rows - 1) / rows, g.Nz);
    k_update_H_vec<T><<<grid, block, 0, st>>>(g, f, src, step_base, off, 0);
    k_update_E_vec<T><<<grid, block, 0, st>>>(g, f, src, step_base, off, 0);
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
    dim3 block(32, VEC_BLOCK_ROWS);
    const int rows = VEC_BLOCK_ROWS * VEC_WARP_ROWS(T);
    dim3 grid((nvec + 31) / 32, (g.Ny + rows - 1) / rows, ni);
    if (half == 0) k_update_H_vec<T><<<grid, block, 0, st>>>(g, f, src, step_base, off, i0);
    else k_update_E_vec<T><<<grid, block, 0, st>>>(g, f, src, step_base, off, i0);
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

}  // namespace fdtdb
