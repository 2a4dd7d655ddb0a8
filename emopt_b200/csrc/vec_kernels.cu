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
    if (sizeof(T) == 4 && vecb::plain_warp<T, 1>(g, src, 3, i, j, blockIdx.x))
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
    if (sizeof(T) == 4 && vecb::plain_warp<T, 1>(g, src, 0, i, j, blockIdx.x))
        vec_update_E<T, false>(g, f, src, step_base, off, i, j, blockIdx.x, threadIdx.x);
    else
        vec_update_E<T, true>(g, f, src, step_base, off, i, j, blockIdx.x, threadIdx.x);
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

}  // namespace fdtdb
