// step_kernels.cu -- device-resident CW-FDTD half-steps (fp32 and fp64).
//
// These kernels implement the Yee leapfrog of src/fdtd.cpp:121-367 (H) and
// src/fdtd.cpp:369-755 (E) on the pitched, ghost-free layout of grid.cuh:
//   * forward-difference curl(E) / backward-difference curl(H) scaled by R/d,
//   * CPML corrections applied in x, y, z order (psi <- c d + b psi and the
//     field correction (psi - d) + d/kappa), the z-max slab starting one plane
//     later than x/y (strict comparison, src/fdtd.cpp:292 and 652),
//   * max-face tangential E = 0 (PEC) for the H update and the min-face H
//     symmetry rule ('0' zero, 'E' odd, 'H' even) for the E update; any other
//     boundary character behaves like the one-rank ghost exchange (periodic),
//   * current sources, with sin(t + phase) expanded as
//     S(t) cos(phase) + C(t) sin(phase) where S = env(t) sin t, C = env(t) cos t
//     come from a per-step fp64 table (k_step_table).
//
// k_update_H / k_update_E: one thread per cell, fields updated in place (two
// launches per time step).  The per-cell arithmetic (h_cell, e_cell) is shared
// with the fused kernel in fused_kernels.cu; the whole-cell updates are
// cell_update_H / cell_update_E (cell.cuh).
#include "cell.cuh"
#include "kernels.h"

namespace fdtdb {

// ============================================================ unfused pair
template <typename T>
__global__ void __launch_bounds__(256) k_update_H(GridView<T> g, Fields<T> f, SourceList<T> src,
                                                  const long long* step_base, int off) {
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 8 + threadIdx.y;
    int i = blockIdx.z;
    if (k >= g.Nx || j >= g.Ny) return;
    cell_update_H<T>(g, f, src, step_base, off, i, j, k);
}

template <typename T>
__global__ void __launch_bounds__(256) k_update_E(GridView<T> g, Fields<T> f, SourceList<T> src,
                                                  const long long* step_base, int off) {
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 8 + threadIdx.y;
    int i = blockIdx.z;
    if (k >= g.Nx || j >= g.Ny) return;
    cell_update_E<T>(g, f, src, step_base, off, i, j, k);
}

template <typename T>
void launch_step_unfused(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                         const long long* step_base, int off, cudaStream_t st) {
    Fields<T> f;
    for (int c = 0; c < 6; c++) f.c[c] = fields[c];
    dim3 block(32, 8);
    dim3 grid((g.Nx + 31) / 32, (g.Ny + 7) / 8, g.Nz);
    k_update_H<T><<<grid, block, 0, st>>>(g, f, src, step_base, off);
    k_update_E<T><<<grid, block, 0, st>>>(g, f, src, step_base, off);
}

template void launch_step_unfused<float>(const GridView<float>&, float* const*,
                                         const SourceList<float>&, const long long*, int,
                                         cudaStream_t);
template void launch_step_unfused<double>(const GridView<double>&, double* const*,
                                          const SourceList<double>&, const long long*, int,
                                          cudaStream_t);

}  // namespace fdtdb
