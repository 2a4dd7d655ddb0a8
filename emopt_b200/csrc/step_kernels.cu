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
// with the fused kernel in fused_kernels.cu.
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
    long long p = (long long)i * g.plane + (long long)j * g.px + k;
    const T *Ex = f.c[0], *Ey = f.c[1], *Ez = f.c[2];
    bool px_ = g.bc[0] != '0' && g.bc[0] != 'E' && g.bc[0] != 'H';
    bool py_ = g.bc[1] != '0' && g.bc[1] != 'E' && g.bc[1] != 'H';
    bool pz_ = g.bc[2] != '0' && g.bc[2] != 'E' && g.bc[2] != 'H';
    HIn<T> e;
    e.ex = Ex[p]; e.ey = Ey[p]; e.ez = Ez[p];
    if (k + 1 < g.Nx) { e.ey_x = Ey[p + 1]; e.ez_x = Ez[p + 1]; }
    else if (px_) { e.ey_x = Ey[p - k]; e.ez_x = Ez[p - k]; }
    else { e.ey_x = T(0); e.ez_x = T(0); }
    if (j + 1 < g.Ny) { e.ex_y = Ex[p + g.px]; e.ez_y = Ez[p + g.px]; }
    else if (py_) { long long q = p - (long long)j * g.px; e.ex_y = Ex[q]; e.ez_y = Ez[q]; }
    else { e.ex_y = T(0); e.ez_y = T(0); }
    if (i + 1 < g.Nz) { e.ex_z = Ex[p + g.plane]; e.ey_z = Ey[p + g.plane]; }
    else if (pz_) { long long q = p - (long long)i * g.plane; e.ex_z = Ex[q]; e.ey_z = Ey[q]; }
    else { e.ex_z = T(0); e.ey_z = T(0); }
    T hx = f.c[3][p], hy = f.c[4][p], hz = f.c[5][p];
    h_cell<T>(g, i, j, k, p, e, hx, hy, hz, g.pml[0].psi, g.pml[0].psi, g.pml[1].psi,
              g.pml[1].psi, g.pml[2].psi, g.pml[2].psi, true);
    if (src.n) {
        double4 st = g.step_tab[*step_base + off];
        add_sources<T>(src, i, j, k, 3, T(st.x), T(st.y), hx, hy, hz, false);
    }
    f.c[3][p] = hx; f.c[4][p] = hy; f.c[5][p] = hz;
}

template <typename T>
__global__ void __launch_bounds__(256) k_update_E(GridView<T> g, Fields<T> f, SourceList<T> src,
                                                  const long long* step_base, int off) {
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 8 + threadIdx.y;
    int i = blockIdx.z;
    if (k >= g.Nx || j >= g.Ny) return;
    long long p = (long long)i * g.plane + (long long)j * g.px + k;
    const T *Hx = f.c[3], *Hy = f.c[4], *Hz = f.c[5];
    EIn<T> h;
    h.hx = Hx[p]; h.hy = Hy[p]; h.hz = Hz[p];
    if (k > 0) { h.hy_x = Hy[p - 1]; h.hz_x = Hz[p - 1]; }
    else {
        long long q = p + g.Nx - 1;
        h.hy_x = h_min_ghost<T>(g.bc[0], h.hy, Hy[q]);
        h.hz_x = h_min_ghost<T>(g.bc[0], h.hz, Hz[q]);
    }
    if (j > 0) { h.hx_y = Hx[p - g.px]; h.hz_y = Hz[p - g.px]; }
    else {
        long long q = p + (long long)(g.Ny - 1) * g.px;
        h.hx_y = h_min_ghost<T>(g.bc[1], h.hx, Hx[q]);
        h.hz_y = h_min_ghost<T>(g.bc[1], h.hz, Hz[q]);
    }
    if (i > 0) { h.hx_z = Hx[p - g.plane]; h.hy_z = Hy[p - g.plane]; }
    else {
        long long q = p + (long long)(g.Nz - 1) * g.plane;
        h.hx_z = h_min_ghost<T>(g.bc[2], h.hx, Hx[q]);
        h.hy_z = h_min_ghost<T>(g.bc[2], h.hy, Hy[q]);
    }
    T ex = f.c[0][p], ey = f.c[1][p], ez = f.c[2][p];
    T bx, by, bz;
    e_cell<T>(g, i, j, k, p, h, ex, ey, ez, g.pml[0].psi, g.pml[0].psi, g.pml[1].psi,
              g.pml[1].psi, g.pml[2].psi, g.pml[2].psi, bx, by, bz);
    if (src.n) {
        double4 st = g.step_tab[*step_base + off];
        add_sources<T>(src, i, j, k, 0, T(st.z), T(st.w), ex, ey, ez, true);
    }
    f.c[0][p] = ex; f.c[1][p] = ey; f.c[2][p] = ez;
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
