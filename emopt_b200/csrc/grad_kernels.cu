// grad_kernels.cu -- FDTD_grad_eps: the permittivity factor of the adjoint
// gradient, fused over a design box.
//
// For a real permittivity change d(eps_c) of Yee component c at one cell, the
// adjoint method gives dF = -2 Re(y_c * 1j * d(eps_c) * x_c) with x the forward
// and y the adjoint steady-state field (the product y^T dA x of
// emopt/fdtd.py:1694-1717, gradient -2 Re(y^T dA x) of
// emopt/adjoint_method.py:505-544).  Per unit d(eps_c) that is
//     g_c = -2 Re(1j y_c x_c) = 2 Im(y_c x_c).
// This kernel evaluates g_c for c = Ex, Ey, Ez over a box of the grid, reading
// the complex128 phasors where FDTD_solve_cw left them in device memory.  For
// planar (extruded) designs it sums g_c along z for each (j, k) column, with
// Kahan-compensated float64 accumulation, which is the reduction that the
// chain rule to a 2-D design density needs; the rest of the chain rule (the
// dependence of eps on the design parameters) is left to the caller.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>

#include "../../include/emopt_fdtd.h"

namespace {

struct GradBox {
    int k0, k1, j0, j1;
    int i0[3], i1[3];
    int imin, imax;
};

__device__ __forceinline__ double g_cell(const fdtd_complex128& a, const fdtd_complex128& b) {
    // 2 Im(a b) = 2 (a.re b.im + a.im b.re)
    return 2.0 * (a.real * b.imag + a.imag * b.real);
}

// Planar: one thread per (c, j, k) column, Kahan sum over i in [i0_c, i1_c).
__global__ void k_grad_planar(const fdtd_complex128* __restrict__ f0, const fdtd_complex128* __restrict__ f1,
                              const fdtd_complex128* __restrict__ f2, const fdtd_complex128* __restrict__ a0,
                              const fdtd_complex128* __restrict__ a1, const fdtd_complex128* __restrict__ a2,
                              int Nx, int Ny, GradBox b, double* __restrict__ out) {
    const int nk = b.k1 - b.k0, nj = b.j1 - b.j0;
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    const int jj = blockIdx.y * blockDim.y + threadIdx.y;
    const int c = blockIdx.z;
    if (kk >= nk || jj >= nj) return;
    const fdtd_complex128* f = c == 0 ? f0 : (c == 1 ? f1 : f2);
    const fdtd_complex128* a = c == 0 ? a0 : (c == 1 ? a1 : a2);
    const long long plane = (long long)Ny * Nx;
    const long long col = (long long)(b.j0 + jj) * Nx + (b.k0 + kk);
    double s = 0.0, comp = 0.0;
    for (int i = b.i0[c]; i < b.i1[c]; i++) {
        const long long q = (long long)i * plane + col;
        const double y = g_cell(a[q], f[q]) - comp;
        const double t = s + y;
        comp = (t - s) - y;
        s = t;
    }
    out[((long long)c * nj + jj) * nk + kk] = s;
}

// Per cell: out[c][i - imin][j][k], zero outside [i0_c, i1_c).
__global__ void k_grad_cells(const fdtd_complex128* __restrict__ f0, const fdtd_complex128* __restrict__ f1,
                             const fdtd_complex128* __restrict__ f2, const fdtd_complex128* __restrict__ a0,
                             const fdtd_complex128* __restrict__ a1, const fdtd_complex128* __restrict__ a2,
                             int Nx, int Ny, GradBox b, double* __restrict__ out) {
    const int nk = b.k1 - b.k0, nj = b.j1 - b.j0, ni = b.imax - b.imin;
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    const int jj = blockIdx.y * blockDim.y + threadIdx.y;
    const int c = blockIdx.z % 3, ii = blockIdx.z / 3;
    if (kk >= nk || jj >= nj || ii >= ni) return;
    const int i = b.imin + ii;
    double v = 0.0;
    if (i >= b.i0[c] && i < b.i1[c]) {
        const fdtd_complex128* f = c == 0 ? f0 : (c == 1 ? f1 : f2);
        const fdtd_complex128* a = c == 0 ? a0 : (c == 1 ? a1 : a2);
        const long long q = ((long long)i * Ny + (b.j0 + jj)) * Nx + (b.k0 + kk);
        v = g_cell(a[q], f[q]);
    }
    out[(((long long)c * ni + ii) * nj + jj) * nk + kk] = v;
}

int fail(char* msg, int msglen, int status, const char* fmt, ...) {
    if (msg && msglen > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(msg, (size_t)msglen, fmt, ap);
        va_end(ap);
    }
    return status;
}

}  // namespace

extern "C" int FDTD_grad_eps(int device, void* stream, const fdtd_complex128* const* fwd,
                             const fdtd_complex128* const* adj, int Nx, int Ny, int Nz,
                             const int* box, int planar, double* out, char* msg, int msglen) {
    if (msg && msglen > 0) msg[0] = '\0';
    if (!fwd || !adj || !box || !out) return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_grad_eps: null argument");
    if (Nx <= 0 || Ny <= 0 || Nz <= 0) return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_grad_eps: empty grid");
    GradBox b;
    b.k0 = box[0]; b.k1 = box[1]; b.j0 = box[2]; b.j1 = box[3];
    b.imin = Nz; b.imax = 0;
    for (int c = 0; c < 3; c++) {
        b.i0[c] = box[4 + 2 * c];
        b.i1[c] = box[5 + 2 * c];
        if (!fwd[c] || !adj[c]) return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_grad_eps: null field");
        if (b.i0[c] < 0 || b.i1[c] > Nz || b.i0[c] > b.i1[c])
            return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_grad_eps: z range %d of [%d, %d) outside [0, %d)",
                        c, b.i0[c], b.i1[c], Nz);
        if (b.i0[c] < b.imin) b.imin = b.i0[c];
        if (b.i1[c] > b.imax) b.imax = b.i1[c];
    }
    if (b.imax < b.imin) b.imax = b.imin;
    if (b.k0 < 0 || b.k1 > Nx || b.k0 >= b.k1 || b.j0 < 0 || b.j1 > Ny || b.j0 >= b.j1)
        return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_grad_eps: box x [%d, %d) y [%d, %d) outside the grid",
                    b.k0, b.k1, b.j0, b.j1);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(msg, msglen, FDTD_ERR_NODEVICE, "FDTD_grad_eps: no CUDA device");
    }
    if (device < 0 || device >= ndev)
        return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_grad_eps: device %d not in [0, %d)", device, ndev);
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != device) e = cudaSetDevice(device);
    cudaStream_t st = stream ? (cudaStream_t)stream : cudaStreamPerThread;
    if (e == cudaSuccess) {
        const int nk = b.k1 - b.k0, nj = b.j1 - b.j0, ni = b.imax - b.imin;
        dim3 blk(32, 8);
        if (planar) {
            dim3 grd((nk + 31) / 32, (nj + 7) / 8, 3);
            k_grad_planar<<<grd, blk, 0, st>>>(fwd[0], fwd[1], fwd[2], adj[0], adj[1], adj[2], Nx, Ny, b, out);
        } else if (ni > 0) {
            dim3 grd((nk + 31) / 32, (nj + 7) / 8, 3 * ni);
            k_grad_cells<<<grd, blk, 0, st>>>(fwd[0], fwd[1], fwd[2], adj[0], adj[1], adj[2], Nx, Ny, b, out);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess)
        return fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_grad_eps: %s", cudaGetErrorString(e));
    return FDTD_OK;
}
