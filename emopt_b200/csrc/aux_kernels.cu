// aux_kernels.cu -- set-up, extraction and convergence kernels of the
// device-resident CW solve.
#include "kernels.h"
#include "probe_body.cuh"

namespace fdtdb {

namespace {

unsigned blocks_for(long long n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

// E-update coefficients of one cell (src/fdtd.cpp:513-552) in fp64.
__device__ __forceinline__ void eps_ab(c128 e, double dt, bool lossy, double& a, double& b) {
    if (!lossy) {
        a = 1.0;
        b = dt / e.real;
    } else {
        double rdt = e.real * (1.0 / dt), ih = e.imag * 0.5;
        a = (rdt - ih) / (rdt + ih);
        b = 1.0 / (rdt + ih);
    }
}

template <typename T>
__global__ void k_material_coeffs(const c128* eps, const c128* mu, int Nx, int Ny, int Nz, int px,
                                  double dt, bool lossy, T* b_out, T* a_out, T* bH_out) {
    long long n = (long long)Nx * Ny * Nz;
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    int k = (int)(g % Nx);
    long long row = g / Nx;  // i*Ny + j
    long long p = row * px + k;
    if (eps) {
        double a, b;
        eps_ab(eps[g], dt, lossy, a, b);
        b_out[p] = T(b);
        if (a_out) a_out[p] = T(a);
    }
    if (mu) bH_out[p] = T(dt / mu[g].real);
}

__global__ void k_uniform_check(const c128* mu, long long n, int* flag) {
    double ref = mu[0].real;
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (long long)gridDim.x * blockDim.x)
        if (mu[g].real != ref) { *flag = 0; return; }
}

template <typename T>
__global__ void k_source_coeffs(const c128* ap, int i0, int j0, int k0, int I, int J, int K,
                                const T* coef_arr, double coef_scalar, int Ny, int px, T* out) {
    long long n = (long long)I * J * K;
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int lk = (int)(q % K), lj = (int)((q / K) % J), li = (int)(q / ((long long)K * J));
    long long p = ((long long)(li + i0) * Ny + (lj + j0)) * px + (lk + k0);
    double coef = coef_arr ? (double)coef_arr[p] : coef_scalar;
    c128 v = ap[q];
    // sin(t + phase) = sin t cos(phase) + cos t sin(phase)
    out[2 * q] = T(v.real * coef * cos(v.imag));
    out[2 * q + 1] = T(v.real * coef * sin(v.imag));
}

template <typename T>
__global__ void k_extract_3t(const T* t0, const T* t1, const T* cur, int Nx, long long n, int px,
                             Fit3 fit, c128* out) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    long long p = (g / Nx) * px + (g % Nx);
    out[g] = phasor_3t(fit, (double)t0[p], (double)t1[p], (double)cur[p]);
}

// Dense copy of one pitched snapshot into .real of complex128 values.
template <typename T>
__global__ void k_snapshot_real(const T* snap, int Nx, long long n, int px, c128* out) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    out[g].real = (double)snap[(g / Nx) * px + (g % Nx)];
}

// (re, im) -> (|z|, -atan2(im, re)), zero kept as (0, 0) (src/fdtd.cpp:1517-1576).
__global__ void k_amp_phase(c128* a, long long n) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    double re = a[q].real, im = a[q].imag;
    a[q].real = sqrt(re * re + im * im);
    a[q].imag = (im == 0 && re == 0) ? 0.0 : -1 * atan2(im, re);
}

// Per-step source constants: (S, C) = env(t)(sin t, cos t) at t = n dt for the
// H half-step and t = (n + 1/2) dt for the E half-step.
__global__ void k_step_table(double4* tab, long long nsteps, double dt, double T, double m,
                             double kk) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nsteps) return;
    double tH = (double)n * dt, tE = ((double)n + 0.5) * dt;
    double eH = src_envelope(tH, T, m, kk), eE = src_envelope(tE, T, m, kk);
    double sH, cH, sE, cE;
    sincos(tH, &sH, &cH);
    sincos(tE, &sE, &cE);
    tab[n] = make_double4(eH * sH, eH * cH, eE * sE, eE * cE);
}

__global__ void k_set_ll(long long* p, long long v) { *p = v; }

// One CTA.  Window shift and per-point refit follow emopt/fdtd.py:1072-1121;
// the change norms follow :1137-1138 (probe_body.cuh).
template <typename T>
__global__ void __launch_bounds__(256) k_probe(const T* Ex, const T* Ey, const T* Ez, ProbeDev pd,
                                               long long* step_base, int last_off,
                                               long long advance, double dt) {
    probe_block<T>(Ex, Ey, Ez, pd, *step_base + last_off, dt);
    if (threadIdx.x == 0) *step_base = *step_base + advance;
}

template <typename T>
__global__ void __launch_bounds__(256) k_slab_sample(const T* Ex, const T* Ey, const T* Ez,
                                                     const long long* map, int np, double* out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const long long off = map[q];
    out[q] = off >= 0 ? (double)Ex[off] : 0.0;
    out[np + q] = off >= 0 ? (double)Ey[off] : 0.0;
    out[2 * np + q] = off >= 0 ? (double)Ez[off] : 0.0;
}

}  // namespace

template <typename T>
void launch_slab_sample(const T* Ex, const T* Ey, const T* Ez, const long long* map, int np,
                        double* out, cudaStream_t st) {
    if (np > 0) k_slab_sample<T><<<(np + 255) / 256, 256, 0, st>>>(Ex, Ey, Ez, map, np, out);
}

template <typename T>
void launch_material_coeffs(const c128* eps, const c128* mu, int Nx, int Ny, int Nz, int px,
                            double dt, bool lossy, T* b_out, T* a_out, T* bH_out,
                            cudaStream_t st) {
    long long n = (long long)Nx * Ny * Nz;
    k_material_coeffs<T><<<blocks_for(n, 256), 256, 0, st>>>(eps, mu, Nx, Ny, Nz, px, dt, lossy,
                                                             b_out, a_out, bH_out);
}

void launch_uniform_check(const c128* mu, long long n, int* flag, cudaStream_t st) {
    k_uniform_check<<<296, 256, 0, st>>>(mu, n, flag);
}

template <typename T>
void launch_source_coeffs(const c128* ap, int i0, int j0, int k0, int I, int J, int K,
                          const T* coef_arr, double coef_scalar, int Ny, int px, T* out,
                          cudaStream_t st) {
    long long n = (long long)I * J * K;
    if (n > 0)
        k_source_coeffs<T><<<blocks_for(n, 256), 256, 0, st>>>(ap, i0, j0, k0, I, J, K, coef_arr,
                                                               coef_scalar, Ny, px, out);
}

template <typename T>
void launch_extract_3t(const T* t0, const T* t1, const T* cur, int Nx, int Ny, int Nz, int px,
                       Fit3 fit, c128* out, cudaStream_t st) {
    long long n = (long long)Nx * Ny * Nz;
    k_extract_3t<T><<<blocks_for(n, 256), 256, 0, st>>>(t0, t1, cur, Nx, n, px, fit, out);
}

template <typename T>
void launch_snapshot_real(const T* snap, int Nx, int Ny, int Nz, int px, c128* out,
                          cudaStream_t st) {
    long long n = (long long)Nx * Ny * Nz;
    k_snapshot_real<T><<<blocks_for(n, 256), 256, 0, st>>>(snap, Nx, n, px, out);
}

void launch_amp_phase(c128* a, long long n, cudaStream_t st) {
    if (n > 0) k_amp_phase<<<blocks_for(n, 256), 256, 0, st>>>(a, n);
}

void launch_step_table(double4* tab, long long nsteps, double dt, double T, double m, double kk,
                       cudaStream_t st) {
    if (nsteps > 0) k_step_table<<<blocks_for(nsteps, 256), 256, 0, st>>>(tab, nsteps, dt, T, m, kk);
}

void launch_set_ll(long long* p, long long v, cudaStream_t st) { k_set_ll<<<1, 1, 0, st>>>(p, v); }

template <typename T>
void launch_probe(const T* Ex, const T* Ey, const T* Ez, ProbeDev pd, long long* step_base,
                  int last_off, long long advance, double dt, cudaStream_t st) {
    k_probe<T><<<1, 256, 0, st>>>(Ex, Ey, Ez, pd, step_base, last_off, advance, dt);
}

#define INST(T)                                                                                 \
    template void launch_material_coeffs<T>(const c128*, const c128*, int, int, int, int,       \
                                            double, bool, T*, T*, T*, cudaStream_t);            \
    template void launch_source_coeffs<T>(const c128*, int, int, int, int, int, int, const T*,   \
                                          double, int, int, T*, cudaStream_t);                  \
    template void launch_extract_3t<T>(const T*, const T*, const T*, int, int, int, int, Fit3,  \
                                       c128*, cudaStream_t);                                    \
    template void launch_snapshot_real<T>(const T*, int, int, int, int, c128*, cudaStream_t);   \
    template void launch_probe<T>(const T*, const T*, const T*, ProbeDev, long long*, int,      \
                                  long long, double, cudaStream_t);                             \
    template void launch_slab_sample<T>(const T*, const T*, const T*, const long long*, int,     \
                                        double*, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace fdtdb
