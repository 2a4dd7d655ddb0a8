// kernels.h -- host-side launch wrappers for the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include "cell.cuh"

namespace fdtdb {

// ---------------------------------------------------------- device layout
template <typename T>
void launch_step_unfused(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                         const long long* step_base, int off, cudaStream_t st);

// In-place H and E half steps, one 16-byte vector of x cells per thread
// (vec_kernels.cu).  Requires non-periodic boundaries.
template <typename T>
cudaError_t launch_step_vec(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                            const long long* step_base, int off, cudaStream_t st);

// The same time step split into an interior launch (no CPML code, multi-warp
// CTAs) and a rim launch (the CPML slabs) per half step (vec_kernels.cu).
template <typename T>
cudaError_t launch_step_split(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                              const long long* step_base, int off, cudaStream_t st);

// Fraction of the warp tasks that the interior launch of the split pair takes.
template <typename T>
double split_interior_fraction(const GridView<T>& g);

// One half step (half 0: H, 1: E) of the vector pair over planes
// [i0, i0 + ni): the z slabs of a distributed solve exchange halo planes
// between the two, and update the planes next to a halo apart from the rest.
template <typename T>
cudaError_t launch_half_vec(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                            const long long* step_base, int off, int half, int i0, int ni,
                            cudaStream_t st);

// One fused time step (zmarch_kernels.cu): H and E of every cell, reading the
// fields and CPML state of (ga, fa) and writing those of (gb, fb); each
// single-warp CTA marches a 60-cell row segment through zc planes.  Requires
// non-periodic boundaries and a whole-grid view.
template <typename T>
cudaError_t launch_step_zmarch(const GridView<T>& ga, const GridView<T>& gb, T* const* fa,
                               T* const* fb, const SourceList<T>& src, const long long* step_base,
                               int off, int zc, cudaStream_t st);

// Planes per z chunk of the fused step: about 32 resident warps per SM on
// `sms` multiprocessors, at least 4 planes.
int zmarch_chunk(int Nx, int Ny, int Nz, int sms);

// eps or mu (complex128, dense [Nz][Ny][Nx]) -> pitched update coefficients.
// b = dt/eps.real, or for lossy media a = (er/dt - ei/2)/(er/dt + ei/2),
// b = 1/(er/dt + ei/2) (src/fdtd.cpp:513-552); bH = dt/mu.real.  Either
// material pointer may be null.
template <typename T>
void launch_material_coeffs(const c128* eps_or_null, const c128* mu_or_null, int Nx, int Ny,
                            int Nz, int px, double dt, bool lossy, T* b_out, T* a_out_or_null,
                            T* bH_out, cudaStream_t st);

// Returns (on the device) 1 in *flag when every mu[c].real equals mu[0].real.
void launch_uniform_check(const c128* mu, long long n, int* flag, cudaStream_t st);

// Source coefficients: comp_out[2m] = coef*A*cos(phase), [2m+1] = coef*A*sin(phase)
// for the source cells of one component; coef is the update coefficient of the
// cell (dt/mu for magnetic currents, the E-update b for electric ones), read
// from the pitched coefficient array or given as a scalar when that is null.
template <typename T>
void launch_source_coeffs(const c128* amp_phase, int i0, int j0, int k0, int I, int J, int K,
                          const T* coef_arr, double coef_scalar, int Ny, int px, T* comp_out,
                          cudaStream_t st);

// Steady-state extraction of one component from its t0/t1 snapshots and the
// live field into a dense complex128 array (src/fdtd.cpp:1346-1443).
template <typename T>
void launch_extract_3t(const T* t0, const T* t1, const T* cur, int Nx, int Ny, int Nz, int px,
                       Fit3 fit, c128* out, cudaStream_t st);

// .real of dense complex128 values := pitched snapshot values.
template <typename T>
void launch_snapshot_real(const T* snap, int Nx, int Ny, int Nz, int px, c128* out,
                          cudaStream_t st);

// In-place (re, im) -> (|z|, -atan2(im, re)) of source arrays (src/fdtd.cpp:1517-1576).
void launch_amp_phase(c128* a, long long n, cudaStream_t st);

// Per-step source constants for steps [0, nsteps).
void launch_step_table(double4* tab, long long nsteps, double dt, double T, double m, double kk,
                       cudaStream_t st);

void launch_set_ll(long long* p, long long v, cudaStream_t st);

// Convergence probe (emopt/fdtd.py:1072-1144): shifts the 3-sample window,
// refits the probe points and writes the amplitude / phase change norms.
struct ProbeDev {
    double* win;        // [3 comps][3 samples][nconv]
    double* A;          // [2][nconv]  (previous, current)
    double* phi;        // [2][nconv]
    double* times;      // [3]
    double* out;        // [0] A_change, [1] phi_change, [2] probe count
    const long long* map;  // per probe point: offset into the pitched E arrays, or -1
    const double* samples; // when set: this probe's E values, [3 comps][nconv], instead of map
    int nconv;
};

// ---------------------------------------------------------------- serving
// Control block of one served request (device memory): its step counter and
// the state of its loop (ServeState, grid.cuh).
struct ServeCtl {
    long long n;            // time steps taken
    long long Tn, last, n0, nprobes;
    double Nmax, amp_tol, phi_tol, dt, A_change, phi_change;
    ProbeDev pd;
    int state, capture, fixed;
    int stop_nf;            // 1: a probe that sees NaN/Inf ends the main loop
};

template <typename T>
struct ServeView {
    GridView<T> g;
    Fields<T> f;
    T* snap[2][6];
    SourceList<T> src;
    long long nxb;          // 32-vector blocks per row
};

// One time step of one served request: its H and E half steps (grid and
// fields in the kernel parameters, as the single-solve kernels) and its loop
// events (step counter, probes, captures, end).  Fixed launch shapes while
// the request is admitted (graph-capturable).
template <typename T>
cudaError_t launch_serve_request_step(const ServeView<T>& v, ServeCtl* ctl, cudaStream_t st);

template <typename T>
void launch_probe(const T* Ex, const T* Ey, const T* Ez, ProbeDev pd, long long* step_base,
                  int last_off, long long advance, double dt, cudaStream_t st);

// out[c * np + q] = E_c[map[q]] (0 where map[q] < 0): the probe values this
// z slab holds, summed over the slabs by the caller.
template <typename T>
void launch_slab_sample(const T* Ex, const T* Ey, const T* Ez, const long long* map, int np,
                        double* out, cudaStream_t st);

// ------------------------------------------------ padded (ABI) layout, fp64
struct LegacyView {
    int Nx, Ny, Nz, I, J, K, i0, j0, k0;
    double odx, ody, odz, dt, odt;
    bool lossy;
    char bc[3];
    int w[6];
    double* psi[3][2][4];
    const double* tab[3][6];   // kappa_H b_H c_H kappa_E b_E c_E (reference order)
    double* E[3];
    double* H[3];
    const c128* eps[3];
    const c128* mu[3];
};

struct LegacySource {
    const c128* comp[6];
    int i0, j0, k0, I, J, K;
};

void legacy_update_H(const LegacyView& v, const LegacySource* srcs, int nsrc, double t,
                     double src_T, double src_min, double src_k, cudaStream_t st);
void legacy_update_E(const LegacyView& v, const LegacySource* srcs, int nsrc, double t,
                     double src_T, double src_min, double src_k, cudaStream_t st);
void legacy_capture(const LegacyView& v, c128* const* dst, cudaStream_t st);
void legacy_extract_2t(const LegacyView& v, c128* const* t0, double t0v, double t1v,
                       cudaStream_t st);
void legacy_extract_3t(const LegacyView& v, c128* const* t0, const c128* const* t1, double t0v,
                       double t1v, double t2v, cudaStream_t st);

}  // namespace fdtdb
