/*
 * emopt_fdtd.h -- C ABI of the B200 CW-FDTD library (emopt_b200/FDTD.so).
 *
 * The first block is the reference library's ABI, symbol for symbol: the same
 * names, argument order, argument meaning and (void) error behaviour as
 * src/fdtd.hpp:571-643 (definitions src/fdtd.cpp:1618-1929), so that the
 * reference binding emopt/fdtd_ctypes.py:26-149 loads this library unchanged.
 * Caller arrays are retained by pointer exactly as in the reference; each
 * per-call entry point reads them, computes on the GPU and writes the results
 * back before returning.
 *
 * The second block adds what the reference does not have: an explicit
 * destructor, error reporting, a precision switch and FDTD_solve_cw, which runs
 * the whole time loop of emopt/fdtd.py:994-1194 on the device and only moves
 * the materials in and the complex steady-state fields out.
 *
 * Layouts (reference conventions): padded local field arrays
 * (I+2)(J+2)(K+2) doubles, x fastest; material, snapshot and source arrays
 * unpadded I*J*K complex128 values {real, imag}.
 */
#ifndef EMOPT_FDTD_H
#define EMOPT_FDTD_H

#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct FDTDHandle FDTDHandle;
typedef struct { double real, imag; } fdtd_complex128;   /* src/fdtd.hpp:22-80 */

/* ----------------------------------------------- reference ABI (32 symbols) */
FDTDHandle *FDTD_new(void);                                          /* src/fdtd.hpp:572, src/fdtd.cpp:1618 */
void FDTD_set_wavelength(FDTDHandle *h, double wavelength);          /* src/fdtd.hpp:575, src/fdtd.cpp:1623 */
void FDTD_set_physical_dims(FDTDHandle *h, double X, double Y, double Z,
                            double dx, double dy, double dz);        /* src/fdtd.hpp:576, src/fdtd.cpp:1628 */
void FDTD_set_grid_dims(FDTDHandle *h, int Nx, int Ny, int Nz);     /* src/fdtd.hpp:579, src/fdtd.cpp:1635 */
void FDTD_set_local_grid(FDTDHandle *h, int k0, int j0, int i0,
                         int K, int J, int I);                      /* src/fdtd.hpp:580, src/fdtd.cpp:1640 */
void FDTD_set_dt(FDTDHandle *h, double dt);                         /* src/fdtd.hpp:583, src/fdtd.cpp:1648 */
void FDTD_set_complex_eps(FDTDHandle *h, bool complex_eps);         /* src/fdtd.hpp:584, src/fdtd.cpp:1653 */
void FDTD_set_field_arrays(FDTDHandle *h, double *Ex, double *Ey, double *Ez,
                           double *Hx, double *Hy, double *Hz);     /* src/fdtd.hpp:585, src/fdtd.cpp:1658 */
void FDTD_set_mat_arrays(FDTDHandle *h,
                         fdtd_complex128 *eps_x, fdtd_complex128 *eps_y, fdtd_complex128 *eps_z,
                         fdtd_complex128 *mu_x, fdtd_complex128 *mu_y, fdtd_complex128 *mu_z);
                                                                     /* src/fdtd.hpp:589, src/fdtd.cpp:1665 */
void FDTD_update_H(FDTDHandle *h, int n, double t);                 /* src/fdtd.hpp:593, src/fdtd.cpp:1672 */
void FDTD_update_E(FDTDHandle *h, int n, double t);                 /* src/fdtd.hpp:594, src/fdtd.cpp:1677 */
void FDTD_set_pml_widths(FDTDHandle *h, int xmin, int xmax, int ymin, int ymax,
                         int zmin, int zmax);                        /* src/fdtd.hpp:597, src/fdtd.cpp:1682 */
void FDTD_set_pml_properties(FDTDHandle *h, double sigma, double alpha,
                             double kappa, double pow);              /* src/fdtd.hpp:600, src/fdtd.cpp:1689 */
void FDTD_build_pml(FDTDHandle *h);                                  /* src/fdtd.hpp:602, src/fdtd.cpp:1695 */
void FDTD_reset_pml(FDTDHandle *h);                                  /* src/fdtd.hpp:603, src/fdtd.cpp:1700 */
void FDTD_set_t0_arrays(FDTDHandle *h,
                        fdtd_complex128 *Ex_t0, fdtd_complex128 *Ey_t0, fdtd_complex128 *Ez_t0,
                        fdtd_complex128 *Hx_t0, fdtd_complex128 *Hy_t0, fdtd_complex128 *Hz_t0);
                                                                     /* src/fdtd.hpp:606, src/fdtd.cpp:1705 */
void FDTD_set_t1_arrays(FDTDHandle *h,
                        fdtd_complex128 *Ex_t1, fdtd_complex128 *Ey_t1, fdtd_complex128 *Ez_t1,
                        fdtd_complex128 *Hx_t1, fdtd_complex128 *Hy_t1, fdtd_complex128 *Hz_t1);
                                                                     /* src/fdtd.hpp:609, src/fdtd.cpp:1712 */
double FDTD_calc_phase_2T(double t0, double t1, double f0, double f1);             /* src/fdtd.hpp:613, src/fdtd.cpp:1719 */
double FDTD_calc_amplitude_2T(double t0, double t1, double f0, double f1,
                              double phase);                                       /* src/fdtd.hpp:614, src/fdtd.cpp:1724 */
double FDTD_calc_phase_3T(double t0, double t1, double t2, double f0, double f1,
                          double f2);                                              /* src/fdtd.hpp:616, src/fdtd.cpp:1729 */
double FDTD_calc_amplitude_3T(double t0, double t1, double t2, double f0, double f1,
                              double f2, double phase);                            /* src/fdtd.hpp:617, src/fdtd.cpp:1734 */
void FDTD_capture_t0_fields(FDTDHandle *h);                          /* src/fdtd.hpp:619, src/fdtd.cpp:1739 */
void FDTD_capture_t1_fields(FDTDHandle *h);                          /* src/fdtd.hpp:620, src/fdtd.cpp:1744 */
void FDTD_calc_complex_fields_2T(FDTDHandle *h, double t0, double t1);             /* src/fdtd.hpp:621, src/fdtd.cpp:1750 */
void FDTD_calc_complex_fields_3T(FDTDHandle *h, double t0, double t1, double t2);  /* src/fdtd.hpp:622, src/fdtd.cpp:1755 */
void FDTD_add_source(FDTDHandle *h,
                     fdtd_complex128 *Jx, fdtd_complex128 *Jy, fdtd_complex128 *Jz,
                     fdtd_complex128 *Mx, fdtd_complex128 *My, fdtd_complex128 *Mz,
                     int i0, int j0, int k0, int I, int J, int K,
                     bool calc_phase);                               /* src/fdtd.hpp:625, src/fdtd.cpp:1760 */
void FDTD_clear_sources(FDTDHandle *h);                              /* src/fdtd.hpp:630, src/fdtd.cpp:1768 */
void FDTD_set_source_properties(FDTDHandle *h, double src_T, double src_min);
                                                                     /* src/fdtd.hpp:632, src/fdtd.cpp:1773 */
double FDTD_src_func_t(FDTDHandle *h, int n, double t, double phase);/* src/fdtd.hpp:634, src/fdtd.cpp:1778 */
void FDTD_set_bc(FDTDHandle *h, char *newbc);                        /* src/fdtd.hpp:637, src/fdtd.cpp:1783 */
void FDTD_copy_to_ghost_comm(double *src, fdtd_complex128 *ghost, int I, int J, int K);
                                                                     /* src/fdtd.hpp:640, src/fdtd.cpp:1789 */
void FDTD_copy_from_ghost_comm(double *dest, fdtd_complex128 *ghost, int I, int J, int K);
                                                                     /* src/fdtd.hpp:641, src/fdtd.cpp:1860 */

/* ---------------------------------------------------------------- additions */

/* Status codes returned by the additions and kept by FDTD_last_error. */
enum {
    FDTD_OK = 0,
    FDTD_ERR_CUDA = 1,        /* a CUDA call failed (message in FDTD_last_error) */
    FDTD_ERR_ARG = 2,         /* invalid argument or configuration */
    FDTD_ERR_NODEVICE = 3,    /* no CUDA device visible */
    FDTD_NMAX = 4,            /* FDTD_solve_cw: step budget Nmax exhausted before convergence */
    FDTD_NONFINITE = 5        /* FDTD_solve_cw: the probe saw NaN/Inf when the budget ran out */
};

/* Releases the handle and its device memory.  The reference has no
 * destructor (src/fdtd.cpp:1618-1621 allocates with no matching delete). */
void FDTD_delete(FDTDHandle *h);

/* Last status of the handle; copies its message into buf (NUL-terminated). */
int FDTD_last_error(FDTDHandle *h, char *buf, int buflen);

/* Selects the CUDA device of the handle (default: the calling thread's current
 * device).  Must precede the first call that touches the device. */
int FDTD_set_device(FDTDHandle *h, int device);

/* Planes per z chunk of the fused time step (kernel 3; 0 = chosen for about
 * 32 resident warps per SM, the default).  A tuning knob; results do not
 * depend on it. */
int FDTD_set_zchunk(FDTDHandle *h, int planes);

/* Storage/arithmetic precision of FDTD_solve_cw: 64 (default, the reference's
 * float64) or 32 (fields, coefficients and CPML state in float32; the
 * steady-state fit, probes and outputs stay float64).  Returns a status. */
int FDTD_set_precision(FDTDHandle *h, int bits);

/* Time-stepping kernel of FDTD_solve_cw: 0 = automatic (default: 6 in
 * float32 when at least 60% of the 64-cell warp tasks lie in no CPML slab,
 * else 5), 1 = H and E kernels with one cell per thread, 3 = one fused H+E
 * kernel per time step whose warps march up z chunks (reads one field/CPML
 * set, writes the other), 5 = H and E kernels with one 2-element vector of x
 * cells per thread, 6 = the kernels of 5 split per half step into an
 * interior launch (tasks in no CPML slab) and a rim launch.  Other values
 * fail with FDTD_ERR_ARG.  Periodic boundaries always use 1. */
int FDTD_set_kernel(FDTDHandle *h, int which);

/* Page-locks (cudaHostRegister, portable) / releases host memory that is
 * copied to or from the GPU on every solve -- material and t0 arrays -- so
 * those copies run at full DMA speed.  No counterpart in the reference.
 * Returns FDTD_OK, FDTD_ERR_ARG, FDTD_ERR_NODEVICE or FDTD_ERR_CUDA and leaves
 * no pending CUDA error behind. */
int FDTD_host_register(void *ptr, long long bytes);
int FDTD_host_unregister(void *ptr);

typedef struct {
    long long Tn;              /* probe period and extraction spacing: int64(Ncycle*3/4) (emopt/fdtd.py:1021) */
    double Nmax;               /* step budget: the loop stops once n > Nmax (emopt/fdtd.py:1054) */
    double rtol;               /* amplitude tolerance; the phase tolerance is sqrt(rtol) (emopt/fdtd.py:1046-1047) */
    const long long *conv_pts; /* probe indices into the padded local E arrays (emopt/fdtd.py:411-413) */
    int nconv;
    long long fixed_steps;     /* > 0: run exactly this many main steps without a convergence test */
    int materials_unchanged;   /* 1: reuse the coefficients of the previous solve on this handle */
    int copy_t1;               /* 1: also write the t1 snapshot into .real of the t1 arrays */
    int stop_nonfinite;        /* 1: end the main loop at the first probe that sees NaN/Inf
                                  (status FDTD_NONFINITE); 0: run on to Nmax as the reference */
} FDTDSolveOptions;

typedef struct {
    long long n_main;          /* steps of the main loop (index of the t0 capture) */
    long long steps;           /* total time steps = n_main + 2*Tn */
    double A_change;           /* last amplitude change norm */
    double phi_change;         /* last phase change norm */
    long long nprobes;         /* number of convergence probes */
    double device_ms;          /* device time of all time steps (CUDA events) */
    double total_ms;           /* device time of the whole call incl. transfers */
    long long launches;        /* kernels this call launched */
    int zchunk;                /* planes per z chunk of the fused step (kernel 3; else 0) */
    int status;                /* FDTD_OK, FDTD_NMAX or FDTD_NONFINITE */
} FDTDSolveResult;

/* The material and t0/t1 arrays that FDTD_solve_cw reads and writes may live
 * in host memory or in device memory of the handle's device (every copy lets
 * the CUDA runtime infer the direction); source arrays are host memory.
 *
 * Device-resident CW solve: equivalent to FDTD_reset_pml, zeroing the fields
 * and the loop of emopt/fdtd.py:1016-1194 (probe window, norm test, capture of
 * t0 and t1 Tn steps apart, 3-sample extraction), run on the GPU.  Reads the
 * material arrays and the sources registered with FDTD_add_source; writes the
 * complex steady-state fields into the t0 arrays.  Returns a status. */
int FDTD_solve_cw(FDTDHandle *h, const FDTDSolveOptions *opt, FDTDSolveResult *res);

/* Permittivity factor of the adjoint gradient, fused over a design box.  No
 * counterpart in the reference as one call: it evaluates, per cell and E
 * component c, g_c = -2 Re(1j * adj_c * fwd_c) = 2 Im(adj_c * fwd_c), the
 * derivative of the objective per unit real change of eps_c in the adjoint
 * product of emopt/fdtd.py:1694-1717 (gradient -2 Re(y^T dA x),
 * emopt/adjoint_method.py:505-544).
 *   fwd, adj: three pointers each (Ex, Ey, Ez) to complex128 [Nz][Ny][Nx]
 *             arrays in device memory of `device`, e.g. t0 arrays that
 *             FDTD_solve_cw wrote;
 *   box:      10 ints: k0, k1, j0, j1 (x and y ranges, half open) and the z
 *             range [i0_c, i1_c) of each component c = 0, 1, 2;
 *   planar:   1: out[c][j-j0][k-k0] = sum over i in [i0_c, i1_c) of g_c
 *             (Kahan-compensated float64); 0: out[c][i-imin][j-j0][k-k0] with
 *             imin / imax the smallest / largest z bound, zero outside a
 *             component's range;
 *   out:      float64 device memory of `device`;
 *   stream:   a cudaStream_t of `device` or NULL (the calling thread's default
 *             stream); the call returns after the kernel has finished.
 * Returns FDTD_OK, FDTD_ERR_ARG or FDTD_ERR_CUDA, with a message in msg. */
int FDTD_grad_eps(int device, void *stream, const fdtd_complex128 *const *fwd,
                  const fdtd_complex128 *const *adj, int Nx, int Ny, int Nz, const int *box,
                  int planar, double *out, char *msg, int msglen);

/* ------------------------------------------------------------------ serving
 * Continuous batching of independent CW solves on one GPU.  No counterpart in
 * the reference (one solve per process there).  A request is a handle
 * configured through the calls above (grid, materials, CPML, sources,
 * FDTD_set_precision(h, 32)) plus its FDTDSolveOptions.  Admitted requests
 * keep their fields resident and advance together: every FDTD_serve_advance
 * replays one CUDA graph of steps_per_replay time steps in which batched
 * kernels step all active requests at once and run each request's probe /
 * convergence / capture schedule on the device; requests whose loop ended
 * stop stepping and wait for FDTD_serve_collect, which extracts their fields
 * into the handle's t0 arrays and frees their memory.  Step counts and fields
 * equal those of FDTD_solve_cw (vector kernel) for the same request. */
typedef struct FDTDServe FDTDServe;

/* Engine on `device` with a device-memory budget for the requests' state,
 * at most max_requests admitted at a time.  Check FDTD_serve_last_error. */
FDTDServe *FDTD_serve_new(int device, double budget_bytes, int max_requests, int steps_per_replay);

/* Status and message of the engine's last failing call. */
int FDTD_serve_last_error(FDTDServe *s, char *buf, int buflen);

/* Admit a request: returns its slot (>= 0), -1 when the budget or the slot
 * table has no room for it now (collect finished requests and retry), or
 * -(status) on an invalid request.  The handle must not be used elsewhere
 * until it has been collected. */
int FDTD_serve_admit(FDTDServe *s, FDTDHandle *h, const FDTDSolveOptions *opt);

/* One graph replay; returns how many requests are ready to collect. */
int FDTD_serve_advance(FDTDServe *s);

/* Handles of up to max finished, not yet collected requests (so that their
 * t0 arrays can be provided just before collection); returns the count. */
int FDTD_serve_finished(FDTDServe *s, FDTDHandle **done, int max);

/* Retire up to max finished requests (fields into their t0 arrays); returns
 * the count, with the handles in done[] and their results in res[]. */
int FDTD_serve_collect(FDTDServe *s, FDTDHandle **done, FDTDSolveResult *res, int max);

/* Device bytes held by admitted requests and their number. */
int FDTD_serve_info(FDTDServe *s, double *used_bytes, int *active);

/* Releases the engine (and the state of requests never collected). */
void FDTD_serve_delete(FDTDServe *s);

/* ---- z slabs of one CW solve split over GPUs (replaces the reference's
 * multi-rank run: a PETSc DMDA chunk per MPI rank with the ghost exchange of
 * GhostComm, emopt/fdtd.py:273-297 and :1733-1873, src/fdtd.cpp:1789-1929).
 * A slab is a handle whose grid dims are the slab's (Nx, Ny, I planes), with
 * materials, sources and t0 arrays in slab coordinates and the global CPML
 * widths.  The caller runs the loop of FDTD_solve_cw and moves one pair of
 * planes per half step between neighbouring slabs:
 *     E halo (Ex, Ey plane 0 of the slab above) -> FDTD_slab_step(n, 0)
 *     H halo (Hx, Hy top plane of the slab below) -> FDTD_slab_step(n, 1)
 * Fields then equal those of the single-GPU solve on the whole grid. */

/* Launch the handle's work on `stream` (a cudaStream_t of the caller, e.g. the
 * stream a collective library orders its transfers on) instead of its own. */
int FDTD_set_stream(FDTDHandle *h, void *stream);

/* The handle holds planes [i0, i0 + Nz) of a grid of Nz_global planes (Nz =
 * its grid dims); has_lo / has_hi: a slab lies below / above (must match i0). */
int FDTD_slab_set(FDTDHandle *h, int i0, int Nz_global, int has_lo, int has_hi);

/* Resident set-up of the slab (vector kernel, non-periodic boundaries): uses
 * o->Tn, o->fixed_steps / o->Nmax (step table) and o->materials_unchanged.
 * cells[q], q < npoints: the probe points of the whole solve as global cells
 * (iz * Ny + j) * Nx + k, or -1 for a point that is always zero. */
int FDTD_slab_begin(FDTDHandle *h, const FDTDSolveOptions *o, const long long *cells, int npoints);

/* Half step of time step n: half 0 updates H, half 1 updates E. */
int FDTD_slab_step(FDTDHandle *h, long long n, int half);

/* Part of a half step, so that an exchange overlaps the planes that do not
 * need it: part 1 = every plane that reads no halo plane (all of them when
 * the slab has no neighbour on that side), part 2 = the plane next to the
 * neighbour's halo (the top plane of the H update, the bottom plane of the E
 * update; nothing without a neighbour), part 0 = all planes.  Parts 1 and 2
 * together equal part 0. */
int FDTD_slab_step_part(FDTDHandle *h, long long n, int half, int part);

/* Device addresses of the exchanged planes (plane_elems elements each, in the
 * slab's precision): ptrs[0..1] Ex, Ey of plane 0 (send down); ptrs[2..3] the
 * Ex, Ey halo above (receive from the slab above); ptrs[4..5] Hx, Hy of the
 * top plane (send up); ptrs[6..7] the Hx, Hy halo below (receive from below). */
int FDTD_slab_halo(FDTDHandle *h, void **ptrs, long long *plane_elems);

/* Where the half steps read the neighbour planes: ptrs[0..1] Ex, Ey of the
 * plane above the slab, ptrs[2..3] Hx, Hy of the plane below (device
 * addresses of Ny x px planes in the slab's precision, e.g. the neighbouring
 * slab's ptrs[0..1] / ptrs[4..5] of FDTD_slab_halo when it lives on the same
 * device: no exchange is then needed); NULL keeps the slab's own halo plane.
 * Holds until the next call. */
int FDTD_slab_set_halo_source(FDTDHandle *h, void *const *ptrs);

/* The half steps read the source table at (device step base) + n.  The base
 * is 0 after FDTD_slab_begin; FDTD_slab_set_step sets it in stream order, so
 * that K steps captured once with n = 0 .. K - 1 (a CUDA graph of
 * FDTD_slab_step calls) replay as steps base .. base + K - 1.  Set it back to
 * 0 before FDTD_slab_probe. */
int FDTD_slab_set_step(FDTDHandle *h, long long base);

/* Writes the probe values this slab holds (3 x npoints doubles, zero for the
 * points of other slabs) into a device buffer and returns its address; the
 * caller sums the buffers of all slabs into every slab's buffer. */
int FDTD_slab_sample(FDTDHandle *h, void **samples);

/* The convergence probe of FDTD_solve_cw (emopt/fdtd.py:1072-1138) on the
 * summed samples after step n_last; returns the amplitude and phase changes. */
int FDTD_slab_probe(FDTDHandle *h, long long n_last, double *A_change, double *phi_change);

/* Snapshot of the fields (which 0: t0 sample, 1: t1 sample). */
int FDTD_slab_capture(FDTDHandle *h, int which);

/* 3-sample extraction with t = n0 dt, (n0 + Tn) dt, (n0 + 2 Tn) dt into the
 * slab's t0 arrays (src/fdtd.cpp:1346-1443). */
int FDTD_slab_finish(FDTDHandle *h, long long n0, long long Tn);

/* Largest n accepted by FDTD_amp_phase_noalloc: 524288 complex128 values, the
 * 8 MiB device array it stages through. */
#define FDTD_NOALLOC_MAX_VALUES 524288

/* No counterpart in the reference.  Rewrites the n complex values of the
 * array a (host memory, or memory the device can address: every copy lets the
 * runtime infer the direction, as FDTD_add_source's do) in place as
 * (|a|, -atan2(im, re)) -- the conversion FDTD_add_source
 * applies to each source component when calc_phase is true -- on GPU `device`,
 * without allocating any device memory.  It is meant for callers that cannot
 * allocate: a process whose device memory is already committed to a memory
 * pool or to resident solves, or a thread preparing sources while solves run
 * on other streams (the cudaFree behind FDTD_add_source's temporary buffer
 * waits for all work on the device).  Convert the six components with it, then
 * register them with FDTD_add_source(..., calc_phase = false).
 *   stream: a cudaStream_t of `device`, or NULL for the calling thread's
 *           default stream; the call returns after that stream has finished.
 *   msg:    optional buffer (msglen bytes) for an error message.
 * n above FDTD_NOALLOC_MAX_VALUES fails with FDTD_ERR_ARG.  Every GPU that
 * loads this library holds the 8 MiB array until the process exits.  Each call
 * looks up the array's address on its device; the first lookup on a device
 * loads the library's device code there (set-up), so make the first call
 * before any stream capture.  All calls on a device share the array, so calls that
 * overlap in time (from several host threads) race and must be serialised. */
int FDTD_amp_phase_noalloc(int device, void *stream, fdtd_complex128 *a, long long n, char *msg,
                           int msglen);

/* ---- field access around a solve, on the device (replaces the numpy forms
 * of emopt/fdtd.py:1401-1667 and emopt/fomutils.py:1282-1426 when the
 * phasors live in device memory).  Arrays are complex128 in device memory,
 * [z][y][x].  geom: 17 ints describing the block an interpolation reads --
 * origin (i, j, k) in the array, extents (ni, nj, nk), the requested domain's
 * offset in the block (di, dj, dk) and extents (oi, oj, ok), the array's
 * dims (NX, NY, NZ), and the sign of the mirrored pad at a symmetric min face
 * in x and y (-1 'E', +1 'H', 0 none); emopt_b200/fieldops.py derives it the
 * way the reference slices its arrays.  comp: 0..5 = Ex Ey Ez Hx Hy Hz.
 * All return a status (message in msg). */

/* The component interpolated onto the Ez grid (get_field_interp,
 * emopt/fdtd.py:1401-1553): out[oi][oj][ok]. */
int FDTD_interp_field(int device, void *stream, int comp, const fdtd_complex128 *raw,
                      const int *geom, fdtd_complex128 *out, char *msg, int msglen);

/* The exact transpose of FDTD_interp_field: the cotangent gout[oi][oj][ok]
 * mapped onto the block read, graw[ni][nj][nk] (overwritten). */
int FDTD_interp_field_T(int device, void *stream, int comp, const fdtd_complex128 *gout,
                        const int *geom, fdtd_complex128 *graw, char *msg, int msglen);

/* interpolated_dFdx_3D of one component (emopt/fomutils.py:1282-1426):
 * dF[nz][ny][nx] (derivative with respect to the interpolated field on a
 * domain) -> out[nz+1][ny+1][nx+1] on the domain grown by one cell towards
 * -x, -y and +z.  qx: the reference's rule for Ex at a symmetric x-min face
 * (0 none, 1 'H', 2 'E'); qy: sign of its rule for Ey, Hx, Hz at a symmetric
 * y-min face (0 none). */
int FDTD_dfdx_interp(int device, void *stream, int comp, const fdtd_complex128 *dF, int nx, int ny,
                     int nz, int qx, int qy, fdtd_complex128 *out, char *msg, int msglen);

/* Poynting sums of the source power (get_source_power, emopt/fdtd.py:1555-
 * 1667): for each of nplanes <= 6 planes, sum over its cells of
 * Re(E1 conj(H2) - E2 conj(H1)) = Re(E x H*) . n -- (Ey, Hz, Ez, Hy) for
 * axes[p] = 0, (Ez, Hx, Ex, Hz) for 1, (Ex, Hy, Ey, Hx) for 2 -- every
 * component interpolated as FDTD_interp_field does.  blocks[6p + c]: component c of plane p's raw
 * block; geoms: 17 ints per plane.  sums: device memory of at least
 * 6 + 6 * 148 doubles (partial sums); sums[p] receives plane p's sum, in a
 * fixed summation order. */
int FDTD_plane_flux(int device, void *stream, int nplanes, const fdtd_complex128 *const *blocks,
                    const int *geoms, const int *axes, double *sums, char *msg, int msglen);

/* ---- layered materials on the GPU (replaces the host evaluation of the
 * reference's StructuredMaterial3D with Rectangle, Polygon and Circle
 * primitives, src/Grid.cpp:141-395 and :460-874, bound by emopt/grid_ctypes.py).
 * zs[0..nzs-1]: ascending layer boundaries; layer l (zs[l]..zs[l+1]) holds the
 * primitives layer_prims[layer_start[l] .. layer_start[l+1]) in priority order.
 * Primitive p: prim_info[4p..4p+3] = outline vertex start and count, convex
 * part start and count (a circle: count -1, centre and (radius, 0) in its two
 * vertex slots, no parts); prim_vals[6p..6p+5] = Re, Im, xmin, xmax, ymin, ymax
 * (outline bounding box).  Part q: parts[2q..2q+1] = vertex start and count
 * (counter-clockwise, convex).  verts: x, y pairs of outlines and parts.
 * Writes the values at fractional indices (k + sx, j + sy, i + sz),
 * k1 <= k < k2, ..., into out[(i - i1)(j2 - j1)(k2 - k1) + (j - j1)(k2 - k1)
 * + (k - k1)] (host or device memory), like StructuredMaterial3D::get_values. */
int FDTD_structured_values(int device, void *stream, const double *zs, int nzs,
                           const int *layer_start, const int *layer_prims, const int *prim_info,
                           const double *prim_vals, int nprims, const int *parts, int nparts,
                           const double *verts, int nverts, double dx, double dy, double dz,
                           int k1, int k2, int j1, int j2, int i1, int i2, double sx, double sy,
                           double sz, fdtd_complex128 *out, char *msg, int msglen);

/* ---- full-vector waveguide modes (replaces the SLEPc/MUMPS solve of the
 * reference's ModeFullVector, emopt/modes.py:1099-2298, which assembles
 * A x = n B x with PETSc and solves it by shift-and-invert about n0).
 * The plane (M rows of N points; row y, column x) is cut into lines: rows of
 * constant y when sweep_y, else columns of constant x.  A line of L points
 * holds nb = 6 L unknowns (Ex Ey Ez Hx Hy Hz blocks of L), NL lines in all;
 * vectors are complex128 in line order ((l * 6 + c) * L + p).  All pointers
 * are device memory; complex values are interleaved (re, im) doubles.  The
 * caller factors the block-tridiagonal A - n0 B (block cyclic reduction with
 * a device LU for the dense inverses) and applies its inverse with
 * FDTD_mode_lines_gemv over the lines of each reduction level. */
typedef struct FDTDModeLines {
    int M, N;
    int sweep_y;
} FDTDModeLines;

/* Message of the last failing FDTD_mode_* call of this host thread. */
const char *FDTD_mode_last_error(void);

/* Blocks D_l of A - sigma B (emopt/modes.py:1361-1585; D: NL x nb x nb) and
 * the couplings of each row to the lines before and after (pcol/ncol: column
 * in that line or -1; pval/nval: the coefficient; NL x nb each).  planes[6]:
 * eps_x eps_y eps_z mu_x mu_y mu_z on the plane ([M][N] complex128, sampled
 * where the reference's build samples them); bc: the plane's two boundary
 * letters; odx, ody: wavelength/(2 pi) over the spacings; dir: +1, or -1 for
 * a backward mode. */
int FDTD_mode_assemble(const FDTDModeLines *g, int device, void *stream, double odx, double ody,
                       double dir, double sigma_re, double sigma_im, const double *const *planes,
                       const char *bc, double *D, int *pcol, double *pval, int *ncol, double *nval);

/* out = B v (line order; B of emopt/modes.py:1361-1585, dir: +1 or -1). */
int FDTD_mode_bmul(const FDTDModeLines *g, int device, void *stream, double dir, const double *v,
                   double *out);

/* Batched over lines: for l = lines[0..nlines-1],
 *   out_l[a] += sum_b W_l[a][b] (rhs_l[b] - corr_l[b])
 * for the rows a in rows[0..nrows-1] (rows null: all nb rows, nrows = nb);
 * W: NL x nb x nb blocks, rhs/corr/out: NL x nb (corr may be null; out is
 * accumulated into, so zero it first). */
int FDTD_mode_lines_gemv(int nb, int device, void *stream, const double *W, const int *lines,
                         int nlines, const int *rows, int nrows, const double *rhs,
                         const double *corr, double *out);

/* Couplings between lines, batched over z < nlines:
 *   dst[lines[z]][rows[i]] += sign * sum_j C[z][i][j] src[nbrs[z]][cols[j]],
 * C: nlines x R x Q dense complex128, src/dst: NL x nb (line order). */
int FDTD_mode_couple(int nb, int device, void *stream, int nlines, int R, int Q, const double *C,
                     const int *lines, const int *nbrs, const int *rows, const int *cols,
                     const double *src, double *dst, double sign);

/* Current sources of a mode (ModeFullVector.get_source, emopt/modes.py:2144-
 * 2296) from its six raw field planes (fields: [6][M][N], solver order):
 * scaled by s = 1/sqrt(S), ekz = exp(i dir neff dz/2); dxn, dyn, dzn: the
 * non-dimensional spacings along the plane's axes and its normal; eps, mu05,
 * mu50: [M][N] material planes; out: [6][M][N] Jx Jy Jz Mx My Mz in the
 * plane's own axes. */
int FDTD_mode_source(int device, void *stream, int M, int N, const double *fields, double s_re,
                     double s_im, double ekz_re, double ekz_im, double dxn, double dyn, double dzn,
                     const double *eps, const double *mu05, const double *mu50, const char *bc,
                     double *out);

#ifdef __cplusplus
}
#endif

#endif /* EMOPT_FDTD_H */
