// legacy_kernels.cu -- fp64 kernels on the reference's padded chunk layout.
//
// These back the per-call ABI entry points FDTD_update_H / FDTD_update_E /
// FDTD_capture_* / FDTD_calc_complex_fields_* when a caller drives the time
// loop itself through the reference ABI (emopt/fdtd_ctypes.py:26-149).  The
// library then works on device mirrors of the caller's padded arrays
// (idx = (i+1)(J+2)(K+2) + (j+1)(K+2) + k+1, src/fdtd.cpp:178), honours the
// chunk offsets of FDTD_set_local_grid, materialises the boundary conditions
// in the ghost layer exactly where src/fdtd.cpp:141-173 and 397-501 do, and
// keeps the CPML state in per-slab arrays sized like src/fdtd.cpp:779-876.
// One thread updates one cell; sources are applied one box per launch so that
// overlapping boxes accumulate in the reference order.
#include "kernels.h"

namespace fdtdb {

namespace {

__device__ __forceinline__ long long pad_idx(const LegacyView& v, int i, int j, int k) {
    return ((long long)(i + 1) * (v.J + 2) + (j + 1)) * (long long)(v.K + 2) + (k + 1);
}

__device__ __forceinline__ long long glob_idx(const LegacyView& v, int i, int j, int k) {
    return ((long long)i * v.J + j) * v.K + k;
}

// CPML slab membership of local cell (i,j,k) along axis a: returns the side
// (0 min, 1 max) or -1, the psi slot and the table index.
__device__ __forceinline__ int slab(const LegacyView& v, int a, int i, int j, int k,
                                    long long& slot, int& tq) {
    int c = a == 0 ? k : (a == 1 ? j : i);
    int lo = a == 0 ? v.k0 : (a == 1 ? v.j0 : v.i0);
    int n = a == 0 ? v.K : (a == 1 ? v.J : v.I);
    int N = a == 0 ? v.Nx : (a == 1 ? v.Ny : v.Nz);
    int g = c + lo, emin = v.w[2 * a], emax = N - v.w[2 * a + 1];
    int side, depth, local;
    if (g < emin) {
        side = 0; depth = emin - lo; local = c; tq = emin - c - lo - 1;
    } else if (a == 2 ? (g > emax) : (g >= emax)) {
        side = 1; depth = lo + n - emax; local = g - emax; tq = g - emax + v.w[2 * a];
    } else {
        return -1;
    }
    if (a == 0) slot = ((long long)i * v.J + j) * depth + local;
    else if (a == 1) slot = ((long long)i * depth + local) * v.K + k;
    else slot = ((long long)local * v.J + j) * v.K + k;
    return side;
}

__device__ __forceinline__ double cpml(double* psi, double kap, double b, double C, double d) {
    double p = C * d + b * *psi;
    *psi = p;
    return p - d + d / kap;
}

__device__ __forceinline__ void eps_coeffs(const LegacyView& v, c128 e, double& a, double& b) {
    if (!v.lossy) {
        a = 1.0;
        b = v.dt / e.real;
    } else {
        double rdt = e.real * v.odt, ih = e.imag * 0.5;
        a = (rdt - ih) / (rdt + ih);
        b = 1.0 / (rdt + ih);
    }
}

// Max faces: tangential E ghost := 0 unless periodic (src/fdtd.cpp:141-173).
__global__ void k_zero_max_E(LegacyView v) {
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    int face = blockIdx.y;
    if (v.bc[face] == 'P') return;
    if (face == 0) {
        if (v.k0 + v.K != v.Nx || u >= v.I * v.J) return;
        long long p = pad_idx(v, u / v.J, u % v.J, v.K);
        v.E[1][p] = 0.0; v.E[2][p] = 0.0;
    } else if (face == 1) {
        if (v.j0 + v.J != v.Ny || u >= v.I * v.K) return;
        long long p = pad_idx(v, u / v.K, v.J, u % v.K);
        v.E[0][p] = 0.0; v.E[2][p] = 0.0;
    } else {
        if (v.i0 + v.I != v.Nz || u >= v.J * v.K) return;
        long long p = pad_idx(v, v.I, u / v.K, u % v.K);
        v.E[0][p] = 0.0; v.E[1][p] = 0.0;
    }
}

// Min faces: H ghost := 0 / -H_first / +H_first for bc '0' / 'E' / 'H'
// (src/fdtd.cpp:397-501); other characters leave the ghost untouched.
__global__ void k_set_min_H(LegacyView v) {
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    int face = blockIdx.y;
    char bc = v.bc[face];
    if (bc != '0' && bc != 'E' && bc != 'H') return;
    long long p, step;
    double *f1, *f2;
    if (face == 0) {
        if (v.k0 != 0 || u >= v.I * v.J) return;
        p = pad_idx(v, u / v.J, u % v.J, -1); step = 1; f1 = v.H[1]; f2 = v.H[2];
    } else if (face == 1) {
        if (v.j0 != 0 || u >= v.I * v.K) return;
        p = pad_idx(v, u / v.K, -1, u % v.K); step = v.K + 2; f1 = v.H[0]; f2 = v.H[2];
    } else {
        if (v.i0 != 0 || u >= v.J * v.K) return;
        p = pad_idx(v, -1, u / v.K, u % v.K); step = (long long)(v.J + 2) * (v.K + 2);
        f1 = v.H[0]; f2 = v.H[1];
    }
    if (bc == '0') { f1[p] = 0.0; f2[p] = 0.0; }
    else if (bc == 'E') { f1[p] = -1 * f1[p + step]; f2[p] = -1 * f2[p + step]; }
    else { f1[p] = f1[p + step]; f2[p] = f2[p + step]; }
}

__global__ void __launch_bounds__(256) k_legacy_H(LegacyView v) {
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 8 + threadIdx.y;
    int i = blockIdx.z;
    if (k >= v.K || j >= v.J) return;
    long long p = pad_idx(v, i, j, k), g = glob_idx(v, i, j, k);
    long long sj = v.K + 2, si = (long long)(v.J + 2) * (v.K + 2);
    const double *Ex = v.E[0], *Ey = v.E[1], *Ez = v.E[2];
    double mx = v.dt / v.mu[0][g].real, my = v.dt / v.mu[1][g].real, mz = v.dt / v.mu[2][g].real;
    double dEzdy = v.ody * (Ez[p + sj] - Ez[p]);
    double dEydz = v.odz * (Ey[p + si] - Ey[p]);
    double dExdz = v.odz * (Ex[p + si] - Ex[p]);
    double dEzdx = v.odx * (Ez[p + 1] - Ez[p]);
    double dEydx = v.odx * (Ey[p + 1] - Ey[p]);
    double dExdy = v.ody * (Ex[p + sj] - Ex[p]);
    double hx = v.H[0][p] + mx * (dEydz - dEzdy);
    double hy = v.H[1][p] + my * (dEzdx - dExdz);
    double hz = v.H[2][p] + mz * (dExdy - dEydx);
    long long s; int tq, side;
    if ((side = slab(v, 0, i, j, k, s, tq)) >= 0) {
        double* const* ps = v.psi[0][side];
        double kap = v.tab[0][0][tq], b = v.tab[0][1][tq], C = v.tab[0][2][tq];
        double cy = cpml(ps[0] + s, kap, b, C, dEydx);
        double cz = cpml(ps[1] + s, kap, b, C, dEzdx);
        hz = hz - mz * cy;
        hy = hy + my * cz;
    }
    if ((side = slab(v, 1, i, j, k, s, tq)) >= 0) {
        double* const* ps = v.psi[1][side];
        double kap = v.tab[1][0][tq], b = v.tab[1][1][tq], C = v.tab[1][2][tq];
        double cx = cpml(ps[0] + s, kap, b, C, dExdy);
        double cz = cpml(ps[1] + s, kap, b, C, dEzdy);
        hz = hz + mz * cx;
        hx = hx - mx * cz;
    }
    if ((side = slab(v, 2, i, j, k, s, tq)) >= 0) {
        double* const* ps = v.psi[2][side];
        double kap = v.tab[2][0][tq], b = v.tab[2][1][tq], C = v.tab[2][2][tq];
        double cx = cpml(ps[0] + s, kap, b, C, dExdz);
        double cy = cpml(ps[1] + s, kap, b, C, dEydz);
        hx = hx + mx * cy;
        hy = hy - my * cx;
    }
    v.H[0][p] = hx; v.H[1][p] = hy; v.H[2][p] = hz;
}

__global__ void __launch_bounds__(256) k_legacy_E(LegacyView v) {
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 8 + threadIdx.y;
    int i = blockIdx.z;
    if (k >= v.K || j >= v.J) return;
    long long p = pad_idx(v, i, j, k), g = glob_idx(v, i, j, k);
    long long sj = v.K + 2, si = (long long)(v.J + 2) * (v.K + 2);
    const double *Hx = v.H[0], *Hy = v.H[1], *Hz = v.H[2];
    double ax, ay, az, bx, by, bz;
    eps_coeffs(v, v.eps[0][g], ax, bx);
    eps_coeffs(v, v.eps[1][g], ay, by);
    eps_coeffs(v, v.eps[2][g], az, bz);
    double dHzdy = v.ody * (Hz[p] - Hz[p - sj]);
    double dHydz = v.odz * (Hy[p] - Hy[p - si]);
    double dHxdz = v.odz * (Hx[p] - Hx[p - si]);
    double dHzdx = v.odx * (Hz[p] - Hz[p - 1]);
    double dHydx = v.odx * (Hy[p] - Hy[p - 1]);
    double dHxdy = v.ody * (Hx[p] - Hx[p - sj]);
    double ex = ax * v.E[0][p] + (dHzdy - dHydz) * bx;
    double ey = ay * v.E[1][p] + (dHxdz - dHzdx) * by;
    double ez = az * v.E[2][p] + (dHydx - dHxdy) * bz;
    long long s; int tq, side;
    if ((side = slab(v, 0, i, j, k, s, tq)) >= 0) {
        double* const* ps = v.psi[0][side];
        double kap = v.tab[0][3][tq], b = v.tab[0][4][tq], C = v.tab[0][5][tq];
        double cy = cpml(ps[2] + s, kap, b, C, dHydx);
        double cz = cpml(ps[3] + s, kap, b, C, dHzdx);
        ez = ez + cy * bz;
        ey = ey - cz * by;
    }
    if ((side = slab(v, 1, i, j, k, s, tq)) >= 0) {
        double* const* ps = v.psi[1][side];
        double kap = v.tab[1][3][tq], b = v.tab[1][4][tq], C = v.tab[1][5][tq];
        double cx = cpml(ps[2] + s, kap, b, C, dHxdy);
        double cz = cpml(ps[3] + s, kap, b, C, dHzdy);
        ez = ez - cx * bz;
        ex = ex + cz * bx;
    }
    if ((side = slab(v, 2, i, j, k, s, tq)) >= 0) {
        double* const* ps = v.psi[2][side];
        double kap = v.tab[2][3][tq], b = v.tab[2][4][tq], C = v.tab[2][5][tq];
        double cx = cpml(ps[2] + s, kap, b, C, dHxdz);
        double cy = cpml(ps[3] + s, kap, b, C, dHydz);
        ex = ex - cy * bx;
        ey = ey + cx * by;
    }
    v.E[0][p] = ex; v.E[1][p] = ey; v.E[2][p] = ez;
}

// One source box: H_c += src_t |M| dt/mu (magnetic) or E_c -= src_t |J| b (electric).
__global__ void k_legacy_source(LegacyView v, LegacySource s, bool electric, double t,
                                double T, double m, double kk) {
    long long n = (long long)s.I * s.J * s.K;
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int lk = (int)(q % s.K), lj = (int)((q / s.K) % s.J), li = (int)(q / ((long long)s.K * s.J));
    long long p = pad_idx(v, li + s.i0, lj + s.j0, lk + s.k0);
    long long g = glob_idx(v, li + s.i0, lj + s.j0, lk + s.k0);
    for (int c = 0; c < 3; c++) {
        if (electric) {
            c128 a = s.comp[c][q];
            double au, b;
            eps_coeffs(v, v.eps[c][g], au, b);
            double st = src_value(t, a.imag, T, m, kk);
            v.E[c][p] = v.E[c][p] - st * a.real * b;
        } else {
            c128 a = s.comp[3 + c][q];
            double st = src_value(t, a.imag, T, m, kk);
            v.H[c][p] = v.H[c][p] + st * a.real * v.dt / v.mu[c][g].real;
        }
    }
}

__global__ void k_legacy_capture(LegacyView v, c128* d0, c128* d1, c128* d2, c128* d3, c128* d4,
                                 c128* d5) {
    long long n = (long long)v.I * v.J * v.K;
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    int k = (int)(g % v.K), j = (int)((g / v.K) % v.J), i = (int)(g / ((long long)v.K * v.J));
    long long p = pad_idx(v, i, j, k);
    d0[g].real = v.E[0][p]; d1[g].real = v.E[1][p]; d2[g].real = v.E[2][p];
    d3[g].real = v.H[0][p]; d4[g].real = v.H[1][p]; d5[g].real = v.H[2][p];
}

struct C6 { c128* c[6]; };
struct CC6 { const c128* c[6]; };

__global__ void k_legacy_extract_2t(LegacyView v, C6 t0, double a, double b, double aH,
                                    double bH) {
    long long n = (long long)v.I * v.J * v.K;
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    int k = (int)(g % v.K), j = (int)((g / v.K) % v.J), i = (int)(g / ((long long)v.K * v.J));
    long long p = pad_idx(v, i, j, k);
    for (int c = 0; c < 6; c++) {
        double f1 = c < 3 ? v.E[c][p] : v.H[c - 3][p];
        t0.c[c][g] = c < 3 ? phasor_2t(a, b, t0.c[c][g].real, f1)
                           : phasor_2t(aH, bH, t0.c[c][g].real, f1);
    }
}

__global__ void k_legacy_extract_3t(LegacyView v, C6 t0, CC6 t1, Fit3 fE, Fit3 fH) {
    long long n = (long long)v.I * v.J * v.K;
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    int k = (int)(g % v.K), j = (int)((g / v.K) % v.J), i = (int)(g / ((long long)v.K * v.J));
    long long p = pad_idx(v, i, j, k);
    for (int c = 0; c < 6; c++) {
        double f2 = c < 3 ? v.E[c][p] : v.H[c - 3][p];
        t0.c[c][g] = phasor_3t(c < 3 ? fE : fH, t0.c[c][g].real, t1.c[c][g].real, f2);
    }
}

unsigned blocks_for(long long n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

}  // namespace

void legacy_update_H(const LegacyView& v, const LegacySource* srcs, int nsrc, double t,
                     double src_T, double src_min, double src_k, cudaStream_t st) {
    int face_max = max(v.I * v.J, max(v.I * v.K, v.J * v.K));
    k_zero_max_E<<<dim3(blocks_for(face_max, 256), 3), 256, 0, st>>>(v);
    if (v.I > 0 && v.J > 0 && v.K > 0)
        k_legacy_H<<<dim3((v.K + 31) / 32, (v.J + 7) / 8, v.I), dim3(32, 8), 0, st>>>(v);
    for (int q = 0; q < nsrc; q++) {
        long long n = (long long)srcs[q].I * srcs[q].J * srcs[q].K;
        if (n > 0)
            k_legacy_source<<<blocks_for(n, 256), 256, 0, st>>>(v, srcs[q], false, t, src_T,
                                                                  src_min, src_k);
    }
}

void legacy_update_E(const LegacyView& v, const LegacySource* srcs, int nsrc, double t,
                     double src_T, double src_min, double src_k, cudaStream_t st) {
    int face_max = max(v.I * v.J, max(v.I * v.K, v.J * v.K));
    k_set_min_H<<<dim3(blocks_for(face_max, 256), 3), 256, 0, st>>>(v);
    if (v.I > 0 && v.J > 0 && v.K > 0)
        k_legacy_E<<<dim3((v.K + 31) / 32, (v.J + 7) / 8, v.I), dim3(32, 8), 0, st>>>(v);
    for (int q = 0; q < nsrc; q++) {
        long long n = (long long)srcs[q].I * srcs[q].J * srcs[q].K;
        if (n > 0)
            k_legacy_source<<<blocks_for(n, 256), 256, 0, st>>>(v, srcs[q], true, t, src_T,
                                                                  src_min, src_k);
    }
}

void legacy_capture(const LegacyView& v, c128* const* dst, cudaStream_t st) {
    long long n = (long long)v.I * v.J * v.K;
    if (n > 0)
        k_legacy_capture<<<blocks_for(n, 256), 256, 0, st>>>(v, dst[0], dst[1], dst[2], dst[3],
                                                              dst[4], dst[5]);
}

void legacy_extract_2t(const LegacyView& v, c128* const* t0, double t0v, double t1v,
                       cudaStream_t st) {
    long long n = (long long)v.I * v.J * v.K;
    C6 a;
    for (int c = 0; c < 6; c++) a.c[c] = t0[c];
    if (n > 0)
        k_legacy_extract_2t<<<blocks_for(n, 256), 256, 0, st>>>(
            v, a, t0v, t1v, t0v - 0.5 * v.dt, t1v - 0.5 * v.dt);
}

void legacy_extract_3t(const LegacyView& v, c128* const* t0, const c128* const* t1, double t0v,
                       double t1v, double t2v, cudaStream_t st) {
    long long n = (long long)v.I * v.J * v.K;
    C6 a;
    CC6 b;
    for (int c = 0; c < 6; c++) { a.c[c] = t0[c]; b.c[c] = t1[c]; }
    Fit3 fE = make_fit3(t0v, t1v, t2v);
    Fit3 fH = make_fit3(t0v - 0.5 * v.dt, t1v - 0.5 * v.dt, t2v - 0.5 * v.dt);
    if (n > 0) k_legacy_extract_3t<<<blocks_for(n, 256), 256, 0, st>>>(v, a, b, fE, fH);
}

}  // namespace fdtdb
