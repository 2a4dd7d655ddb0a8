/*
 * fdtd_oracle.c -- CPU restatement of EMopt's 3D CW-FDTD hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: the parity tests, the
 * smoke check and bench.py's CPU-baseline leg use it as a checker.  Nothing in
 * the emopt_b200 product path loads, links or calls it.
 *
 * It exports the same C ABI as the reference FDTD.so (src/fdtd.hpp:571-643) so
 * that one Python driver (oracle/driver.py) can run either this restatement or
 * the reference library compiled from its own sources (oracle/_ref/FDTD.so).
 * Parity pin: tests/test_oracle.py checks this file bit-for-bit against the
 * reference build and against the committed golden vectors in tests/golden/.
 *
 * The floating-point expressions are kept in the reference's association order
 * (compiled with -ffp-contract=off) because the oracle is required to be
 * bit-identical to the reference on the same inputs; the code structure
 * (per-axis CPML helper, source/table handling) is this project's own.
 *
 * Layout conventions (src/fdtd.cpp:178-183): local field arrays are padded by
 * one ghost layer, x fastest:  p(i,j,k) = (i+1)(J+2)(K+2) + (j+1)(K+2) + (k+1);
 * material, snapshot and source arrays are unpadded: g = i*J*K + j*K + k.
 */
#include <math.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { double real, imag; } c128;

enum { AX_X = 0, AX_Y = 1, AX_Z = 2 };
/* coefficient table slots per axis */
enum { T_KH = 0, T_BH, T_CH, T_KE, T_BE, T_CE, T_COUNT };

typedef struct {
    c128 *cur[6];          /* Jx Jy Jz Mx My Mz: (amplitude, phase) after conversion */
    int i0, j0, k0, I, J, K;
} orc_src;

typedef struct {
    int Nx, Ny, Nz;
    int I, J, K, i0, j0, k0;
    double X, Y, Z, dx, dy, dz;
    double wavelength, R, dt, odt;
    double src_T, src_min, src_k;
    bool complex_eps;
    double *E[3], *H[3];
    c128 *eps[3], *mu[3];
    c128 *t0[6], *t1[6];
    int w[6];                       /* xmin xmax ymin ymax zmin zmax (cells) */
    double sigma, alpha, kappa, pw;
    char bc[3];
    /* CPML auxiliary arrays: psi[axis][side][slot]; slots 0,1 are the two
     * E-derivative accumulators used by the H update, slots 2,3 the two
     * H-derivative accumulators used by the E update. */
    double *psi[3][2][4];
    double *tab[3][T_COUNT];
    orc_src *src;
    int nsrc, src_cap;
} orc_fdtd;

/* ---------------------------------------------------------------- setup -- */

void *FDTD_new(void)
{
    orc_fdtd *s = (orc_fdtd *)calloc(1, sizeof(orc_fdtd));
    s->bc[0] = s->bc[1] = s->bc[2] = '0';
    return s;
}

void FDTD_delete(void *h)
{
    orc_fdtd *s = (orc_fdtd *)h;
    if (!s) return;
    for (int a = 0; a < 3; a++)
        for (int sd = 0; sd < 2; sd++)
            for (int q = 0; q < 4; q++) free(s->psi[a][sd][q]);
    for (int a = 0; a < 3; a++)
        for (int q = 0; q < T_COUNT; q++) free(s->tab[a][q]);
    free(s->src);
    free(s);
}

/* src/fdtd.cpp:89-93 */
void FDTD_set_wavelength(void *h, double wavelength)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->wavelength = wavelength;
    s->R = wavelength / (2 * M_PI);
}

/* src/fdtd.cpp:66-71 */
void FDTD_set_physical_dims(void *h, double X, double Y, double Z,
                            double dx, double dy, double dz)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->X = X; s->Y = Y; s->Z = Z;
    s->dx = dx; s->dy = dy; s->dz = dz;
}

/* src/fdtd.cpp:73-78 */
void FDTD_set_grid_dims(void *h, int Nx, int Ny, int Nz)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->Nx = Nx; s->Ny = Ny; s->Nz = Nz;
}

/* src/fdtd.cpp:81-86 (argument order k0,j0,i0,K,J,I) */
void FDTD_set_local_grid(void *h, int k0, int j0, int i0, int K, int J, int I)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->k0 = k0; s->j0 = j0; s->i0 = i0;
    s->K = K; s->J = J; s->I = I;
}

/* src/fdtd.cpp:96-100: the CPML tables are NOT rebuilt here */
void FDTD_set_dt(void *h, double dt)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->dt = dt;
    s->odt = 1.0 / dt;
}

void FDTD_set_complex_eps(void *h, bool complex_eps)
{
    ((orc_fdtd *)h)->complex_eps = complex_eps;
}

void FDTD_set_field_arrays(void *h, double *Ex, double *Ey, double *Ez,
                           double *Hx, double *Hy, double *Hz)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->E[0] = Ex; s->E[1] = Ey; s->E[2] = Ez;
    s->H[0] = Hx; s->H[1] = Hy; s->H[2] = Hz;
}

void FDTD_set_mat_arrays(void *h, c128 *ex, c128 *ey, c128 *ez,
                         c128 *mx, c128 *my, c128 *mz)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->eps[0] = ex; s->eps[1] = ey; s->eps[2] = ez;
    s->mu[0] = mx; s->mu[1] = my; s->mu[2] = mz;
}

void FDTD_set_bc(void *h, char *bc)
{
    orc_fdtd *s = (orc_fdtd *)h;
    for (int a = 0; a < 3; a++) s->bc[a] = bc[a];
}

/* ---------------------------------------------------------------- CPML --- */

void FDTD_set_pml_widths(void *h, int xmin, int xmax, int ymin, int ymax,
                         int zmin, int zmax)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->w[0] = xmin; s->w[1] = xmax; s->w[2] = ymin;
    s->w[3] = ymax; s->w[4] = zmin; s->w[5] = zmax;
}

/* One CPML coefficient triple for a ramp value f (src/fdtd.cpp:992-997). */
static void orc_cpml_coeffs(const orc_fdtd *s, double f, double *kap, double *b,
                            double *c)
{
    double sigma = s->sigma * f;
    double alpha = s->alpha * (1 - f);
    double kappa = (s->kappa - 1.0) * f + 1.0;
    double bb = exp(-s->dt * (sigma / kappa + alpha));
    *kap = kappa;
    *b = bb;
    *c = (bb == 1) ? 0.0 : (bb - 1) * sigma / (sigma * kappa + kappa * kappa * alpha);
}

/* Ramp value pow(d, pow), optionally clamped at zero (src/fdtd.cpp:1183-1186). */
static double orc_ramp(const orc_fdtd *s, double d, bool clamp)
{
    double f = pow(d, s->pw);
    if (clamp && f < 0) f = 0;
    return f;
}

/*
 * Build the per-axis 1-D tables (src/fdtd.cpp:950-1181).  Entry q < w_min
 * belongs to the min-side slab, w_min + q to the max side.  The distance
 * offsets differ between H and E and between x/y and z:
 *     x,y min : H (q-0.5)/w clamped, E q/w        x,y max : H (q+0.5)/w, E q/w
 *     z   min : H q/w, E (q+0.5)/w                z   max : H q/w, E (q-0.5)/w clamped
 */
static void orc_compute_tables(orc_fdtd *s)
{
    for (int a = 0; a < 3; a++) {
        int w0 = s->w[2 * a], w1 = s->w[2 * a + 1];
        for (int q = 0; q < T_COUNT; q++) {
            free(s->tab[a][q]);
            s->tab[a][q] = (double *)malloc(sizeof(double) * (size_t)(w0 + w1 > 0 ? w0 + w1 : 1));
        }
        for (int side = 0; side < 2; side++) {
            int w = side ? w1 : w0;
            for (int q = 0; q < w; q++) {
                double dH, dE;
                bool clampH = false, clampE = false;
                if (a != AX_Z) {
                    dH = side ? (double)(q + 0.5) / w : (double)(q - 0.5) / w;
                    clampH = !side;
                    dE = (double)q / w;
                } else {
                    dH = (double)q / w;
                    dE = side ? (double)(q - 0.5) / w : (double)(q + 0.5) / w;
                    clampE = side;
                }
                int at = side ? w0 + q : q;
                orc_cpml_coeffs(s, orc_ramp(s, dH, clampH), &s->tab[a][T_KH][at],
                                &s->tab[a][T_BH][at], &s->tab[a][T_CH][at]);
                orc_cpml_coeffs(s, orc_ramp(s, dE, clampE), &s->tab[a][T_KE][at],
                                &s->tab[a][T_BE][at], &s->tab[a][T_CE][at]);
            }
        }
    }
}

void FDTD_set_pml_properties(void *h, double sigma, double alpha, double kappa,
                             double pw)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->sigma = sigma; s->alpha = alpha; s->kappa = kappa; s->pw = pw;
    orc_compute_tables(s);
}

/* Number of cells of the local chunk covered by a slab (src/fdtd.cpp:786-876). */
static long orc_slab_cells(const orc_fdtd *s, int a, int side)
{
    int lo[3] = {s->k0, s->j0, s->i0};
    int n[3] = {s->K, s->J, s->I};
    int N[3] = {s->Nx, s->Ny, s->Nz};
    int depth;
    if (!side) {
        int edge = s->w[2 * a];
        if (!(lo[a] < edge)) return 0;
        depth = edge - lo[a];
    } else {
        int edge = N[a] - s->w[2 * a + 1];
        if (!(lo[a] + n[a] > edge)) return 0;
        depth = lo[a] + n[a] - edge;
    }
    long cells = depth;
    for (int b = 0; b < 3; b++)
        if (b != a) cells *= n[b];
    return cells;
}

void FDTD_build_pml(void *h)
{
    orc_fdtd *s = (orc_fdtd *)h;
    for (int a = 0; a < 3; a++)
        for (int sd = 0; sd < 2; sd++) {
            long n = orc_slab_cells(s, a, sd);
            for (int q = 0; q < 4; q++) {
                free(s->psi[a][sd][q]);
                s->psi[a][sd][q] = n ? (double *)calloc((size_t)n, sizeof(double)) : NULL;
            }
        }
    orc_compute_tables(s);
}

void FDTD_reset_pml(void *h)
{
    orc_fdtd *s = (orc_fdtd *)h;
    for (int a = 0; a < 3; a++)
        for (int sd = 0; sd < 2; sd++) {
            long n = orc_slab_cells(s, a, sd);
            for (int q = 0; q < 4; q++)
                if (s->psi[a][sd][q]) memset(s->psi[a][sd][q], 0, sizeof(double) * (size_t)n);
        }
}

/*
 * Locate cell (i,j,k) of the chunk inside the CPML slab of axis a.  Returns -1
 * when the cell is outside; otherwise *slot receives the psi index and *tq the
 * table index.  The z-max slab uses a strict comparison (src/fdtd.cpp:292,652),
 * so its first plane is never a PML cell.
 */
static int orc_slab_locate(const orc_fdtd *s, int a, int i, int j, int k,
                           long *slot, int *tq)
{
    int c[3] = {k, j, i};
    int lo[3] = {s->k0, s->j0, s->i0};
    int n[3] = {s->K, s->J, s->I};
    int N[3] = {s->Nx, s->Ny, s->Nz};
    int g = c[a] + lo[a];
    int edge_min = s->w[2 * a];
    int edge_max = N[a] - s->w[2 * a + 1];
    int side, depth, local;
    if (g < edge_min) {
        side = 0;
        depth = edge_min - lo[a];
        local = c[a];
        *tq = edge_min - c[a] - lo[a] - 1;
    } else if (a == AX_Z ? (g > edge_max) : (g >= edge_max)) {
        side = 1;
        depth = lo[a] + n[a] - edge_max;
        local = g - edge_max;
        *tq = g - edge_max + s->w[2 * a];
    } else {
        return -1;
    }
    /* psi layouts follow src/fdtd.cpp:214,231,247,262,278,293 */
    if (a == AX_X)
        *slot = ((long)i * s->J + j) * depth + local;
    else if (a == AX_Y)
        *slot = ((long)i * depth + local) * s->K + k;
    else
        *slot = ((long)local * s->J + j) * s->K + k;
    return side;
}

/* psi <- C*d + b*psi; returns the CPML correction psi - d + d/kappa. */
static inline double orc_cpml(double *psi, double kap, double b, double C, double d)
{
    *psi = C * d + b * *psi;
    return *psi - d + d / kap;
}

/* -------------------------------------------------------------- sources -- */

/* src/fdtd.cpp:1595-1602 */
static double orc_src_t(const orc_fdtd *s, double t, double phase)
{
    if (t <= s->src_T)
        return sin(t + phase) * ((1 + s->src_min) * exp(-(t - s->src_T) * (t - s->src_T) / s->src_k) - s->src_min);
    return sin(t + phase);
}

double FDTD_src_func_t(void *h, int n, double t, double phase)
{
    return orc_src_t((orc_fdtd *)h, t, phase);
}

/* src/fdtd.cpp:1586-1593 */
void FDTD_set_source_properties(void *h, double src_T, double src_min)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->src_T = src_T;
    s->src_min = src_min;
    s->src_k = src_T * src_T / log((1 + src_min) / src_min);
}

/* src/fdtd.cpp:1498-1579: complex currents are rewritten in place as
 * (|J|, -atan2(im, re)) when calc_phase is set; the arrays are retained. */
void FDTD_add_source(void *h, c128 *Jx, c128 *Jy, c128 *Jz, c128 *Mx, c128 *My,
                     c128 *Mz, int i0, int j0, int k0, int I, int J, int K,
                     bool calc_phase)
{
    orc_fdtd *s = (orc_fdtd *)h;
    c128 *arr[6] = {Jx, Jy, Jz, Mx, My, Mz};
    if (calc_phase) {
        long n = (long)I * J * K;
        for (long q = 0; q < n; q++)
            for (int c = 0; c < 6; c++) {
                double re = arr[c][q].real, im = arr[c][q].imag;
                arr[c][q].real = sqrt(re * re + im * im);
                arr[c][q].imag = (im == 0 && re == 0) ? 0.0 : -1 * atan2(im, re);
            }
    }
    if (s->nsrc == s->src_cap) {
        s->src_cap = s->src_cap ? 2 * s->src_cap : 4;
        s->src = (orc_src *)realloc(s->src, sizeof(orc_src) * (size_t)s->src_cap);
    }
    orc_src *q = &s->src[s->nsrc++];
    for (int c = 0; c < 6; c++) q->cur[c] = arr[c];
    q->i0 = i0; q->j0 = j0; q->k0 = k0; q->I = I; q->J = J; q->K = K;
}

void FDTD_clear_sources(void *h) { ((orc_fdtd *)h)->nsrc = 0; }

/* ------------------------------------------------------------ updates ---- */

static inline long orc_pad(const orc_fdtd *s, int i, int j, int k)
{
    return ((long)(i + 1) * (s->J + 2) + (j + 1)) * (s->K + 2) + (k + 1);
}

static inline long orc_glob(const orc_fdtd *s, int i, int j, int k)
{
    return ((long)i * s->J + j) * s->K + k;
}

/*
 * H half-step (src/fdtd.cpp:121-367): tangential E on the max faces is forced
 * to zero unless the axis is periodic, then H += dt/mu * curl(E) with forward
 * differences, CPML corrections in x, y, z order, and finally the magnetic
 * current sources.
 */
void FDTD_update_H(void *h, int n, double t)
{
    orc_fdtd *s = (orc_fdtd *)h;
    double *Ex = s->E[0], *Ey = s->E[1], *Ez = s->E[2];
    double *Hx = s->H[0], *Hy = s->H[1], *Hz = s->H[2];
    double odx = s->R / s->dx, ody = s->R / s->dy, odz = s->R / s->dz;
    long sj = s->K + 2, si = (long)(s->J + 2) * (s->K + 2);

    if (s->bc[0] != 'P' && s->k0 + s->K == s->Nx)
        for (int i = 0; i < s->I; i++)
            for (int j = 0; j < s->J; j++) {
                long p = orc_pad(s, i, j, s->K);
                Ey[p] = 0.0; Ez[p] = 0.0;
            }
    if (s->bc[1] != 'P' && s->j0 + s->J == s->Ny)
        for (int i = 0; i < s->I; i++)
            for (int k = 0; k < s->K; k++) {
                long p = orc_pad(s, i, s->J, k);
                Ex[p] = 0.0; Ez[p] = 0.0;
            }
    if (s->bc[2] != 'P' && s->i0 + s->I == s->Nz)
        for (int j = 0; j < s->J; j++)
            for (int k = 0; k < s->K; k++) {
                long p = orc_pad(s, s->I, j, k);
                Ex[p] = 0.0; Ey[p] = 0.0;
            }

    for (int i = 0; i < s->I; i++)
        for (int j = 0; j < s->J; j++)
            for (int k = 0; k < s->K; k++) {
                long p = orc_pad(s, i, j, k), g = orc_glob(s, i, j, k);
                double mx = s->dt / s->mu[0][g].real;
                double my = s->dt / s->mu[1][g].real;
                double mz = s->dt / s->mu[2][g].real;
                double dEzdy = ody * (Ez[p + sj] - Ez[p]);
                double dEydz = odz * (Ey[p + si] - Ey[p]);
                double dExdz = odz * (Ex[p + si] - Ex[p]);
                double dEzdx = odx * (Ez[p + 1] - Ez[p]);
                double dEydx = odx * (Ey[p + 1] - Ey[p]);
                double dExdy = ody * (Ex[p + sj] - Ex[p]);
                Hx[p] = Hx[p] + mx * (dEydz - dEzdy);
                Hy[p] = Hy[p] + my * (dEzdx - dExdz);
                Hz[p] = Hz[p] + mz * (dExdy - dEydx);

                long slot; int tq, side;
                if ((side = orc_slab_locate(s, AX_X, i, j, k, &slot, &tq)) >= 0) {
                    double **ps = s->psi[AX_X][side];
                    double kap = s->tab[AX_X][T_KH][tq], b = s->tab[AX_X][T_BH][tq], C = s->tab[AX_X][T_CH][tq];
                    double cy = orc_cpml(&ps[0][slot], kap, b, C, dEydx);
                    double cz = orc_cpml(&ps[1][slot], kap, b, C, dEzdx);
                    Hz[p] = Hz[p] - mz * cy;
                    Hy[p] = Hy[p] + my * cz;
                }
                if ((side = orc_slab_locate(s, AX_Y, i, j, k, &slot, &tq)) >= 0) {
                    double **ps = s->psi[AX_Y][side];
                    double kap = s->tab[AX_Y][T_KH][tq], b = s->tab[AX_Y][T_BH][tq], C = s->tab[AX_Y][T_CH][tq];
                    double cx = orc_cpml(&ps[0][slot], kap, b, C, dExdy);
                    double cz = orc_cpml(&ps[1][slot], kap, b, C, dEzdy);
                    Hz[p] = Hz[p] + mz * cx;
                    Hx[p] = Hx[p] - mx * cz;
                }
                if ((side = orc_slab_locate(s, AX_Z, i, j, k, &slot, &tq)) >= 0) {
                    double **ps = s->psi[AX_Z][side];
                    double kap = s->tab[AX_Z][T_KH][tq], b = s->tab[AX_Z][T_BH][tq], C = s->tab[AX_Z][T_CH][tq];
                    double cx = orc_cpml(&ps[0][slot], kap, b, C, dExdz);
                    double cy = orc_cpml(&ps[1][slot], kap, b, C, dEydz);
                    Hx[p] = Hx[p] + mx * cy;
                    Hy[p] = Hy[p] - my * cx;
                }
            }

    /* magnetic currents: H += src_t * |M| * dt / mu  (src/fdtd.cpp:313-366) */
    for (int q = 0; q < s->nsrc; q++) {
        const orc_src *sr = &s->src[q];
        for (int c = 0; c < 3; c++) {
            const c128 *M = sr->cur[3 + c];
            for (int i = 0; i < sr->I; i++)
                for (int j = 0; j < sr->J; j++)
                    for (int k = 0; k < sr->K; k++) {
                        long p = orc_pad(s, i + sr->i0, j + sr->j0, k + sr->k0);
                        long g = orc_glob(s, i + sr->i0, j + sr->j0, k + sr->k0);
                        long m = ((long)i * sr->J + j) * sr->K + k;
                        double st = orc_src_t(s, t, M[m].imag);
                        s->H[c][p] = s->H[c][p] + st * M[m].real * s->dt / s->mu[c][g].real;
                    }
        }
    }
}

/* E-update coefficients (src/fdtd.cpp:513-552). */
static inline void orc_eps_coeffs(const orc_fdtd *s, c128 e, double *a, double *b)
{
    if (!s->complex_eps) {
        *a = 1.0;
        *b = s->dt / e.real;
    } else {
        double rdt = e.real * s->odt, ih = e.imag * 0.5;
        *a = (rdt - ih) / (rdt + ih);
        *b = 1.0 / (rdt + ih);
    }
}

/*
 * E half-step (src/fdtd.cpp:369-755): the min-face H ghosts are set from the
 * boundary condition ('0' zero, 'E' odd copy, 'H' even copy, 'P' untouched),
 * then E = a E + b curl(H) with backward differences, CPML corrections in
 * x, y, z order, and the electric current sources (subtracted).
 */
void FDTD_update_E(void *h, int n, double t)
{
    orc_fdtd *s = (orc_fdtd *)h;
    double *Ex = s->E[0], *Ey = s->E[1], *Ez = s->E[2];
    double *Hx = s->H[0], *Hy = s->H[1], *Hz = s->H[2];
    double odx = s->R / s->dx, ody = s->R / s->dy, odz = s->R / s->dz;
    long sj = s->K + 2, si = (long)(s->J + 2) * (s->K + 2);

    /* ghost := sign * first interior value, or 0 */
    struct { int active; double *f1, *f2; } face[3] = {
        {s->k0 == 0, Hy, Hz}, {s->j0 == 0, Hx, Hz}, {s->i0 == 0, Hx, Hy}};
    long step[3] = {1, sj, si};
    for (int a = 0; a < 3; a++) {
        char bc = s->bc[a];
        if (!face[a].active || (bc != '0' && bc != 'E' && bc != 'H')) continue;
        int n1 = a == AX_X ? s->I : (a == AX_Y ? s->I : s->J);
        int n2 = a == AX_X ? s->J : (a == AX_Y ? s->K : s->K);
        for (int u = 0; u < n1; u++)
            for (int v = 0; v < n2; v++) {
                long p;
                if (a == AX_X) p = orc_pad(s, u, v, -1);
                else if (a == AX_Y) p = orc_pad(s, u, -1, v);
                else p = orc_pad(s, -1, u, v);
                long q = p + step[a];
                if (bc == '0') {
                    face[a].f1[p] = 0.0; face[a].f2[p] = 0.0;
                } else if (bc == 'E') {
                    face[a].f1[p] = -1 * face[a].f1[q]; face[a].f2[p] = -1 * face[a].f2[q];
                } else {
                    face[a].f1[p] = face[a].f1[q]; face[a].f2[p] = face[a].f2[q];
                }
            }
    }

    for (int i = 0; i < s->I; i++)
        for (int j = 0; j < s->J; j++)
            for (int k = 0; k < s->K; k++) {
                long p = orc_pad(s, i, j, k), g = orc_glob(s, i, j, k);
                double ax, ay, az, bx, by, bz;
                orc_eps_coeffs(s, s->eps[0][g], &ax, &bx);
                orc_eps_coeffs(s, s->eps[1][g], &ay, &by);
                orc_eps_coeffs(s, s->eps[2][g], &az, &bz);
                double dHzdy = ody * (Hz[p] - Hz[p - sj]);
                double dHydz = odz * (Hy[p] - Hy[p - si]);
                double dHxdz = odz * (Hx[p] - Hx[p - si]);
                double dHzdx = odx * (Hz[p] - Hz[p - 1]);
                double dHydx = odx * (Hy[p] - Hy[p - 1]);
                double dHxdy = ody * (Hx[p] - Hx[p - sj]);
                Ex[p] = ax * Ex[p] + (dHzdy - dHydz) * bx;
                Ey[p] = ay * Ey[p] + (dHxdz - dHzdx) * by;
                Ez[p] = az * Ez[p] + (dHydx - dHxdy) * bz;

                long slot; int tq, side;
                if ((side = orc_slab_locate(s, AX_X, i, j, k, &slot, &tq)) >= 0) {
                    double **ps = s->psi[AX_X][side];
                    double kap = s->tab[AX_X][T_KE][tq], b = s->tab[AX_X][T_BE][tq], C = s->tab[AX_X][T_CE][tq];
                    double cy = orc_cpml(&ps[2][slot], kap, b, C, dHydx);
                    double cz = orc_cpml(&ps[3][slot], kap, b, C, dHzdx);
                    Ez[p] = Ez[p] + cy * bz;
                    Ey[p] = Ey[p] - cz * by;
                }
                if ((side = orc_slab_locate(s, AX_Y, i, j, k, &slot, &tq)) >= 0) {
                    double **ps = s->psi[AX_Y][side];
                    double kap = s->tab[AX_Y][T_KE][tq], b = s->tab[AX_Y][T_BE][tq], C = s->tab[AX_Y][T_CE][tq];
                    double cx = orc_cpml(&ps[2][slot], kap, b, C, dHxdy);
                    double cz = orc_cpml(&ps[3][slot], kap, b, C, dHzdy);
                    Ez[p] = Ez[p] - cx * bz;
                    Ex[p] = Ex[p] + cz * bx;
                }
                if ((side = orc_slab_locate(s, AX_Z, i, j, k, &slot, &tq)) >= 0) {
                    double **ps = s->psi[AX_Z][side];
                    double kap = s->tab[AX_Z][T_KE][tq], b = s->tab[AX_Z][T_BE][tq], C = s->tab[AX_Z][T_CE][tq];
                    double cx = orc_cpml(&ps[2][slot], kap, b, C, dHxdz);
                    double cy = orc_cpml(&ps[3][slot], kap, b, C, dHydz);
                    Ex[p] = Ex[p] - cy * bx;
                    Ey[p] = Ey[p] + cx * by;
                }
            }

    /* electric currents: E -= src_t * |J| * b  (src/fdtd.cpp:672-754) */
    for (int q = 0; q < s->nsrc; q++) {
        const orc_src *sr = &s->src[q];
        for (int c = 0; c < 3; c++) {
            const c128 *Jc = sr->cur[c];
            for (int i = 0; i < sr->I; i++)
                for (int j = 0; j < sr->J; j++)
                    for (int k = 0; k < sr->K; k++) {
                        long p = orc_pad(s, i + sr->i0, j + sr->j0, k + sr->k0);
                        long g = orc_glob(s, i + sr->i0, j + sr->j0, k + sr->k0);
                        long m = ((long)i * sr->J + j) * sr->K + k;
                        double a_unused, b;
                        orc_eps_coeffs(s, s->eps[c][g], &a_unused, &b);
                        double st = orc_src_t(s, t, Jc[m].imag);
                        s->E[c][p] = s->E[c][p] - st * Jc[m].real * b;
                    }
        }
    }
}

/* ------------------------------------------------- steady-state extraction */

/* src/fdtd.cpp:1445-1463 */
double FDTD_calc_phase_2T(double t0, double t1, double f0, double f1)
{
    if (f0 == 0.0 && f1 == 0) return 0.0;
    return atan((f1 * sin(t0) - f0 * sin(t1)) / (f0 * cos(t1) - f1 * cos(t0)));
}

double FDTD_calc_amplitude_2T(double t0, double t1, double f0, double f1, double phase)
{
    if (f0 * f0 > f1 * f1) return f1 / (sin(t1) * cos(phase) + cos(t1) * sin(phase));
    return f0 / (sin(t0) * cos(phase) + cos(t0) * sin(phase));
}

/* src/fdtd.cpp:1465-1493 */
double FDTD_calc_phase_3T(double t0, double t1, double t2, double f0, double f1, double f2)
{
    double f10 = f1 - f0, f21 = f2 - f1;
    if (f10 == 0 && f21 == 0) return 0.0;
    return atan2(f10 * (sin(t2) - sin(t1)) - f21 * (sin(t1) - sin(t0)),
                 f21 * (cos(t1) - cos(t0)) - f10 * (cos(t2) - cos(t1)));
}

double FDTD_calc_amplitude_3T(double t0, double t1, double t2, double f0, double f1,
                              double f2, double phase)
{
    double f21 = f2 - f1, f10 = f1 - f0;
    if (f21 == 0 && f10 == 0) return 0.0;
    if (f21 * f21 >= f10 * f10)
        return f21 / (cos(phase) * (sin(t2) - sin(t1)) + sin(phase) * (cos(t2) - cos(t1)));
    return f10 / (cos(phase) * (sin(t1) - sin(t0)) + sin(phase) * (cos(t1) - cos(t0)));
}

void FDTD_set_t0_arrays(void *h, c128 *a, c128 *b, c128 *c, c128 *d, c128 *e, c128 *f)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->t0[0] = a; s->t0[1] = b; s->t0[2] = c; s->t0[3] = d; s->t0[4] = e; s->t0[5] = f;
}

void FDTD_set_t1_arrays(void *h, c128 *a, c128 *b, c128 *c, c128 *d, c128 *e, c128 *f)
{
    orc_fdtd *s = (orc_fdtd *)h;
    s->t1[0] = a; s->t1[1] = b; s->t1[2] = c; s->t1[3] = d; s->t1[4] = e; s->t1[5] = f;
}

/* Snapshot the six real fields into .real of the unpadded arrays
 * (src/fdtd.cpp:1205-1251); .imag is left untouched. */
static void orc_capture(orc_fdtd *s, c128 **dst)
{
    for (int i = 0; i < s->I; i++)
        for (int j = 0; j < s->J; j++)
            for (int k = 0; k < s->K; k++) {
                long p = orc_pad(s, i, j, k), g = orc_glob(s, i, j, k);
                for (int c = 0; c < 3; c++) {
                    dst[c][g].real = s->E[c][p];
                    dst[3 + c][g].real = s->H[c][p];
                }
            }
}

void FDTD_capture_t0_fields(void *h) { orc_capture((orc_fdtd *)h, ((orc_fdtd *)h)->t0); }
void FDTD_capture_t1_fields(void *h) { orc_capture((orc_fdtd *)h, ((orc_fdtd *)h)->t1); }

/* A e^{-i phi} after folding a negative amplitude into phi + pi. */
static inline c128 orc_phasor(double A, double phi)
{
    if (A < 0) {
        A *= -1;
        phi += M_PI;
    }
    c128 r = {A * cos(phi), -A * sin(phi)};
    return r;
}

/* src/fdtd.cpp:1253-1343; H samples are labelled half a step earlier. */
void FDTD_calc_complex_fields_2T(void *h, double t0, double t1)
{
    orc_fdtd *s = (orc_fdtd *)h;
    double t0H = t0 - 0.5 * s->dt, t1H = t1 - 0.5 * s->dt;
    for (int i = 0; i < s->I; i++)
        for (int j = 0; j < s->J; j++)
            for (int k = 0; k < s->K; k++) {
                long p = orc_pad(s, i, j, k), g = orc_glob(s, i, j, k);
                for (int c = 0; c < 6; c++) {
                    double a = c < 3 ? t0 : t0H, b = c < 3 ? t1 : t1H;
                    double f0 = s->t0[c][g].real;
                    double f1 = c < 3 ? s->E[c][p] : s->H[c - 3][p];
                    double phi = FDTD_calc_phase_2T(a, b, f0, f1);
                    double A = FDTD_calc_amplitude_2T(a, b, f0, f1, phi);
                    s->t0[c][g] = orc_phasor(A, phi);
                }
            }
}

/* src/fdtd.cpp:1346-1443 */
void FDTD_calc_complex_fields_3T(void *h, double t0, double t1, double t2)
{
    orc_fdtd *s = (orc_fdtd *)h;
    double tH[3] = {t0 - 0.5 * s->dt, t1 - 0.5 * s->dt, t2 - 0.5 * s->dt};
    double tE[3] = {t0, t1, t2};
    for (int i = 0; i < s->I; i++)
        for (int j = 0; j < s->J; j++)
            for (int k = 0; k < s->K; k++) {
                long p = orc_pad(s, i, j, k), g = orc_glob(s, i, j, k);
                for (int c = 0; c < 6; c++) {
                    const double *tt = c < 3 ? tE : tH;
                    double f0 = s->t0[c][g].real, f1 = s->t1[c][g].real;
                    double f2 = c < 3 ? s->E[c][p] : s->H[c - 3][p];
                    double phi = FDTD_calc_phase_3T(tt[0], tt[1], tt[2], f0, f1, f2);
                    double A = FDTD_calc_amplitude_3T(tt[0], tt[1], tt[2], f0, f1, f2, phi);
                    s->t0[c][g] = orc_phasor(A, phi);
                }
            }
}

/* --------------------------------------------- ghost exchange helpers ---- */

/* Face packing order xmin, xmax, ymin, ymax, zmin, zmax (src/fdtd.cpp:1789-1858). */
void FDTD_copy_to_ghost_comm(double *src, c128 *ghost, int I, int J, int K)
{
    long sj = K + 2, si = (long)(J + 2) * (K + 2), o = 0;
    for (int side = 0; side < 2; side++, o += (long)I * J)
        for (int i = 0; i < I; i++)
            for (int j = 0; j < J; j++)
                ghost[o + j + (long)i * J].real = src[(i + 1) * si + (j + 1) * sj + (side ? K : 1)];
    for (int side = 0; side < 2; side++, o += (long)I * K)
        for (int i = 0; i < I; i++)
            for (int k = 0; k < K; k++)
                ghost[o + k + (long)i * K].real = src[(i + 1) * si + (side ? J : 1) * sj + k + 1];
    for (int side = 0; side < 2; side++, o += (long)J * K)
        for (int j = 0; j < J; j++)
            for (int k = 0; k < K; k++)
                ghost[o + k + (long)j * K].real = src[(side ? I : 1) * si + (j + 1) * sj + k + 1];
}

/* Unpacks from the ghost region that follows the owned block
 * (src/fdtd.cpp:1860-1929). */
void FDTD_copy_from_ghost_comm(double *dest, c128 *ghost, int I, int J, int K)
{
    long sj = K + 2, si = (long)(J + 2) * (K + 2);
    long o = 2L * I * J + 2L * I * K + 2L * J * K;
    for (int side = 0; side < 2; side++, o += (long)I * J)
        for (int i = 0; i < I; i++)
            for (int j = 0; j < J; j++)
                dest[(i + 1) * si + (j + 1) * sj + (side ? K + 1 : 0)] = ghost[o + j + (long)i * J].real;
    for (int side = 0; side < 2; side++, o += (long)I * K)
        for (int i = 0; i < I; i++)
            for (int k = 0; k < K; k++)
                dest[(i + 1) * si + (side ? J + 1 : 0) * sj + k + 1] = ghost[o + k + (long)i * K].real;
    for (int side = 0; side < 2; side++, o += (long)J * K)
        for (int j = 0; j < J; j++)
            for (int k = 0; k < K; k++)
                dest[(side ? I + 1 : 0) * si + (j + 1) * sj + k + 1] = ghost[o + k + (long)j * K].real;
}
