// Full-vector waveguide mode solver on the GPU: the kernels behind
// emopt_b200/modes.py (the reference's ModeFullVector, emopt/modes.py:1099-2298).
//
// The reference assembles A and B of A x = n B x over the six field
// components of a plane (6 M N unknowns, emopt/modes.py:1278-1588) and hands
// them to SLEPc with a shift-and-invert transform about the target n0 and a
// MUMPS LU.  Here the same rows are assembled straight into the blocks of a
// block-tridiagonal matrix: the plane is cut into lines (rows of constant y,
// or columns of constant x, whichever are shorter), every unknown of a line
// couples only to its own line and the two lines beside it, so A - n0 B is
// block tridiagonal with blocks of 6 L (L = the line length), each row with
// at most one entry in the previous and one in the next line.  The caller
// (emopt_b200/modes.py) factors it by block cyclic reduction -- batched
// inverses of the lines eliminated at each level, and dense corrections on
// the 2L x 2L coupling blocks -- and one application of (A - n0 B)^-1 is a
// reduction and a back-substitution over the levels, each level one batched
// matrix-vector product over the inverted blocks of its lines (HBM-bound:
// every inverted block is read once per application, the reduction reading
// only the rows the neighbouring lines couple to).
//
// Vectors on the device are in line order: index (l * 6 + c) * L + p for
// line l, component c (Ex Ey Ez Hx Hy Hz) and position p along the line.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/emopt_fdtd.h"

namespace modes {

struct C2 {
    double x, y;
};
__device__ __forceinline__ C2 c2(double a, double b) { return {a, b}; }
__device__ __forceinline__ C2 operator+(C2 a, C2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ C2 operator-(C2 a, C2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ C2 operator*(C2 a, C2 b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ C2 operator*(double s, C2 a) { return {s * a.x, s * a.y}; }
__device__ __forceinline__ C2 ld2(const double* p) { return {p[0], p[1]}; }
__device__ __forceinline__ void st2(double* p, C2 v) { p[0] = v.x; p[1] = v.y; }
__device__ __forceinline__ C2 times_i(C2 a) { return {-a.y, a.x}; }

// One row of A (emopt/modes.py:1361-1585): at most six entries, each a
// component and grid point with its coefficient; assignments replace an
// earlier entry of the same column, as the reference's A[I, J] = v does.
struct Row {
    int c[6], y[6], x[6];
    C2 v[6];
    int n;
    __device__ void set(int cc, int yy, int xx, C2 val) {
        for (int q = 0; q < n; q++)
            if (c[q] == cc && y[q] == yy && x[q] == xx) { v[q] = val; return; }
        c[n] = cc; y[n] = yy; x[n] = xx; v[n] = val; n++;
    }
};

struct Planes {
    const double* p[6];   // eps_x eps_y eps_z mu_x mu_y mu_z, complex [M][N]
};

// Row `blk` (the equation block: 0..5) at grid point (y, x).  bc0, bc1: the
// boundary letters of the plane's first (x) and second (y) axes.
__device__ void mode_row(Row& r, int blk, int y, int x, int M, int N, double odx, double ody,
                         const Planes& P, char bc0, char bc1) {
    r.n = 0;
    const long long q = (long long)y * N + x;
    auto coef = [&](int w) { return ld2(P.p[w] + 2 * q); };
    const C2 zero = c2(0, 0);
    switch (blk) {
    case 0:   // Ex row: d/dy Hz + i eps_x Ex = n (i d) Hy
        if (y > 0) r.set(5, y - 1, x, c2(-ody, 0));
        r.set(5, y, x, c2(ody, 0));
        r.set(0, y, x, times_i(coef(0)));
        if (y == 0) {
            if (bc1 == '0') r.set(0, y, x, zero);
            else if (bc1 == 'E') r.set(5, y, x, c2(2 * ody, 0));
            else if (bc1 == 'H') { r.set(5, y, x, zero); r.set(0, y, x, zero); }
        }
        break;
    case 1:   // Ey row
        if (x > 0) r.set(5, y, x - 1, c2(odx, 0));
        r.set(5, y, x, c2(-odx, 0));
        r.set(1, y, x, times_i(coef(1)));
        if (x == 0) {
            if (bc0 == '0') r.set(1, y, x, zero);
            else if (bc0 == 'E') r.set(5, y, x, c2(-2 * odx, 0));
            else if (bc0 == 'H') r.set(5, y, x, zero);
        }
        break;
    case 2:   // Ez row (no B entry)
        r.set(1, y, x, c2(-odx, 0));
        if (x < N - 1) r.set(1, y, x + 1, c2(odx, 0));
        r.set(0, y, x, c2(ody, 0));
        if (y < M - 1) r.set(0, y + 1, x, c2(-ody, 0));
        r.set(5, y, x, -1.0 * times_i(coef(5)));
        if (x == 0 && bc0 == '0') r.set(1, y, x, zero);
        if (y == 0 && (bc1 == '0' || bc1 == 'H')) r.set(0, y, x, zero);
        break;
    case 3:   // Hx row
        r.set(2, y, x, c2(-ody, 0));
        if (y < M - 1) r.set(2, y + 1, x, c2(ody, 0));
        r.set(3, y, x, -1.0 * times_i(coef(3)));
        if (x == 0 && bc0 == '0') r.set(3, y, x, zero);
        if (y == 0 && (bc1 == '0' || bc1 == 'H')) r.set(2, y, x, zero);
        break;
    case 4:   // Hy row
        r.set(2, y, x, c2(odx, 0));
        if (x < N - 1) r.set(2, y, x + 1, c2(-odx, 0));
        r.set(4, y, x, -1.0 * times_i(coef(4)));
        if (x == 0 && bc0 == '0') r.set(2, y, x, zero);
        if (y == 0 && (bc1 == '0' || bc1 == 'H')) r.set(4, y, x, zero);
        break;
    default:  // Hz row (no B entry)
        if (x > 0) r.set(4, y, x - 1, c2(-odx, 0));
        r.set(4, y, x, c2(odx, 0));
        if (y > 0) r.set(3, y - 1, x, c2(ody, 0));
        r.set(3, y, x, c2(-ody, 0));
        r.set(2, y, x, times_i(coef(2)));
        if (x == 0) {
            if (bc0 == '0') { r.set(3, y, x, zero); if (y > 0) r.set(3, y - 1, x, zero); }
            else if (bc0 == 'E') r.set(4, y, x, c2(2 * odx, 0));
            else if (bc0 == 'H') r.set(4, y, x, zero);
        }
        if (y == 0) {
            if (bc1 == '0') { r.set(4, y, x, zero); if (x > 0) r.set(4, y, x - 1, zero); }
            else if (bc1 == 'E') r.set(3, y, x, c2(-2 * ody, 0));
            else if (bc1 == 'H') { r.set(3, y, x, zero); r.set(4, y, x, zero); if (x > 0) r.set(4, y, x - 1, zero); }
        }
        break;
    }
}

// B: one entry per row of the Ex, Ey, Hx, Hy blocks, at the same grid point.
__device__ __forceinline__ int b_col(int blk) { return blk == 0 ? 4 : blk == 1 ? 3 : blk == 3 ? 1 : blk == 4 ? 0 : -1; }
__device__ __forceinline__ double b_sign(int blk) { return (blk == 0 || blk == 3) ? 1.0 : -1.0; }

struct Lines {
    int M, N, L, NL, nb;
    int sweep_y;           // lines are rows of constant y (else columns of constant x)
    __device__ void grid_point(int l, int p, int& y, int& x) const {
        if (sweep_y) { y = l; x = p; } else { y = p; x = l; }
    }
    __device__ void line_of(int y, int x, int& l, int& p) const {
        if (sweep_y) { l = y; p = x; } else { l = x; p = y; }
    }
};

// D_l (dense, [nb][nb], zeroed by the caller) and the couplings to the lines
// before and after: pcol/pval (column in line l-1, -1 if none), ncol/nval.
__global__ void k_assemble(Lines G, double odx, double ody, double dir, C2 sigma, Planes P, char bc0,
                           char bc1, double* D, int* pcol, double* pval, int* ncol, double* nval) {
    const int l = blockIdx.y;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < G.nb; r += gridDim.x * blockDim.x) {
        const int blk = r / G.L, p = r % G.L;
        int y, x;
        G.grid_point(l, p, y, x);
        Row row;
        mode_row(row, blk, y, x, G.M, G.N, odx, ody, P, bc0, bc1);
        double* Dr = D + 2 * ((long long)l * G.nb * G.nb + (long long)r * G.nb);
        const long long cr = (long long)l * G.nb + r;
        pcol[cr] = -1; ncol[cr] = -1;
        st2(pval + 2 * cr, c2(0, 0)); st2(nval + 2 * cr, c2(0, 0));
        for (int q = 0; q < row.n; q++) {
            int ln, pn;
            G.line_of(row.y[q], row.x[q], ln, pn);
            const int col = row.c[q] * G.L + pn;
            if (ln == l) {
                st2(Dr + 2 * col, ld2(Dr + 2 * col) + row.v[q]);
            } else if (ln == l - 1) {
                pcol[cr] = col; st2(pval + 2 * cr, row.v[q]);
            } else {
                ncol[cr] = col; st2(nval + 2 * cr, row.v[q]);
            }
        }
        const int bc = b_col(blk);
        if (bc >= 0) {   // - sigma * B[r, col]: B = i d (sign) at the same point
            const C2 b = c2(0, b_sign(blk) * dir);
            const int col = bc * G.L + p;
            st2(Dr + 2 * col, ld2(Dr + 2 * col) - sigma * b);
        }
    }
}

// out = B v (line order).
__global__ void k_bmul(Lines G, double dir, const double* v, double* out) {
    const long long n = (long long)G.NL * G.nb;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(t / G.nb), r = (int)(t % G.nb);
        const int blk = r / G.L, p = r % G.L;
        const int bc = b_col(blk);
        C2 o = c2(0, 0);
        if (bc >= 0) o = c2(0, b_sign(blk) * dir) * ld2(v + 2 * ((long long)l * G.nb + bc * G.L + p));
        st2(out + 2 * t, o);
    }
}

// Batched over lines: for each line l = lines[z] (blockIdx.z),
//   out_l[a] += sum_b W_l[a][b] (rhs_l[b] - corr_l[b])
// for the rows a listed in `rows` (all nb rows when rows is null), over one
// tile of GEMV_COLS columns (blockIdx.x); corr may be null.  The tile of the
// vector is staged in shared memory; a CTA covers 8 rows (a warp each), every
// lane issues its GEMV_COLS/32 loads of the row before it reduces, and the
// partial sums of the column tiles meet in `out` (zeroed by the caller) by
// atomic adds.
constexpr int GEMV_COLS = 256;

__global__ void __launch_bounds__(256) k_lines_gemv(int nb, const double* W, const int* lines,
                                                    const int* rows, int nrows, const double* rhs,
                                                    const double* corr, double* out) {
    __shared__ double2 vs[GEMV_COLS];
    const long long line = lines[blockIdx.z];
    const double* Wl = W + 2 * line * nb * nb;
    const double* rl = rhs + 2 * line * nb;
    const double* cl = corr ? corr + 2 * line * nb : nullptr;
    double* ol = out + 2 * line * nb;
    const int c0 = blockIdx.x * GEMV_COLS;
    const int ncols = min(GEMV_COLS, nb - c0);
    for (int t = threadIdx.x; t < ncols; t += blockDim.x) {
        C2 v = ld2(rl + 2 * (c0 + t));
        if (cl) v = v - ld2(cl + 2 * (c0 + t));
        vs[t] = make_double2(v.x, v.y);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int q = blockIdx.y * 8 + (threadIdx.x >> 5); q < nrows; q += gridDim.y * 8) {
        const int a = rows ? rows[q] : q;
        const double2* Wa = reinterpret_cast<const double2*>(Wl + 2 * ((long long)a * nb + c0));
        double2 w[GEMV_COLS / 32];
#pragma unroll
        for (int e = 0; e < GEMV_COLS / 32; e++) {
            const int t = lane + 32 * e;
            w[e] = t < ncols ? Wa[t] : make_double2(0.0, 0.0);
        }
        double sr = 0, si = 0;
#pragma unroll
        for (int e = 0; e < GEMV_COLS / 32; e++) {
            const int t = lane + 32 * e;
            if (t < ncols) {
                const double2 v = vs[t];
                sr = fma(w[e].x, v.x, fma(-w[e].y, v.y, sr));
                si = fma(w[e].x, v.y, fma(w[e].y, v.x, si));
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        if (lane == 0) {
            atomicAdd(ol + 2 * a, sr);
            atomicAdd(ol + 2 * a + 1, si);
        }
    }
}

// Couplings between lines, batched: for z < nlines,
//   dst[lines[z]][rows[i]] += sign * sum_j C[z][i][j] src[nbrs[z]][cols[j]]
// (C: nlines x R x Q, dense).  A warp per (z, i); lanes walk j.  Every
// (line, row) pair is written by one warp only.
__global__ void __launch_bounds__(256) k_couple(int nb, int R, int Q, const double* C, const int* lines,
                                                const int* nbrs, const int* rows, const int* cols,
                                                const double* src, double* dst, double sign) {
    const int z = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (i >= R) return;
    const double* Ci = C + 2 * ((long long)z * R + i) * Q;
    const double* s = src + 2 * (long long)nbrs[z] * nb;
    double sr = 0, si = 0;
    for (int j = lane; j < Q; j += 32) {
        const C2 c = ld2(Ci + 2 * j), v = ld2(s + 2 * cols[j]);
        sr = fma(c.x, v.x, fma(-c.y, v.y, sr));
        si = fma(c.x, v.y, fma(c.y, v.x, si));
    }
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
        double* d = dst + 2 * ((long long)lines[z] * nb + rows[i]);
        d[0] += sign * sr;
        d[1] += sign * si;
    }
}

// The mode's current sources on the plane (emopt/modes.py:2144-2296), raw
// solver components in, [M][N] planes out (solver order Jx Jy Jz Mx My Mz).
// f: the six raw field planes; s: 1/sqrt(S) of the power normalisation.
__global__ void k_source(int M, int N, const double* f, C2 s, C2 ekz, double dxn, double dyn, double dzn,
                         const double* eps, const double* mu05, const double* mu50, char bc0, char bc1,
                         double* out) {
    const long long MN = (long long)M * N;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < MN; t += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(t / N), x = (int)(t % N);
        auto F = [&](int c, int yy, int xx) {
            if (yy < 0 || yy >= M || xx < 0 || xx >= N) return c2(0, 0);
            return s * ld2(f + 2 * (c * MN + (long long)yy * N + xx));
        };
        const C2 Ex = F(0, y, x), Ey = F(1, y, x), Ez = F(2, y, x);
        const C2 Ez_y1 = F(2, y + 1, x), Ez_x1 = F(2, y, x + 1);
        const C2 Hx = F(3, y, x), Hy = F(4, y, x);
        C2 Hx_m = F(3, y - 1, x), Hy_m = F(4, y, x - 1);
        if (y == 0) Hx_m = bc1 == 'E' ? -1.0 * F(3, 0, x) : bc1 == 'H' ? F(3, 0, x) : c2(0, 0);
        if (x == 0) Hy_m = bc0 == 'E' ? -1.0 * F(4, y, 0) : bc0 == 'H' ? F(4, y, 0) : c2(0, 0);
        const C2 e = ld2(eps + 2 * t), m05 = ld2(mu05 + 2 * t), m50 = ld2(mu50 + 2 * t);
        // accumulated in the reference's order
        C2 Jx = c2(0, 0), Jy = c2(0, 0), Jz = c2(0, 0), Mx = c2(0, 0), My = c2(0, 0);
        My = My + (1.0 / dzn) * (Ex * ekz);
        Mx = Mx + (1.0 / dzn) * (-1.0 * Ey * ekz);
        Jz = Jz + times_i(e) * Ez;
        Mx = Mx + (1.0 / dyn) * (Ez_y1 - Ez);
        My = My + (1.0 / dxn) * (-1.0 * (Ez_x1 - Ez));
        Jy = Jy + (1.0 / dzn) * Hx;
        Jz = Jz + (1.0 / dyn) * (-1.0 * (Hx - Hx_m));
        Mx = Mx + -1.0 * times_i(m05) * Hx;
        Jx = Jx + (1.0 / dzn) * (-1.0 * Hy);
        Jz = Jz + (1.0 / dxn) * (Hy - Hy_m);
        My = My + -1.0 * times_i(m50) * Hy;
        st2(out + 2 * (0 * MN + t), Jx);
        st2(out + 2 * (1 * MN + t), Jy);
        st2(out + 2 * (2 * MN + t), Jz);
        st2(out + 2 * (3 * MN + t), Mx);
        st2(out + 2 * (4 * MN + t), My);
        st2(out + 2 * (5 * MN + t), c2(0, 0));
    }
}

thread_local char g_msg[256];

int fail(int code, const char* what) {
    std::snprintf(g_msg, sizeof(g_msg), "%s", what);
    return code;
}

int cuda_fail(cudaError_t e, const char* where) {
    std::snprintf(g_msg, sizeof(g_msg), "%s: %s", where, cudaGetErrorString(e));
    return FDTD_ERR_CUDA;
}

bool lines_ok(const FDTDModeLines* g, Lines& G) {
    if (!g || g->M < 1 || g->N < 1) return false;
    G.M = g->M; G.N = g->N; G.sweep_y = g->sweep_y ? 1 : 0;
    G.L = G.sweep_y ? g->N : g->M;
    G.NL = G.sweep_y ? g->M : g->N;
    G.nb = 6 * G.L;
    return true;
}

}  // namespace modes

using namespace modes;

#define MCK(call, where)                                               \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, where);            \
    } while (0)

extern "C" {

const char* FDTD_mode_last_error(void) { return g_msg; }

int FDTD_mode_assemble(const FDTDModeLines* g, int device, void* stream, double odx, double ody, double dir,
                       double sigma_re, double sigma_im, const double* const* planes, const char* bc,
                       double* D, int* pcol, double* pval, int* ncol, double* nval) {
    Lines G;
    if (!lines_ok(g, G) || !planes || !bc || !D || !pcol || !pval || !ncol || !nval)
        return fail(FDTD_ERR_ARG, "FDTD_mode_assemble: bad arguments");
    if (G.NL > 65535) return fail(FDTD_ERR_ARG, "FDTD_mode_assemble: more than 65535 lines");
    MCK(cudaSetDevice(device), "FDTD_mode_assemble");
    Planes P;
    for (int q = 0; q < 6; q++) {
        if (!planes[q]) return fail(FDTD_ERR_ARG, "FDTD_mode_assemble: a material plane is null");
        P.p[q] = planes[q];
    }
    cudaStream_t st = (cudaStream_t)stream;
    MCK(cudaMemsetAsync(D, 0, sizeof(double) * 2 * (size_t)G.NL * G.nb * G.nb, st), "FDTD_mode_assemble");
    dim3 grid((G.nb + 127) / 128, G.NL);
    k_assemble<<<grid, 128, 0, st>>>(G, odx, ody, dir, {sigma_re, sigma_im}, P, bc[0], bc[1], D, pcol, pval,
                                      ncol, nval);
    MCK(cudaGetLastError(), "FDTD_mode_assemble");
    return FDTD_OK;
}

int FDTD_mode_bmul(const FDTDModeLines* g, int device, void* stream, double dir, const double* v,
                   double* out) {
    Lines G;
    if (!lines_ok(g, G) || !v || !out) return fail(FDTD_ERR_ARG, "FDTD_mode_bmul: bad arguments");
    MCK(cudaSetDevice(device), "FDTD_mode_bmul");
    const long long n = (long long)G.NL * G.nb;
    k_bmul<<<(unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, (cudaStream_t)stream>>>(
        G, dir, v, out);
    MCK(cudaGetLastError(), "FDTD_mode_bmul");
    return FDTD_OK;
}

int FDTD_mode_lines_gemv(int nb, int device, void* stream, const double* W, const int* lines, int nlines,
                         const int* rows, int nrows, const double* rhs, const double* corr, double* out) {
    if (nb < 1 || !W || !lines || nlines < 1 || nlines > 65535 || !rhs || !out || (rows && nrows < 1) ||
        (!rows && nrows != nb))
        return fail(FDTD_ERR_ARG, "FDTD_mode_lines_gemv: bad arguments");
    MCK(cudaSetDevice(device), "FDTD_mode_lines_gemv");
    const unsigned tiles = (unsigned)((nb + GEMV_COLS - 1) / GEMV_COLS);
    dim3 grid(tiles, (unsigned)((nrows + 7) / 8), (unsigned)nlines);
    k_lines_gemv<<<grid, 256, 0, (cudaStream_t)stream>>>(nb, W, lines, rows, nrows, rhs, corr, out);
    MCK(cudaGetLastError(), "FDTD_mode_lines_gemv");
    return FDTD_OK;
}

int FDTD_mode_couple(int nb, int device, void* stream, int nlines, int R, int Q, const double* C,
                     const int* lines, const int* nbrs, const int* rows, const int* cols, const double* src,
                     double* dst, double sign) {
    if (nb < 1 || nlines < 1 || nlines > 65535 || R < 1 || Q < 1 || !C || !lines || !nbrs || !rows || !cols ||
        !src || !dst)
        return fail(FDTD_ERR_ARG, "FDTD_mode_couple: bad arguments");
    MCK(cudaSetDevice(device), "FDTD_mode_couple");
    dim3 grid((unsigned)((R + 7) / 8), (unsigned)nlines);
    k_couple<<<grid, 256, 0, (cudaStream_t)stream>>>(nb, R, Q, C, lines, nbrs, rows, cols, src, dst, sign);
    MCK(cudaGetLastError(), "FDTD_mode_couple");
    return FDTD_OK;
}

int FDTD_mode_source(int device, void* stream, int M, int N, const double* fields, double s_re, double s_im,
                     double ekz_re, double ekz_im, double dxn, double dyn, double dzn, const double* eps,
                     const double* mu05, const double* mu50, const char* bc, double* out) {
    if (M < 1 || N < 1 || !fields || !eps || !mu05 || !mu50 || !bc || !out)
        return fail(FDTD_ERR_ARG, "FDTD_mode_source: bad arguments");
    MCK(cudaSetDevice(device), "FDTD_mode_source");
    const long long MN = (long long)M * N;
    const unsigned blocks = (unsigned)((MN + 255) / 256 < 4096 ? (MN + 255) / 256 : 4096);
    k_source<<<blocks, 256, 0, (cudaStream_t)stream>>>(M, N, fields, {s_re, s_im}, {ekz_re, ekz_im}, dxn, dyn,
                                                       dzn, eps, mu05, mu50, bc[0], bc[1], out);
    MCK(cudaGetLastError(), "FDTD_mode_source");
    return FDTD_OK;
}

}  // extern "C"
