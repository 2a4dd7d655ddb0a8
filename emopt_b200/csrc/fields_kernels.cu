// fields_kernels.cu -- field access around a solve on the device: the
// interpolation of a field component onto the Ez grid (emopt/fdtd.py:1401-1553,
// FDTD.get_field_interp), its exact transpose, the reference's adjoint-source
// mapping interpolated_dFdx_3D (emopt/fomutils.py:1282-1426) and the source
// power through six planes (emopt/fdtd.py:1555-1667).
//
// Interpolation geometry.  The reference pads the block it reads (the
// requested domain grown by one cell where the grid allows, clipped to the
// grid) with one zero cell on every side, fills the pad column k = 0 (row
// j = 0) with the mirrored first column (row) when the block starts at a
// symmetric min face ('E': negated, 'H': as is), averages neighbouring samples
// in place and crops the requested domain out.  Here a block of ni x nj x nk
// cells starts at (ri1, rj1, rk1) of an array with row length NX and plane
// size NX*NY; padded coordinates run 0 .. n+1; output cell (oi, oj, ok) sits
// at padded (1 + di + oi, 1 + dj + oj, 1 + dk + ok).  The additions follow the
// reference's order, so the device and host values agree to the last bit.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>

#include "../../include/emopt_fdtd.h"
#include "kernels.h"

namespace fdtdb {
namespace {

struct Geom {
    int ri1, rj1, rk1;   // block origin in the array
    int ni, nj, nk;      // block extents
    int di, dj, dk;      // crop offsets
    int oi, oj, ok;      // output extents
    int NX, NY, NZ;      // array row length, rows per plane, planes
    int sx, sy;          // mirrored pad at a symmetric min face: -1 ('E'), +1 ('H'), 0
};

__device__ __forceinline__ c128 cz() { c128 r; r.real = 0; r.imag = 0; return r; }
__device__ __forceinline__ c128 cadd(c128 a, c128 b) { a.real += b.real; a.imag += b.imag; return a; }
__device__ __forceinline__ c128 cscale(c128 a, double s) { a.real *= s; a.imag *= s; return a; }
__device__ __forceinline__ c128 cdiv(c128 a, double s) { a.real /= s; a.imag /= s; return a; }

// Block value at padded coordinates (a, b, c), zero on the pad.
__device__ __forceinline__ c128 base(const c128* f, const Geom& g, int a, int b, int c) {
    if (a < 1 || a > g.ni || b < 1 || b > g.nj || c < 1 || c > g.nk) return cz();
    return f[((long long)(g.ri1 + a - 1) * g.NY + (g.rj1 + b - 1)) * g.NX + (g.rk1 + c - 1)];
}

// Which pads a component mirrors: x for Ex, Hy, Hz; y for Ey, Hx, Hz.
__device__ __forceinline__ bool mirrors_x(int comp) { return comp == 0 || comp == 4 || comp == 5; }
__device__ __forceinline__ bool mirrors_y(int comp) { return comp == 1 || comp == 3 || comp == 5; }

// Padded value with the mirrored pads (x first, then y, as the reference).
__device__ __forceinline__ c128 pval(const c128* f, const Geom& g, int comp, int a, int b, int c) {
    const int sx = mirrors_x(comp) ? g.sx : 0, sy = mirrors_y(comp) ? g.sy : 0;
    if (b == 0 && sy) {
        if (c == 0) return sx ? cscale(base(f, g, a, 1, 1), (double)(sy * sx)) : cz();
        return cscale(base(f, g, a, 1, c), (double)sy);
    }
    if (c == 0 && sx) return cscale(base(f, g, a, b, 1), (double)sx);
    return base(f, g, a, b, c);
}

// Interpolated value at padded coordinates (a, b, c).
__device__ c128 interp_at(const c128* f, const Geom& g, int comp, int a, int b, int c) {
    c128 v = pval(f, g, comp, a, b, c);
    switch (comp) {
        case 0:   // Ex: (i, k), (i, k-1), (i+1, k), (i+1, k-1)
            if (a >= 1 && a <= g.ni && c >= 1 && c <= g.nk) {
                v = cadd(v, pval(f, g, comp, a, b, c - 1));
                v = cadd(v, pval(f, g, comp, a + 1, b, c));
                v = cadd(v, pval(f, g, comp, a + 1, b, c - 1));
            }
            return cdiv(v, 4.0);
        case 1:   // Ey: (i, j), (i, j-1), (i+1, j), (i+1, j-1)
            if (a >= 1 && a <= g.ni && b >= 1 && b <= g.nj) {
                v = cadd(v, pval(f, g, comp, a, b - 1, c));
                v = cadd(v, pval(f, g, comp, a + 1, b, c));
                v = cadd(v, pval(f, g, comp, a + 1, b - 1, c));
            }
            return cdiv(v, 4.0);
        case 2:   // Ez: on its own grid
            return v;
        case 3:   // Hx: (j), (j-1)
            if (b >= 1) v = cadd(v, pval(f, g, comp, a, b - 1, c));
            return cdiv(v, 2.0);
        case 4:   // Hy: (k), (k-1)
            if (c >= 1) v = cadd(v, pval(f, g, comp, a, b, c - 1));
            return cdiv(v, 2.0);
        default:  // Hz: the eight corners, in the reference's order
            if (a <= g.ni && b >= 1 && c >= 1) {
                v = cadd(v, pval(f, g, comp, a, b, c - 1));
                v = cadd(v, pval(f, g, comp, a, b - 1, c));
                v = cadd(v, pval(f, g, comp, a, b - 1, c - 1));
                v = cadd(v, pval(f, g, comp, a + 1, b, c));
                v = cadd(v, pval(f, g, comp, a + 1, b, c - 1));
                v = cadd(v, pval(f, g, comp, a + 1, b - 1, c));
                v = cadd(v, pval(f, g, comp, a + 1, b - 1, c - 1));
            }
            return cdiv(v, 8.0);
    }
}

__global__ void k_interp(const c128* f, Geom g, int comp, c128* out) {
    const long long n = (long long)g.oi * g.oj * g.ok;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int ok = (int)(q % g.ok);
        const long long r = q / g.ok;
        const int oj = (int)(r % g.oj), oi = (int)(r / g.oj);
        out[q] = interp_at(f, g, comp, 1 + g.di + oi, 1 + g.dj + oj, 1 + g.dk + ok);
    }
}

// Cotangent of the output at padded coordinates (a, b, c), zero outside it.
__device__ __forceinline__ c128 gout(const c128* go, const Geom& g, int a, int b, int c) {
    const int oi = a - 1 - g.di, oj = b - 1 - g.dj, ok = c - 1 - g.dk;
    if (oi < 0 || oi >= g.oi || oj < 0 || oj >= g.oj || ok < 0 || ok >= g.ok) return cz();
    return go[((long long)oi * g.oj + oj) * g.ok + ok];
}

// Transpose of interp_at onto the padded value (a, b, c): every output cell
// whose average reads (a, b, c), with its weight.
__device__ c128 dpad(const c128* go, const Geom& g, int comp, int a, int b, int c) {
    c128 s = gout(go, g, a, b, c);
    auto in_ex = [&](int A, int C) { return A >= 1 && A <= g.ni && C >= 1 && C <= g.nk; };
    auto in_ey = [&](int A, int B) { return A >= 1 && A <= g.ni && B >= 1 && B <= g.nj; };
    switch (comp) {
        case 0:
            if (in_ex(a, c + 1)) s = cadd(s, gout(go, g, a, b, c + 1));
            if (in_ex(a - 1, c)) s = cadd(s, gout(go, g, a - 1, b, c));
            if (in_ex(a - 1, c + 1)) s = cadd(s, gout(go, g, a - 1, b, c + 1));
            return cdiv(s, 4.0);
        case 1:
            if (in_ey(a, b + 1)) s = cadd(s, gout(go, g, a, b + 1, c));
            if (in_ey(a - 1, b)) s = cadd(s, gout(go, g, a - 1, b, c));
            if (in_ey(a - 1, b + 1)) s = cadd(s, gout(go, g, a - 1, b + 1, c));
            return cdiv(s, 4.0);
        case 2:
            return s;
        case 3:
            if (b + 1 >= 1) s = cadd(s, gout(go, g, a, b + 1, c));
            return cdiv(s, 2.0);
        case 4:
            if (c + 1 >= 1) s = cadd(s, gout(go, g, a, b, c + 1));
            return cdiv(s, 2.0);
        default: {
            // output (A, B, C) reads (A + da, B - db, C - dc), da, db, dc in {0, 1},
            // when A <= ni, B >= 1, C >= 1 (otherwise only its own cell)
            c128 t = cz();
            for (int da = 0; da <= 1; da++)
                for (int db = 0; db <= 1; db++)
                    for (int dc = 0; dc <= 1; dc++) {
                        if (!da && !db && !dc) continue;
                        const int A = a - da, B = b + db, C = c + dc;
                        if (A <= g.ni && B >= 1 && C >= 1) t = cadd(t, gout(go, g, A, B, C));
                    }
            // the own-cell term counts once whatever the range
            return cdiv(cadd(s, t), 8.0);
        }
    }
}

__global__ void k_interp_T(const c128* go, Geom g, int comp, c128* graw) {
    const long long n = (long long)g.ni * g.nj * g.nk;
    const int sx = mirrors_x(comp) ? g.sx : 0, sy = mirrors_y(comp) ? g.sy : 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(q % g.nk);
        const long long r = q / g.nk;
        const int y = (int)(r % g.nj), x = (int)(r / g.nj);
        const int A = x + 1, B = y + 1, C = z + 1;
        c128 s = dpad(go, g, comp, A, B, C);
        if (C == 1 && sx) s = cadd(s, cscale(dpad(go, g, comp, A, B, 0), (double)sx));
        if (B == 1 && sy) s = cadd(s, cscale(dpad(go, g, comp, A, 0, C), (double)sy));
        if (B == 1 && C == 1 && sx && sy) s = cadd(s, cscale(dpad(go, g, comp, A, 0, 0), (double)(sx * sy)));
        graw[q] = s;
    }
}

// interpolated_dFdx_3D of one component (emopt/fomutils.py:1282-1426):
// the derivative v = w dF on the domain (nz x ny x nx) is added to a
// (nz+2) x (ny+2) x (nx+2) array at the taps of the component, the
// mirrored-sample terms are added at a symmetric min face, and the block
// [1:, 0:-1, 0:-1] of that array is returned.  qx: 0 none, 1 the 'H' rule on
// the x face for Ex, 2 the 'E' rule (applied on the y face, as the
// reference); qy: the sign of the y-face rule for Ey, Hx, Hz (0 none).
__device__ __forceinline__ c128 dfv(const c128* dF, int nz, int ny, int nx, double w, int i, int j, int k) {
    if (i < 0 || i >= nz || j < 0 || j >= ny || k < 0 || k >= nx) return cz();
    return cscale(dF[((long long)i * ny + j) * nx + k], w);
}

__global__ void k_dfdx_interp(const c128* dF, int nz, int ny, int nx, int comp, int qx, int qy,
                              c128* out) {
    const int Oz = nz + 1, Oy = ny + 1, Ox = nx + 1;
    const long long n = (long long)Oz * Oy * Ox;
    // taps (dz, dy, dx) in the reference's order and the weight
    int tz[8], ty[8], tx[8], nt;
    double w;
    switch (comp) {
        case 0: nt = 4; w = 0.25;
            tz[0] = 0; ty[0] = 0; tx[0] = 0; tz[1] = 0; ty[1] = 0; tx[1] = -1;
            tz[2] = 1; ty[2] = 0; tx[2] = 0; tz[3] = 1; ty[3] = 0; tx[3] = -1; break;
        case 1: nt = 4; w = 0.25;
            tz[0] = 0; ty[0] = 0; tx[0] = 0; tz[1] = 0; ty[1] = -1; tx[1] = 0;
            tz[2] = 1; ty[2] = 0; tx[2] = 0; tz[3] = 1; ty[3] = -1; tx[3] = 0; break;
        case 2: nt = 1; w = 1.0; tz[0] = 0; ty[0] = 0; tx[0] = 0; break;
        case 3: nt = 2; w = 0.5;
            tz[0] = 0; ty[0] = 0; tx[0] = 0; tz[1] = 0; ty[1] = -1; tx[1] = 0; break;
        case 4: nt = 2; w = 0.5;
            tz[0] = 0; ty[0] = 0; tx[0] = 0; tz[1] = 0; ty[1] = 0; tx[1] = -1; break;
        default: nt = 8; w = 0.125;
            for (int q = 0; q < 8; q++) { tz[q] = q >> 2; ty[q] = (q >> 1) & 1 ? -1 : 0; tx[q] = q & 1 ? -1 : 0; }
            break;
    }
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int C = (int)(q % Ox);
        const long long r = q / Ox;
        const int B = (int)(r % Oy), A = (int)(r / Oy) + 1;   // array row A = 1 + output row
        c128 s = cz();
        if (comp == 2) {
            // Ez: the interior of the array is dF itself
            if (A >= 1 && A <= nz && B >= 1 && B <= ny && C >= 1 && C <= nx)
                s = dF[((long long)(A - 1) * ny + (B - 1)) * nx + (C - 1)];
            out[q] = s;
            continue;
        }
        for (int t = 0; t < nt; t++)
            s = cadd(s, dfv(dF, nz, ny, nx, w, A - 1 - tz[t], B - 1 - ty[t], C - 1 - tx[t]));
        if (comp == 0 && qx == 1 && C == 1)
            for (int dz = 0; dz <= 1; dz++) s = cadd(s, dfv(dF, nz, ny, nx, w, A - 1 - dz, B - 1, 0));
        if (comp == 0 && qx == 2 && B == 1)
            for (int dz = 0; dz <= 1; dz++)
                s = cadd(s, cscale(dfv(dF, nz, ny, nx, w, A - 1 - dz, 0, C - 1), -1.0));
        if ((comp == 1 || comp == 3 || comp == 5) && qy != 0 && B == 1)
            for (int t = 0; t < nt; t++)
                if (ty[t] == 0)
                    s = cadd(s, cscale(dfv(dF, nz, ny, nx, w, A - 1 - tz[t], 0, C - 1 - tx[t]), (double)qy));
        out[q] = s;
    }
}

// Source power: per plane p, the sum over its cells of
// Re(E1 conj(H2) - E2 conj(H1)) = Re(E x H*) . n with (E1, H2, E2, H1) =
// (Ey, Hz, Ez, Hy) for a plane normal to x, (Ez, Hx, Ex, Hz) for y, (Ex, Hy,
// Ey, Hx) for z (kFluxComps), every component interpolated as above.  One CTA sums a stretch of cells (warp
// shuffles, then shared memory, in a fixed order) into partial[p][block];
// k_sum_partials adds the partials of each plane in order.
struct PlaneSet {
    const c128* f[6][6];   // per plane: Ex Ey Ez Hx Hy Hz blocks
    Geom g[6];
    int axis[6];
    int n;
};

constexpr int kPowThreads = 256;

// (E1, H2, E2, H1) of the flux through a plane normal to x, y, z
__constant__ int kFluxComps[3][4] = {{1, 5, 2, 4}, {2, 3, 0, 5}, {0, 4, 1, 3}};

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[kPowThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kPowThreads / 32; w++) s += red[w];
    __syncthreads();
    return s;
}

__global__ void __launch_bounds__(kPowThreads) k_power_partials(PlaneSet ps, double* partial, int nblk) {
    const int p = blockIdx.y;
    const Geom& g = ps.g[p];
    const int ax = ps.axis[p];
    const int c1 = kFluxComps[ax][0], c2 = kFluxComps[ax][1], c3 = kFluxComps[ax][2], c4 = kFluxComps[ax][3];
    const long long n = (long long)g.oi * g.oj * g.ok;
    double acc = 0;
    for (long long q = blockIdx.x * (long long)kPowThreads + threadIdx.x; q < n;
         q += (long long)nblk * kPowThreads) {
        const int ok = (int)(q % g.ok);
        const long long r = q / g.ok;
        const int oj = (int)(r % g.oj), oi = (int)(r / g.oj);
        const int a = 1 + g.di + oi, b = 1 + g.dj + oj, c = 1 + g.dk + ok;
        const c128 e1 = interp_at(ps.f[p][c1], g, c1, a, b, c), h2 = interp_at(ps.f[p][c2], g, c2, a, b, c);
        const c128 e2 = interp_at(ps.f[p][c3], g, c3, a, b, c), h1 = interp_at(ps.f[p][c4], g, c4, a, b, c);
        // Re(e1 conj(h2) - e2 conj(h1))
        acc += (e1.real * h2.real + e1.imag * h2.imag) - (e2.real * h1.real + e2.imag * h1.imag);
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) partial[p * nblk + blockIdx.x] = s;
}

__global__ void k_sum_partials(const double* partial, int nblk, double* out) {
    const int p = blockIdx.x;
    double v = 0;
    for (int q = threadIdx.x; q < nblk; q += kPowThreads) v += partial[p * nblk + q];
    const double s = block_sum(v);
    if (threadIdx.x == 0) out[p] = s;
}

int blocks_for_n(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

int fail(char* msg, int msglen, int status, const char* fmt, ...) __attribute__((format(printf, 4, 5)));
int fail(char* msg, int msglen, int status, const char* fmt, ...) {
    if (msg && msglen > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(msg, (size_t)msglen, fmt, ap);
        va_end(ap);
    }
    return status;
}

bool geom_from(const int* gi, Geom* g) {
    g->ri1 = gi[0]; g->rj1 = gi[1]; g->rk1 = gi[2];
    g->ni = gi[3]; g->nj = gi[4]; g->nk = gi[5];
    g->di = gi[6]; g->dj = gi[7]; g->dk = gi[8];
    g->oi = gi[9]; g->oj = gi[10]; g->ok = gi[11];
    g->NX = gi[12]; g->NY = gi[13]; g->NZ = gi[14];
    g->sx = gi[15]; g->sy = gi[16];
    const bool signs = g->sx >= -1 && g->sx <= 1 && g->sy >= -1 && g->sy <= 1;
    const bool ext = g->ni >= 0 && g->nj >= 0 && g->nk >= 0 && g->oi >= 0 && g->oj >= 0 && g->ok >= 0;
    const bool in = g->ri1 >= 0 && g->rj1 >= 0 && g->rk1 >= 0 && g->ri1 + g->ni <= g->NZ &&
                    g->rj1 + g->nj <= g->NY && g->rk1 + g->nk <= g->NX && g->NX > 0 && g->NY > 0;
    // every output cell reads padded cells 0 .. n+1 only
    const bool crop = g->di >= 0 && g->dj >= 0 && g->dk >= 0 && g->di + g->oi <= g->ni &&
                      g->dj + g->oj <= g->nj && g->dk + g->ok <= g->nk;
    return signs && ext && in && crop;
}

// Enter the caller's device for the call, restore the previous one after.
struct DeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int dev) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace
}  // namespace fdtdb

using fdtdb::c128;

extern "C" int FDTD_interp_field(int device, void* stream, int comp, const fdtd_complex128* raw,
                                 const int* geom, fdtd_complex128* out, char* msg, int msglen) {
    fdtdb::Geom g;
    if (comp < 0 || comp > 5 || !geom || !fdtdb::geom_from(geom, &g))
        return fdtdb::fail(msg, msglen, FDTD_ERR_ARG, "FDTD_interp_field: invalid component or geometry");
    const long long n = (long long)g.oi * g.oj * g.ok;
    if (n == 0) return FDTD_OK;   // an empty domain (null pointers allowed)
    if (!raw || !out) return fdtdb::fail(msg, msglen, FDTD_ERR_ARG, "FDTD_interp_field: null array");
    fdtdb::DeviceScope ds(device);
    if (ds.err != cudaSuccess) return fdtdb::fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_interp_field: %s", cudaGetErrorString(ds.err));
    cudaStream_t st = (cudaStream_t)stream;
    cudaGetLastError();
    fdtdb::k_interp<<<fdtdb::blocks_for_n(n), 256, 0, st>>>(reinterpret_cast<const c128*>(raw), g, comp,
                                                            reinterpret_cast<c128*>(out));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fdtdb::fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_interp_field: %s", cudaGetErrorString(e));
    return FDTD_OK;
}

extern "C" int FDTD_interp_field_T(int device, void* stream, int comp, const fdtd_complex128* gout,
                                   const int* geom, fdtd_complex128* graw, char* msg, int msglen) {
    fdtdb::Geom g;
    if (comp < 0 || comp > 5 || !geom || !fdtdb::geom_from(geom, &g))
        return fdtdb::fail(msg, msglen, FDTD_ERR_ARG, "FDTD_interp_field_T: invalid component or geometry");
    const long long n = (long long)g.ni * g.nj * g.nk;
    if (n == 0) return FDTD_OK;   // an empty block (null pointers allowed)
    // an empty output: the block's cotangent is zero (the kernel reads no gout)
    if (!graw || (!gout && (long long)g.oi * g.oj * g.ok > 0))
        return fdtdb::fail(msg, msglen, FDTD_ERR_ARG, "FDTD_interp_field_T: null array");
    fdtdb::DeviceScope ds(device);
    if (ds.err != cudaSuccess) return fdtdb::fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_interp_field_T: %s", cudaGetErrorString(ds.err));
    cudaStream_t st = (cudaStream_t)stream;
    cudaGetLastError();
    fdtdb::k_interp_T<<<fdtdb::blocks_for_n(n), 256, 0, st>>>(reinterpret_cast<const c128*>(gout), g, comp,
                                                              reinterpret_cast<c128*>(graw));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fdtdb::fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_interp_field_T: %s", cudaGetErrorString(e));
    return FDTD_OK;
}

extern "C" int FDTD_dfdx_interp(int device, void* stream, int comp, const fdtd_complex128* dF, int nx,
                                int ny, int nz, int qx, int qy, fdtd_complex128* out, char* msg,
                                int msglen) {
    if (comp < 0 || comp > 5 || !out || nx < 0 || ny < 0 || nz < 0 || qx < 0 || qx > 2 ||
        qy < -1 || qy > 1 || (!dF && (long long)nx * ny * nz > 0))
        return fdtdb::fail(msg, msglen, FDTD_ERR_ARG, "FDTD_dfdx_interp: invalid argument");
    fdtdb::DeviceScope ds(device);
    if (ds.err != cudaSuccess) return fdtdb::fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_dfdx_interp: %s", cudaGetErrorString(ds.err));
    const long long n = (long long)(nz + 1) * (ny + 1) * (nx + 1);
    cudaStream_t st = (cudaStream_t)stream;
    cudaGetLastError();
    fdtdb::k_dfdx_interp<<<fdtdb::blocks_for_n(n), 256, 0, st>>>(reinterpret_cast<const c128*>(dF), nz, ny, nx,
                                                                 comp, qx, qy, reinterpret_cast<c128*>(out));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fdtdb::fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_dfdx_interp: %s", cudaGetErrorString(e));
    return FDTD_OK;
}

extern "C" int FDTD_plane_flux(int device, void* stream, int nplanes, const fdtd_complex128* const* blocks,
                               const int* geoms, const int* axes, double* sums, char* msg, int msglen) {
    if (nplanes < 0 || nplanes > 6 || (nplanes > 0 && (!blocks || !geoms || !axes || !sums)))
        return fdtdb::fail(msg, msglen, FDTD_ERR_ARG, "FDTD_plane_flux: invalid argument");
    if (nplanes == 0) return FDTD_OK;
    fdtdb::PlaneSet ps;
    ps.n = nplanes;
    long long most = 1;
    for (int p = 0; p < nplanes; p++) {
        if (!fdtdb::geom_from(geoms + 17 * p, &ps.g[p]) || axes[p] < 0 || axes[p] > 2)
            return fdtdb::fail(msg, msglen, FDTD_ERR_ARG, "FDTD_plane_flux: plane %d has an invalid geometry", p);
        for (int c = 0; c < 6; c++) {
            ps.f[p][c] = reinterpret_cast<const c128*>(blocks[6 * p + c]);
            if (!ps.f[p][c]) return fdtdb::fail(msg, msglen, FDTD_ERR_ARG, "FDTD_plane_flux: null block");
        }
        ps.axis[p] = axes[p];
        const long long n = (long long)ps.g[p].oi * ps.g[p].oj * ps.g[p].ok;
        if (n > most) most = n;
    }
    fdtdb::DeviceScope ds(device);
    if (ds.err != cudaSuccess) return fdtdb::fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_plane_flux: %s", cudaGetErrorString(ds.err));
    cudaStream_t st = (cudaStream_t)stream;
    // partial sums and results in one small buffer of the caller's: sums
    // must hold 6 + 6 * 148 doubles (device memory)
    const int nblk = (int)std::min<long long>(148, (most + fdtdb::kPowThreads - 1) / fdtdb::kPowThreads);
    double* partial = sums + 6;
    cudaGetLastError();
    fdtdb::k_power_partials<<<dim3(nblk, nplanes), fdtdb::kPowThreads, 0, st>>>(ps, partial, nblk);
    fdtdb::k_sum_partials<<<nplanes, fdtdb::kPowThreads, 0, st>>>(partial, nblk, sums);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fdtdb::fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_plane_flux: %s", cudaGetErrorString(e));
    return FDTD_OK;
}
