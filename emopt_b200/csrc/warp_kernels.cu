// warp_kernels.cu -- fused time step on warp-independent register tiles.
//
// Each warp owns an x-y column tile and marches it up through a chunk of
// planes.  Lane l holds column k = x0 - 1 + l (x0 = 30 * tile), and every
// thread holds R rows of its column in registers: row slot q = 0 .. R+1 is
// row j = r0 - 1 + q.
//   * lane 0 and row slot 0 are the low halo: H is computed there (the E
//     update reads it at k-1 and j-1) but not stored;
//   * lane 31 and row slot R+1 only provide E (the H update reads it at k+1
//     and j+1);
//   * lanes 1..30 x rows 1..R are the 30 x R cells the warp writes.
// x neighbours come from warp shuffles, y neighbours from the thread's own
// rows, z neighbours from the next/previous plane registers (E(i+1) is loaded
// every plane and becomes E(i) of the next, H(i-1) of the own rows stays in
// registers).  There is no shared memory and no block-wide barrier: warps are
// independent.
//
// Each plane is processed as   loads -> compute -> stores:  E(i+1), H(i), the
// E coefficients and every CPML accumulator the plane needs are loaded into
// registers first (about 9R + 9 row loads of 32 consecutive values plus the
// CPML rows), the H and E updates run on registers, and all results are
// stored at the end.  With no store between two loads of a plane every load
// is in flight at once.  The halo recomputation reads the previous time level,
// so the kernel reads set A and writes set B (double-buffered fields and CPML
// state).
//
// Arithmetic per cell follows src/fdtd.cpp:175-310 (H) and :503-669 (E): curl
// scaled by R/d, CPML corrections in x, y, z order with psi <- c d + b psi and
// (psi - d) + d/kappa, sources after each half step, zero E beyond the max
// faces (PEC) and the symmetry rule at j = 0, k = 0, i = 0.
#include "cell.cuh"
#include "kernels.h"

namespace fdtdb {

template <typename T, int R, int WPB>
__global__ void __launch_bounds__(32 * WPB)
    k_step_warp(const GridView<T> ga, const GridView<T> gb, const Fields<T> fa, Fields<T> fb,
                const SourceList<T> src, const long long* __restrict__ step_base, int off,
                int zc) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int Nx = ga.Nx, Ny = ga.Ny, Nz = ga.Nz, px = ga.px;
    const int x0 = blockIdx.x * 30;
    const int k = x0 - 1 + lane;
    const int r0 = (blockIdx.y * WPB + w) * R;
    if (r0 >= Ny) return;   // warp-uniform; warps never synchronise with each other
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, Nz);
    const bool kin = k >= 0 && k < Nx;
    const bool hcol = kin && lane <= 30;
    const bool ecol = kin && lane >= 1 && lane <= 30;

    const T* __restrict__ Ea0 = fa.c[0];
    const T* __restrict__ Ea1 = fa.c[1];
    const T* __restrict__ Ea2 = fa.c[2];
    const T* __restrict__ Ha0 = fa.c[3];
    const T* __restrict__ Ha1 = fa.c[4];
    const T* __restrict__ Ha2 = fa.c[5];
    const T* __restrict__ B0 = ga.bE[0];
    const T* __restrict__ B1 = ga.bE[1];
    const T* __restrict__ B2 = ga.bE[2];
    const T odx = ga.odx, ody = ga.ody, odz = ga.odz;
    const T mx0 = ga.bH[0], my0 = ga.bH[1], mz0 = ga.bH[2];
    const bool mu_arr = ga.bHarr[0] != nullptr;
    const bool lossy = ga.aE[0] != nullptr;

    // CPML slab membership: x per lane, y per row slot, z per plane
    const PmlAxis<T>& PX = ga.pml[0];
    const PmlAxis<T>& PY = ga.pml[1];
    const PmlAxis<T>& PZ = ga.pml[2];
    const int lx = hcol ? slab_local(PX, k, false) : -1;
    int ly[R + 1];
#pragma unroll
    for (int q = 0; q <= R; q++) {
        const int j = r0 - 1 + q;
        ly[q] = (j >= 0 && j < Ny) ? slab_local(PY, j, false) : -1;
    }
    T kxH = T(1), bxH = T(0), cxH = T(0), kxE = T(1), bxE = T(0), cxE = T(0);
    if (lx >= 0) {
        kxH = ld(PX.kinvH + lx); bxH = ld(PX.bH + lx); cxH = ld(PX.cH + lx);
        kxE = ld(PX.kinvE + lx); bxE = ld(PX.bE + lx); cxE = ld(PX.cE + lx);
    }

    // sources overlapping this warp's H/E cells
    unsigned smask = 0;
    for (int q = 0; q < src.n; q++) {
        const DevSource<T>& s = src.s[q];
        if (s.j0 <= r0 + R - 1 && s.j0 + s.J > r0 - 1 && s.k0 <= x0 + 29 && s.k0 + s.K > x0 - 1)
            smask |= 1u << q;
    }
    T SH = T(0), CH = T(0), SE = T(0), CE = T(0);
    if (smask) {
        double4 st = ga.step_tab[*step_base + off];
        SH = T(st.x); CH = T(st.y); SE = T(st.z); CE = T(st.w);
    }

    T ec[3][R + 2], en[3][R + 2];   // E at planes i and i+1, row slots 0 .. R+1
    T hh[3][R + 1];                 // H at plane i, row slots 0 .. R (old, then new)
    T hp[2][R];                     // Hx, Hy at plane i-1 of the own rows
    T ph[R + 1][6];                 // H-update CPML accumulators (x0 x1 y0 y1 z0 z1)
    T pe[R][6];                     // E-update CPML accumulators

    auto row_ok = [&](int q) { const int j = r0 - 1 + q; return j >= 0 && j < Ny; };
    auto off_of = [&](int i, int q) { return (i * Ny + (r0 - 1 + q)) * px + k; };

    auto load_E = [&](T (&d)[3][R + 2], int i) {
#pragma unroll
        for (int q = 0; q < R + 2; q++) {
            const bool ok = kin && i < Nz && row_ok(q);
            const int p = ok ? off_of(i, q) : 0;
            d[0][q] = ok ? ld(Ea0 + p) : T(0);
            d[1][q] = ok ? ld(Ea1 + p) : T(0);
            d[2][q] = ok ? ld(Ea2 + p) : T(0);
        }
    };
    // H of plane i (row slots qlo..R) and the CPML accumulators the H update
    // of those rows needs; with_e: also the E-update accumulators of rows 1..R.
    auto load_H_psi = [&](int i, int qlo, bool with_e) {
        const int lz = slab_local(PZ, i, true);
#pragma unroll
        for (int q = 0; q <= R; q++) {
            const bool ok = q >= qlo && hcol && row_ok(q);
            const int p = ok ? off_of(i, q) : 0;
            hh[0][q] = ok ? ld(Ha0 + p) : T(0);
            hh[1][q] = ok ? ld(Ha1 + p) : T(0);
            hh[2][q] = ok ? ld(Ha2 + p) : T(0);
            const int j = r0 - 1 + q;
            const bool eok = with_e && q >= 1 && ecol && row_ok(q);
            if (ok && lx >= 0) {
                const int s = (i * Ny + j) * PX.wsum + lx;
                ph[q][0] = ld(PX.psi[0] + s); ph[q][1] = ld(PX.psi[1] + s);
                if (eok) { pe[q - 1][0] = ld(PX.psi[2] + s); pe[q - 1][1] = ld(PX.psi[3] + s); }
            }
            if (ok && ly[q] >= 0) {
                const int s = (i * PY.wsum + ly[q]) * px + k;
                ph[q][2] = ld(PY.psi[0] + s); ph[q][3] = ld(PY.psi[1] + s);
                if (eok) { pe[q - 1][2] = ld(PY.psi[2] + s); pe[q - 1][3] = ld(PY.psi[3] + s); }
            }
            if (ok && lz >= 0) {
                const int s = (lz * Ny + j) * px + k;
                ph[q][4] = ld(PZ.psi[0] + s); ph[q][5] = ld(PZ.psi[1] + s);
                if (eok) { pe[q - 1][4] = ld(PZ.psi[2] + s); pe[q - 1][5] = ld(PZ.psi[3] + s); }
            }
        }
    };

    // H(i) of row slots qlo..R in place (registers only; new CPML values in ph).
    auto h_rows = [&](int i, int qlo) {
        const int lz = slab_local(PZ, i, true);
        T kzH = T(1), bzH = T(0), czH = T(0);
        if (lz >= 0) { kzH = ld(PZ.kinvH + lz); bzH = ld(PZ.bH + lz); czH = ld(PZ.cH + lz); }
#pragma unroll
        for (int q = 0; q <= R; q++) {
            const T ey_x = __shfl_down_sync(FULL, ec[1][q], 1);
            const T ez_x = __shfl_down_sync(FULL, ec[2][q], 1);
            if (q < qlo || !hcol || !row_ok(q)) continue;
            const int j = r0 - 1 + q;
            const T ex = ec[0][q], ey = ec[1][q], ez = ec[2][q];
            const T dEzdy = ody * (ec[2][q + 1] - ez);
            const T dEydz = odz * (en[1][q] - ey);
            const T dExdz = odz * (en[0][q] - ex);
            const T dEzdx = odx * (ez_x - ez);
            const T dEydx = odx * (ey_x - ey);
            const T dExdy = ody * (ec[0][q + 1] - ex);
            T mx = mx0, my = my0, mz = mz0;
            if (mu_arr) {
                const int p = off_of(i, q);
                mx = ld(ga.bHarr[0] + p); my = ld(ga.bHarr[1] + p); mz = ld(ga.bHarr[2] + p);
            }
            T hx = hh[0][q] + mx * (dEydz - dEzdy);
            T hy = hh[1][q] + my * (dEzdx - dExdz);
            T hz = hh[2][q] + mz * (dExdy - dEydx);
            if (lx >= 0) {
                const T p0 = cxH * dEydx + bxH * ph[q][0];
                const T p1 = cxH * dEzdx + bxH * ph[q][1];
                ph[q][0] = p0; ph[q][1] = p1;
                hz = hz - mz * ((p0 - dEydx) + dEydx * kxH);
                hy = hy + my * ((p1 - dEzdx) + dEzdx * kxH);
            }
            if (ly[q] >= 0) {
                const T kv = ld(PY.kinvH + ly[q]), bv = ld(PY.bH + ly[q]), cv = ld(PY.cH + ly[q]);
                const T p0 = cv * dExdy + bv * ph[q][2];
                const T p1 = cv * dEzdy + bv * ph[q][3];
                ph[q][2] = p0; ph[q][3] = p1;
                hz = hz + mz * ((p0 - dExdy) + dExdy * kv);
                hx = hx - mx * ((p1 - dEzdy) + dEzdy * kv);
            }
            if (lz >= 0) {
                const T p0 = czH * dExdz + bzH * ph[q][4];
                const T p1 = czH * dEydz + bzH * ph[q][5];
                ph[q][4] = p0; ph[q][5] = p1;
                hx = hx + mx * ((p1 - dEydz) + dEydz * kzH);
                hy = hy - my * ((p0 - dExdz) + dExdz * kzH);
            }
            if (smask) add_sources<T>(src, i, j, k, 3, SH, CH, hx, hy, hz, false);
            hh[0][q] = hx; hh[1][q] = hy; hh[2][q] = hz;
        }
    };

    // ---- chunk prologue: H(z0-1) of the own rows (kept for dH/dz at z0)
    if (z0 > 0) {
        load_E(ec, z0 - 1);
        load_E(en, z0);
        load_H_psi(z0 - 1, 1, false);
        h_rows(z0 - 1, 1);
#pragma unroll
        for (int q = 0; q < R; q++) { hp[0][q] = hh[0][q + 1]; hp[1][q] = hh[1][q + 1]; }
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int q = 0; q < R + 2; q++) ec[c][q] = en[c][q];
    } else {
        load_E(ec, 0);
#pragma unroll
        for (int q = 0; q < R; q++) { hp[0][q] = T(0); hp[1][q] = T(0); }
    }

    for (int i = z0; i < z1; i++) {
        // ---------------- loads
        load_E(en, i + 1);
        load_H_psi(i, 0, true);
        T bb[3][R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            const bool ok = ecol && row_ok(q + 1);
            const int p = ok ? off_of(i, q + 1) : 0;
            bb[0][q] = ok ? ld(B0 + p) : T(0);
            bb[1][q] = ok ? ld(B1 + p) : T(0);
            bb[2][q] = ok ? ld(B2 + p) : T(0);
        }
        // ---------------- H(i): tile rows + halo row/column
        h_rows(i, 0);
        // ---------------- E(i) of the own rows
        const int lz = slab_local(PZ, i, true);
        T kzE = T(1), bzE = T(0), czE = T(0);
        if (lz >= 0) { kzE = ld(PZ.kinvE + lz); bzE = ld(PZ.bE + lz); czE = ld(PZ.cE + lz); }
        T eo[3][R];
#pragma unroll
        for (int q = 1; q <= R; q++) {
            const T hy_k = __shfl_up_sync(FULL, hh[1][q], 1);
            const T hz_k = __shfl_up_sync(FULL, hh[2][q], 1);
            const int j = r0 - 1 + q;
            const T hx = hh[0][q], hy = hh[1][q], hz = hh[2][q];
            T hy_x = hy_k, hz_x = hz_k, hx_y = hh[0][q - 1], hz_y = hh[2][q - 1];
            T hx_z = hp[0][q - 1], hy_z = hp[1][q - 1];
            if (k == 0) { hy_x = h_min_ghost<T>(ga.bc[0], hy, T(0)); hz_x = h_min_ghost<T>(ga.bc[0], hz, T(0)); }
            if (j == 0) { hx_y = h_min_ghost<T>(ga.bc[1], hx, T(0)); hz_y = h_min_ghost<T>(ga.bc[1], hz, T(0)); }
            if (i == 0) { hx_z = h_min_ghost<T>(ga.bc[2], hx, T(0)); hy_z = h_min_ghost<T>(ga.bc[2], hy, T(0)); }
            const T dHzdy = ody * (hz - hz_y);
            const T dHydz = odz * (hy - hy_z);
            const T dHxdz = odz * (hx - hx_z);
            const T dHzdx = odx * (hz - hz_x);
            const T dHydx = odx * (hy - hy_x);
            const T dHxdy = ody * (hx - hx_y);
            const T bx = bb[0][q - 1], by = bb[1][q - 1], bz = bb[2][q - 1];
            T ex = ec[0][q], ey = ec[1][q], ez = ec[2][q];
            if (lossy) {
                const int p = (ecol && row_ok(q)) ? off_of(i, q) : 0;
                ex = ld(ga.aE[0] + p) * ex + (dHzdy - dHydz) * bx;
                ey = ld(ga.aE[1] + p) * ey + (dHxdz - dHzdx) * by;
                ez = ld(ga.aE[2] + p) * ez + (dHydx - dHxdy) * bz;
            } else {
                ex = ex + (dHzdy - dHydz) * bx;
                ey = ey + (dHxdz - dHzdx) * by;
                ez = ez + (dHydx - dHxdy) * bz;
            }
            if (lx >= 0) {
                const T p2 = cxE * dHydx + bxE * pe[q - 1][0];
                const T p3 = cxE * dHzdx + bxE * pe[q - 1][1];
                pe[q - 1][0] = p2; pe[q - 1][1] = p3;
                ez = ez + ((p2 - dHydx) + dHydx * kxE) * bz;
                ey = ey - ((p3 - dHzdx) + dHzdx * kxE) * by;
            }
            if (ly[q] >= 0) {
                const T kv = ld(PY.kinvE + ly[q]), bv = ld(PY.bE + ly[q]), cv = ld(PY.cE + ly[q]);
                const T p2 = cv * dHxdy + bv * pe[q - 1][2];
                const T p3 = cv * dHzdy + bv * pe[q - 1][3];
                pe[q - 1][2] = p2; pe[q - 1][3] = p3;
                ez = ez - ((p2 - dHxdy) + dHxdy * kv) * bz;
                ex = ex + ((p3 - dHzdy) + dHzdy * kv) * bx;
            }
            if (lz >= 0) {
                const T p2 = czE * dHxdz + bzE * pe[q - 1][4];
                const T p3 = czE * dHydz + bzE * pe[q - 1][5];
                pe[q - 1][4] = p2; pe[q - 1][5] = p3;
                ex = ex - ((p3 - dHydz) + dHydz * kzE) * bx;
                ey = ey + ((p2 - dHxdz) + dHxdz * kzE) * by;
            }
            if (smask && ecol && row_ok(q)) add_sources<T>(src, i, j, k, 0, SE, CE, ex, ey, ez, true);
            eo[0][q - 1] = ex; eo[1][q - 1] = ey; eo[2][q - 1] = ez;
        }
        // ---------------- stores (own rows, lanes 1..30)
#pragma unroll
        for (int q = 1; q <= R; q++) {
            if (!ecol || !row_ok(q)) continue;
            const int j = r0 - 1 + q;
            const int p = off_of(i, q);
            fb.c[0][p] = eo[0][q - 1]; fb.c[1][p] = eo[1][q - 1]; fb.c[2][p] = eo[2][q - 1];
            fb.c[3][p] = hh[0][q]; fb.c[4][p] = hh[1][q]; fb.c[5][p] = hh[2][q];
            if (lx >= 0) {
                const int s = (i * Ny + j) * PX.wsum + lx;
                gb.pml[0].psi[0][s] = ph[q][0]; gb.pml[0].psi[1][s] = ph[q][1];
                gb.pml[0].psi[2][s] = pe[q - 1][0]; gb.pml[0].psi[3][s] = pe[q - 1][1];
            }
            if (ly[q] >= 0) {
                const int s = (i * PY.wsum + ly[q]) * px + k;
                gb.pml[1].psi[0][s] = ph[q][2]; gb.pml[1].psi[1][s] = ph[q][3];
                gb.pml[1].psi[2][s] = pe[q - 1][2]; gb.pml[1].psi[3][s] = pe[q - 1][3];
            }
            if (lz >= 0) {
                const int s = (lz * Ny + j) * px + k;
                gb.pml[2].psi[0][s] = ph[q][4]; gb.pml[2].psi[1][s] = ph[q][5];
                gb.pml[2].psi[2][s] = pe[q - 1][4]; gb.pml[2].psi[3][s] = pe[q - 1][5];
            }
        }
#pragma unroll
        for (int q = 0; q < R; q++) { hp[0][q] = hh[0][q + 1]; hp[1][q] = hh[1][q + 1]; }
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int q = 0; q < R + 2; q++) ec[c][q] = en[c][q];
    }
}

namespace {
constexpr int kWarpRows = 2;   // R: rows per thread
constexpr int kWPB = 4;        // warps per block

// Planes per CTA: balance the last wave against the per-chunk prologue (one
// extra plane of H for the own rows).
int pick_zchunk(int Nz, long long tiles, int slots) {
    int best = Nz;
    double best_eff = 0;
    for (int zc = 2; zc <= Nz; zc++) {
        long long chunks = (Nz + zc - 1) / zc;
        long long blocks = tiles * chunks;
        long long waves = (blocks + slots - 1) / slots;
        double tail = (double)blocks / (double)(waves * slots);
        double prologue = (double)Nz / (double)(Nz + (chunks - 1) * 0.6);
        double eff = tail * prologue;
        if (eff > best_eff + 1e-9) { best_eff = eff; best = zc; }
    }
    return best;
}
}  // namespace

template <typename T>
cudaError_t warp_zchunk(int Nx, int Ny, int Nz, int* zc, int* slots_out) {
    int per_sm = 0, sms = 0, dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_warp<T, kWarpRows, kWPB>,
                                                          32 * kWPB, 0);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (per_sm <= 0 || sms <= 0) return cudaErrorInvalidConfiguration;
    long long tiles = (long long)((Nx + 29) / 30) * ((Ny + kWarpRows * kWPB - 1) / (kWarpRows * kWPB));
    *zc = pick_zchunk(Nz, tiles, per_sm * sms);
    if (slots_out) *slots_out = per_sm * sms;
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_step_warp(const GridView<T>& ga, const GridView<T>& gb, T* const* fa,
                             T* const* fb, const SourceList<T>& src, const long long* step_base,
                             int off, int zc, cudaStream_t st) {
    if (zc <= 0) return cudaErrorInvalidValue;
    Fields<T> A, B;
    for (int c = 0; c < 6; c++) { A.c[c] = fa[c]; B.c[c] = fb[c]; }
    dim3 grid((ga.Nx + 29) / 30, (ga.Ny + kWarpRows * kWPB - 1) / (kWarpRows * kWPB),
              (ga.Nz + zc - 1) / zc);
    k_step_warp<T, kWarpRows, kWPB><<<grid, 32 * kWPB, 0, st>>>(ga, gb, A, B, src, step_base, off, zc);
    return cudaGetLastError();
}

template cudaError_t warp_zchunk<float>(int, int, int, int*, int*);
template cudaError_t warp_zchunk<double>(int, int, int, int*, int*);
template cudaError_t launch_step_warp<float>(const GridView<float>&, const GridView<float>&,
                                             float* const*, float* const*,
                                             const SourceList<float>&, const long long*, int, int,
                                             cudaStream_t);
template cudaError_t launch_step_warp<double>(const GridView<double>&, const GridView<double>&,
                                              double* const*, double* const*,
                                              const SourceList<double>&, const long long*, int,
                                              int, cudaStream_t);

}  // namespace fdtdb
