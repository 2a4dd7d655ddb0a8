// tma_kernels.cu -- fused time step with TMA-staged planes (sm_100a).
//
// Same decomposition as a z-marching fused step: a CTA owns a 32 (x) by TY
// (y) column tile and a chunk of planes; for every plane i it computes H(i)
// for the tile plus the low halo row/column (the cells the E update reads at
// j-1 and k-1), then E(i) for the tile, reading the previous time level from
// set A and writing set B (double-buffered fields and CPML state, so the
// redundant halo H keeps CTAs independent).
//
// Data movement:
//   * one elected thread streams the planes ahead of the computation with
//     cp.async.bulk.tensor (TMA) into an S-stage shared-memory ring, one
//     mbarrier per stage: per plane E (tile + one-cell ring, box 40 x TY+2),
//     the previous H (tile + low halo, box 36 x TY+1) and the three E-update
//     coefficients (tile, box 32 x TY).  The x origin of every box is x0 - 4
//     or x0 with x0 a multiple of 32, i.e. 16-byte aligned; boxes that start
//     before the grid or reach past it are zero-filled, which doubles as the
//     PEC condition on the max faces;
//   * CPML auxiliary values are read with ordinary loads issued one plane
//     ahead into registers (their layouts are per slab);
//   * H(i-1) of the own cell stays in registers, the new H of the tile and
//     halo goes through shared memory for the E update.
// Every mbarrier wait is bounded; a wait that runs out sets *err and the CTA
// finishes without further waits (its output is then flagged as invalid by
// the host).
#include <cuda.h>

#include "async.cuh"
#include "cell.cuh"
#include "kernels.h"

namespace fdtdb {

namespace {

constexpr int align128(int b) { return (b + 127) / 128 * 128; }

}  // namespace

template <typename T, int TY>
struct TmaGeom {
    static constexpr int EW = 40, HW = 36, BW = 32;
    static constexpr int EB = align128((int)sizeof(T) * (TY + 2) * EW);
    static constexpr int HB = align128((int)sizeof(T) * (TY + 1) * HW);
    static constexpr int BB = align128((int)sizeof(T) * TY * BW);
    static constexpr int STAGE = 3 * (EB + HB + BB);
    static constexpr uint32_t TX = 3u * sizeof(T) * ((TY + 2) * EW + (TY + 1) * HW + TY * BW);
    static constexpr int HN = (int)sizeof(T) * 3 * (TY + 1) * 33;
    static int smem_bytes(int S) { return 128 + S * STAGE + 64 + HN; }
};

template <typename T, int TY, int S, int MINB>
__global__ void __launch_bounds__(32 * (TY + 2), MINB)
    k_step_tma(const __grid_constant__ StepMaps maps, const GridView<T> ga, const GridView<T> gb,
               Fields<T> fb, const SourceList<T> src, const long long* __restrict__ step_base,
               int off, int zc, int* err) {
    using G = TmaGeom<T, TY>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        smem_raw + ((128 - (smem_addr(smem_raw) & 127)) & 127);   // 128-byte aligned ring
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S * G::STAGE);
    T(*sHn)[TY + 1][33] = reinterpret_cast<T(*)[TY + 1][33]>(smem + S * G::STAGE + 64);

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int Nx = ga.Nx, Ny = ga.Ny, Nz = ga.Nz, px = ga.px;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, Nz);
    const int pstart = z0 > 0 ? z0 - 1 : 0;
    const int nplanes = z1 - pstart + 1;   // planes pstart .. z1 are staged

    // H cell of this thread: warps 0..TY-1 own rows, warp TY the halo row
    // y0-1, warp TY+1 (lanes 0..TY) the halo column x0-1.
    int hr, hc;
    if (w < TY) { hr = w + 1; hc = lane + 1; }
    else if (w == TY) { hr = 0; hc = lane + 1; }
    else { hr = lane; hc = 0; }
    const int hj = y0 - 1 + hr, hk = x0 - 1 + hc;
    const bool hact = (w <= TY || lane <= TY) && hj >= 0 && hj < Ny && hk >= 0 && hk < Nx;
    const bool own = w < TY && hact;
    const int ec = hc + 3;   // column in the E/H staging boxes (origin x0-4)

    auto sE = [&](int st, int c) {
        return reinterpret_cast<T(*)[G::EW]>(smem + st * G::STAGE + c * G::EB);
    };
    auto sH = [&](int st, int c) {
        return reinterpret_cast<T(*)[G::HW]>(smem + st * G::STAGE + 3 * G::EB + c * G::HB);
    };
    auto sB = [&](int st, int c) {
        return reinterpret_cast<T(*)[G::BW]>(smem + st * G::STAGE + 3 * (G::EB + G::HB) +
                                             c * G::BB);
    };
    auto issue = [&](int st, int plane) {
        fence_proxy_async();
        mbar_expect_tx(&bars[st], G::TX);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            tma_load_3d(sE(st, c), &maps.E[c], &bars[st], x0 - 4, y0 - 1, plane);
            tma_load_3d(sH(st, c), &maps.H[c], &bars[st], x0 - 4, y0 - 1, plane);
            tma_load_3d(sB(st, c), &maps.B[c], &bars[st], x0, y0, plane);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(&bars[s], 1);
        fence_mbar_init();
        for (int q = 0; q < S && q < nplanes; q++) issue(q, pstart + q);
    }
    __syncthreads();

    // ---- per-thread constants: CPML slab membership and coefficients in x and y
    const PmlAxis<T>& PX = ga.pml[0];
    const PmlAxis<T>& PY = ga.pml[1];
    const PmlAxis<T>& PZ = ga.pml[2];
    const int lx = hact ? slab_local(PX, hk, false) : -1;
    const int ly = hact ? slab_local(PY, hj, false) : -1;
    const T mx0 = ga.bH[0], my0 = ga.bH[1], mz0 = ga.bH[2];
    const bool mu_arr = ga.bHarr[0] != nullptr;
    const bool lossy = ga.aE[0] != nullptr;

    // psi of set A for one plane: h[] for the H update, e[] for the E update,
    // (x0, x1, y0, y1, z0, z1) = two accumulators per slab.
    struct Psi { T h[6]; T e[6]; };
    auto load_psi = [&](int i, Psi& r) {
        if (lx >= 0) {
            int s = (i * Ny + hj) * PX.wsum + lx;
            r.h[0] = PX.psi[0][s]; r.h[1] = PX.psi[1][s];
            if (own) { r.e[0] = PX.psi[2][s]; r.e[1] = PX.psi[3][s]; }
        }
        if (ly >= 0) {
            int s = (i * PY.wsum + ly) * px + hk;
            r.h[2] = PY.psi[0][s]; r.h[3] = PY.psi[1][s];
            if (own) { r.e[2] = PY.psi[2][s]; r.e[3] = PY.psi[3][s]; }
        }
        int lz = slab_local(PZ, i, true);
        if (lz >= 0 && hact) {
            int s = (lz * Ny + hj) * px + hk;
            r.h[4] = PZ.psi[0][s]; r.h[5] = PZ.psi[1][s];
            if (own) { r.e[4] = PZ.psi[2][s]; r.e[5] = PZ.psi[3][s]; }
        }
    };

    // sources touching this tile (bit q set: box q overlaps the tile's rows/columns)
    unsigned smask = 0;
    for (int q = 0; q < src.n; q++) {
        const DevSource<T>& s = src.s[q];
        if (s.j0 <= y0 + TY - 1 && s.j0 + s.J > y0 - 1 && s.k0 <= x0 + 31 && s.k0 + s.K > x0 - 1)
            smask |= 1u << q;
    }
    T SH = T(0), CH = T(0), SE = T(0), CE = T(0);
    if (smask) {
        double4 st = ga.step_tab[*step_base + off];
        SH = T(st.x); CH = T(st.y); SE = T(st.z); CE = T(st.w);
    }

    Psi cur, nxt;
#pragma unroll
    for (int q = 0; q < 6; q++) { cur.h[q] = T(0); cur.e[q] = T(0); nxt.h[q] = T(0); nxt.e[q] = T(0); }
    load_psi(pstart, cur);

    bool ok = true;
    T hpx = T(0), hpy = T(0);
    for (int p = pstart; p < z1; p++) {
        const int q = p - pstart, cs = q % S, ns = (q + 1) % S;
        if (ok) ok = mbar_wait(&bars[cs], (q / S) & 1, err);
        if (ok) ok = mbar_wait(&bars[ns], ((q + 1) / S) & 1, err);
        if (p + 1 < z1) load_psi(p + 1, nxt);

        const int lz = slab_local(PZ, p, true);
        const bool interior = p >= z0;
        const bool do_h = interior ? hact : own;
        const int pidx = (p * Ny + hj) * px + hk;   // pitched offset of (p, hj, hk)

        // ---------------- H(p) for the tile and its low halo
        T hx = T(0), hy = T(0), hz = T(0);
        if (do_h) {
            auto Ec = [&](int c) { return sE(cs, c); };
            auto En = [&](int c) { return sE(ns, c); };
            const T ex = Ec(0)[hr][ec], ey = Ec(1)[hr][ec], ez = Ec(2)[hr][ec];
            const T dEzdy = ga.ody * (Ec(2)[hr + 1][ec] - ez);
            const T dEydz = ga.odz * (En(1)[hr][ec] - ey);
            const T dExdz = ga.odz * (En(0)[hr][ec] - ex);
            const T dEzdx = ga.odx * (Ec(2)[hr][ec + 1] - ez);
            const T dEydx = ga.odx * (Ec(1)[hr][ec + 1] - ey);
            const T dExdy = ga.ody * (Ec(0)[hr + 1][ec] - ex);
            T mx = mx0, my = my0, mz = mz0;
            if (mu_arr) { mx = ga.bHarr[0][pidx]; my = ga.bHarr[1][pidx]; mz = ga.bHarr[2][pidx]; }
            hx = sH(cs, 0)[hr][ec] + mx * (dEydz - dEzdy);
            hy = sH(cs, 1)[hr][ec] + my * (dEzdx - dExdz);
            hz = sH(cs, 2)[hr][ec] + mz * (dExdy - dEydx);
            const bool wpsi = own && interior;
            if (lx >= 0) {
                const T kHx = ld(PX.kinvH + lx), bHx = ld(PX.bH + lx), cHx = ld(PX.cH + lx);
                T p0 = cHx * dEydx + bHx * cur.h[0];
                T p1 = cHx * dEzdx + bHx * cur.h[1];
                if (wpsi) {
                    int s = (p * Ny + hj) * PX.wsum + lx;
                    gb.pml[0].psi[0][s] = p0; gb.pml[0].psi[1][s] = p1;
                }
                hz = hz - mz * ((p0 - dEydx) + dEydx * kHx);
                hy = hy + my * ((p1 - dEzdx) + dEzdx * kHx);
            }
            if (ly >= 0) {
                const T kHy = ld(PY.kinvH + ly), bHy = ld(PY.bH + ly), cHy = ld(PY.cH + ly);
                T p0 = cHy * dExdy + bHy * cur.h[2];
                T p1 = cHy * dEzdy + bHy * cur.h[3];
                if (wpsi) {
                    int s = (p * PY.wsum + ly) * px + hk;
                    gb.pml[1].psi[0][s] = p0; gb.pml[1].psi[1][s] = p1;
                }
                hz = hz + mz * ((p0 - dExdy) + dExdy * kHy);
                hx = hx - mx * ((p1 - dEzdy) + dEzdy * kHy);
            }
            if (lz >= 0) {
                const T kHz = ld(PZ.kinvH + lz), bHz = ld(PZ.bH + lz), cHz = ld(PZ.cH + lz);
                T p0 = cHz * dExdz + bHz * cur.h[4];
                T p1 = cHz * dEydz + bHz * cur.h[5];
                if (wpsi) {
                    int s = (lz * Ny + hj) * px + hk;
                    gb.pml[2].psi[0][s] = p0; gb.pml[2].psi[1][s] = p1;
                }
                hx = hx + mx * ((p1 - dEydz) + dEydz * kHz);
                hy = hy - my * ((p0 - dExdz) + dExdz * kHz);
            }
            if (smask) add_sources<T>(src, p, hj, hk, 3, SH, CH, hx, hy, hz, false);
            if (interior) { sHn[0][hr][hc] = hx; sHn[1][hr][hc] = hy; sHn[2][hr][hc] = hz; }
        }
        if (interior) {
            __syncthreads();
            // ---------------- E(p) for the tile
            if (own) {
                T hy_x, hz_x, hx_y, hz_y, hx_z, hy_z;
                if (hk > 0) { hy_x = sHn[1][hr][hc - 1]; hz_x = sHn[2][hr][hc - 1]; }
                else { hy_x = h_min_ghost<T>(ga.bc[0], hy, T(0)); hz_x = h_min_ghost<T>(ga.bc[0], hz, T(0)); }
                if (hj > 0) { hx_y = sHn[0][hr - 1][hc]; hz_y = sHn[2][hr - 1][hc]; }
                else { hx_y = h_min_ghost<T>(ga.bc[1], hx, T(0)); hz_y = h_min_ghost<T>(ga.bc[1], hz, T(0)); }
                if (p > 0) { hx_z = hpx; hy_z = hpy; }
                else { hx_z = h_min_ghost<T>(ga.bc[2], hx, T(0)); hy_z = h_min_ghost<T>(ga.bc[2], hy, T(0)); }
                const T dHzdy = ga.ody * (hz - hz_y);
                const T dHydz = ga.odz * (hy - hy_z);
                const T dHxdz = ga.odz * (hx - hx_z);
                const T dHzdx = ga.odx * (hz - hz_x);
                const T dHydx = ga.odx * (hy - hy_x);
                const T dHxdy = ga.ody * (hx - hx_y);
                const T bx = sB(cs, 0)[hr - 1][hc - 1], by = sB(cs, 1)[hr - 1][hc - 1],
                        bz = sB(cs, 2)[hr - 1][hc - 1];
                T ex = sE(cs, 0)[hr][ec], ey = sE(cs, 1)[hr][ec], ez = sE(cs, 2)[hr][ec];
                if (lossy) {
                    ex = ga.aE[0][pidx] * ex + (dHzdy - dHydz) * bx;
                    ey = ga.aE[1][pidx] * ey + (dHxdz - dHzdx) * by;
                    ez = ga.aE[2][pidx] * ez + (dHydx - dHxdy) * bz;
                } else {
                    ex = ex + (dHzdy - dHydz) * bx;
                    ey = ey + (dHxdz - dHzdx) * by;
                    ez = ez + (dHydx - dHxdy) * bz;
                }
                if (lx >= 0) {
                    const T kEx = ld(PX.kinvE + lx), bEx = ld(PX.bE + lx), cEx = ld(PX.cE + lx);
                    T p2 = cEx * dHydx + bEx * cur.e[0];
                    T p3 = cEx * dHzdx + bEx * cur.e[1];
                    int s = (p * Ny + hj) * PX.wsum + lx;
                    gb.pml[0].psi[2][s] = p2; gb.pml[0].psi[3][s] = p3;
                    ez = ez + ((p2 - dHydx) + dHydx * kEx) * bz;
                    ey = ey - ((p3 - dHzdx) + dHzdx * kEx) * by;
                }
                if (ly >= 0) {
                    const T kEy = ld(PY.kinvE + ly), bEy = ld(PY.bE + ly), cEy = ld(PY.cE + ly);
                    T p2 = cEy * dHxdy + bEy * cur.e[2];
                    T p3 = cEy * dHzdy + bEy * cur.e[3];
                    int s = (p * PY.wsum + ly) * px + hk;
                    gb.pml[1].psi[2][s] = p2; gb.pml[1].psi[3][s] = p3;
                    ez = ez - ((p2 - dHxdy) + dHxdy * kEy) * bz;
                    ex = ex + ((p3 - dHzdy) + dHzdy * kEy) * bx;
                }
                if (lz >= 0) {
                    const T kEz = ld(PZ.kinvE + lz), bEz = ld(PZ.bE + lz), cEz = ld(PZ.cE + lz);
                    T p2 = cEz * dHxdz + bEz * cur.e[4];
                    T p3 = cEz * dHydz + bEz * cur.e[5];
                    int s = (lz * Ny + hj) * px + hk;
                    gb.pml[2].psi[2][s] = p2; gb.pml[2].psi[3][s] = p3;
                    ex = ex - ((p3 - dHydz) + dHydz * kEz) * bx;
                    ey = ey + ((p2 - dHxdz) + dHxdz * kEz) * by;
                }
                if (smask) add_sources<T>(src, p, hj, hk, 0, SE, CE, ex, ey, ez, true);
                fb.c[0][pidx] = ex; fb.c[1][pidx] = ey; fb.c[2][pidx] = ez;
                fb.c[3][pidx] = hx; fb.c[4][pidx] = hy; fb.c[5][pidx] = hz;
            }
        }
        if (own) { hpx = hx; hpy = hy; }
        __syncthreads();
        if (tid == 0 && ok && q + S < nplanes) issue(cs, p + S);
        cur = nxt;
    }
}

template <typename T, int TY, int S, int MINB>
static cudaError_t launch_tma(const StepMaps& maps, const GridView<T>& ga, const GridView<T>& gb,
                              T* const* fb, const SourceList<T>& src, const long long* step_base,
                              int off, int zc, int* err, cudaStream_t st) {
    using G = TmaGeom<T, TY>;
    static unsigned long long configured = 0;   // bit d: attribute set on device d
    int smem = G::smem_bytes(S);
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(configured >> dev & 1ull)) {
        cudaError_t e = cudaFuncSetAttribute(k_step_tma<T, TY, S, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        configured |= 1ull << dev;
    }
    Fields<T> B;
    for (int c = 0; c < 6; c++) B.c[c] = fb[c];
    dim3 grid((ga.Nx + 31) / 32, (ga.Ny + TY - 1) / TY, (ga.Nz + zc - 1) / zc);
    k_step_tma<T, TY, S, MINB><<<grid, 32 * (TY + 2), smem, st>>>(maps, ga, gb, B, src, step_base, off,
                                                             zc, err);
    return cudaGetLastError();
}

int tma_tile_rows() { return 8; }

template <>
cudaError_t launch_step_tma<float>(const StepMaps& maps, const GridView<float>& ga,
                                   const GridView<float>& gb, float* const* fb,
                                   const SourceList<float>& src, const long long* step_base,
                                   int off, int zc, int* err, cudaStream_t st) {
    return launch_tma<float, 8, 4, 3>(maps, ga, gb, fb, src, step_base, off, zc, err, st);
}

template <>
cudaError_t launch_step_tma<double>(const StepMaps& maps, const GridView<double>& ga,
                                    const GridView<double>& gb, double* const* fb,
                                    const SourceList<double>& src, const long long* step_base,
                                    int off, int zc, int* err, cudaStream_t st) {
    return launch_tma<double, 8, 3, 2>(maps, ga, gb, fb, src, step_base, off, zc, err, st);
}

}  // namespace fdtdb
