// fused_kernels.cu -- one launch per time step: H and E half-steps fused.
//
// A CTA owns a 32 (x) by TY (y) column tile and a chunk of zc planes.  It
// marches up through z; for every plane i it
//   1. stages E(i+1) for the tile plus a one-cell ring in shared memory
//      (E(i) is already there from the previous plane),
//   2. computes H(i) for the tile and for its low halo row/column (the cells
//      the E update reads at j-1 and k-1) into shared memory, adding the
//      magnetic currents,
//   3. computes E(i) for the tile from H(i) (shared memory), H(i-1) (kept in
//      registers from the previous plane) and its own E, adding the electric
//      currents, and writes H(i) and E(i) of the tile.
// The halo H is recomputed redundantly from the previous time level, which is
// what makes CTAs independent inside one launch; for that the fields and the
// CPML state are double-buffered: step n reads set (n & 1) and writes the
// other set.  At a chunk start the CTA first recomputes H(z0-1) for its tile.
//
// Traffic per cell and step is one read of E, H, the three E coefficients and
// the CPML state, and one write of E, H and the CPML state -- the 60 B (fp32)
// bulk figure -- instead of the 84 B of separate H and E sweeps.  Halo reads
// hit L2 (they are neighbouring tiles' own cells of the same plane).
//
// The max-face PEC condition enters as zero E outside the grid; the min-face
// symmetry rule ('0', 'E', 'H') is applied by the cell on the face.  Periodic
// axes need H(i) of the opposite face, which this launch has not produced, so
// the solver uses the in-place kernel pair for them.
#include "cell.cuh"
#include "kernels.h"

namespace fdtdb {

template <typename T, int TY>
__global__ void __launch_bounds__(32 * (TY + 2))
    k_step_fused(GridView<T> ga, GridView<T> gb, Fields<T> fa, Fields<T> fb, SourceList<T> src,
                 const long long* step_base, int off, int zc) {
    constexpr int EW = 34;  // staged columns: x0-1 .. x0+32
    __shared__ T sE[2][3][TY + 2][EW];
    __shared__ T sH[3][TY + 1][33];

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int Nx = ga.Nx, Ny = ga.Ny, Nz = ga.Nz;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, Nz);

    // H cell of this thread: warps 0..TY-1 own rows, warp TY the halo row
    // y0-1, warp TY+1 (lanes 0..TY) the halo column x0-1.
    int hr, hc;
    if (w < TY) { hr = w + 1; hc = lane + 1; }
    else if (w == TY) { hr = 0; hc = lane + 1; }
    else { hr = lane; hc = 0; }
    const int hj = y0 - 1 + hr, hk = x0 - 1 + hc;
    const bool hact = (w <= TY || lane <= TY) && hj >= 0 && hj < Ny && hk >= 0 && hk < Nx;
    const bool own = w < TY && hact;

    T SH = T(0), CH = T(0), SE = T(0), CE = T(0);
    if (src.n) {
        double4 st = ga.step_tab[*step_base + off];
        SH = T(st.x); CH = T(st.y); SE = T(st.z); CE = T(st.w);
    }

    auto stage_E = [&](int buf, int i) {
        for (int e = threadIdx.x; e < (TY + 2) * EW; e += blockDim.x) {
            int r = e / EW, c = e - r * EW;
            int j = y0 - 1 + r, k = x0 - 1 + c;
            T v0 = T(0), v1 = T(0), v2 = T(0);
            if (i < Nz && j >= 0 && j < Ny && k >= 0 && k < Nx) {
                long long p = (long long)i * ga.plane + (long long)j * ga.px + k;
                v0 = ld(fa.c[0] + p); v1 = ld(fa.c[1] + p); v2 = ld(fa.c[2] + p);
            }
            sE[buf][0][r][c] = v0; sE[buf][1][r][c] = v1; sE[buf][2][r][c] = v2;
        }
    };
    auto gather_HIn = [&](int cur, int nxt) {
        HIn<T> e;
        e.ex = sE[cur][0][hr][hc]; e.ey = sE[cur][1][hr][hc]; e.ez = sE[cur][2][hr][hc];
        e.ey_x = sE[cur][1][hr][hc + 1]; e.ez_x = sE[cur][2][hr][hc + 1];
        e.ex_y = sE[cur][0][hr + 1][hc]; e.ez_y = sE[cur][2][hr + 1][hc];
        e.ex_z = sE[nxt][0][hr][hc]; e.ey_z = sE[nxt][1][hr][hc];
        return e;
    };

    T hpx = T(0), hpy = T(0);   // H(i-1) of the own cell
    int cur = 0;
    if (z0 > 0) {
        stage_E(0, z0 - 1);
        stage_E(1, z0);
        __syncthreads();
        if (own) {
            const int i = z0 - 1;
            long long p = (long long)i * ga.plane + (long long)hj * ga.px + hk;
            T hx = ld(fa.c[3] + p), hy = ld(fa.c[4] + p), hz = ld(fa.c[5] + p);
            HIn<T> e = gather_HIn(0, 1);
            h_cell<T>(ga, i, hj, hk, p, e, hx, hy, hz, ga.pml[0].psi, gb.pml[0].psi, ga.pml[1].psi,
                      gb.pml[1].psi, ga.pml[2].psi, gb.pml[2].psi, false);
            if (src.n) add_sources<T>(src, i, hj, hk, 3, SH, CH, hx, hy, hz, false);
            hpx = hx; hpy = hy;
        }
        cur = 1;
        __syncthreads();
    } else {
        stage_E(0, 0);
    }

    for (int i = z0; i < z1; i++) {
        const int nxt = cur ^ 1;
        stage_E(nxt, i + 1);
        long long p = (long long)i * ga.plane + (long long)hj * ga.px + hk;
        T hx = T(0), hy = T(0), hz = T(0);
        if (hact) { hx = ld(fa.c[3] + p); hy = ld(fa.c[4] + p); hz = ld(fa.c[5] + p); }
        __syncthreads();
        if (hact) {
            HIn<T> e = gather_HIn(cur, nxt);
            h_cell<T>(ga, i, hj, hk, p, e, hx, hy, hz, ga.pml[0].psi, gb.pml[0].psi, ga.pml[1].psi,
                      gb.pml[1].psi, ga.pml[2].psi, gb.pml[2].psi, own);
            if (src.n) add_sources<T>(src, i, hj, hk, 3, SH, CH, hx, hy, hz, false);
            sH[0][hr][hc] = hx; sH[1][hr][hc] = hy; sH[2][hr][hc] = hz;
        }
        __syncthreads();
        if (own) {
            EIn<T> h;
            h.hx = hx; h.hy = hy; h.hz = hz;
            if (hk > 0) { h.hy_x = sH[1][hr][hc - 1]; h.hz_x = sH[2][hr][hc - 1]; }
            else { h.hy_x = h_min_ghost<T>(ga.bc[0], hy, T(0)); h.hz_x = h_min_ghost<T>(ga.bc[0], hz, T(0)); }
            if (hj > 0) { h.hx_y = sH[0][hr - 1][hc]; h.hz_y = sH[2][hr - 1][hc]; }
            else { h.hx_y = h_min_ghost<T>(ga.bc[1], hx, T(0)); h.hz_y = h_min_ghost<T>(ga.bc[1], hz, T(0)); }
            if (i > 0) { h.hx_z = hpx; h.hy_z = hpy; }
            else { h.hx_z = h_min_ghost<T>(ga.bc[2], hx, T(0)); h.hy_z = h_min_ghost<T>(ga.bc[2], hy, T(0)); }
            T ex = sE[cur][0][hr][hc], ey = sE[cur][1][hr][hc], ez = sE[cur][2][hr][hc];
            T bx, by, bz;
            e_cell<T>(ga, i, hj, hk, p, h, ex, ey, ez, ga.pml[0].psi, gb.pml[0].psi, ga.pml[1].psi,
                      gb.pml[1].psi, ga.pml[2].psi, gb.pml[2].psi, bx, by, bz);
            if (src.n) add_sources<T>(src, i, hj, hk, 0, SE, CE, ex, ey, ez, true);
            fb.c[0][p] = ex; fb.c[1][p] = ey; fb.c[2][p] = ez;
            fb.c[3][p] = hx; fb.c[4][p] = hy; fb.c[5][p] = hz;
            hpx = hx; hpy = hy;
        }
        cur = nxt;
        __syncthreads();
    }
}

constexpr int kFusedTY = 8;

int fused_zchunk(int Nz) { return Nz < 16 ? Nz : 16; }

template <typename T>
void launch_step_fused(const GridView<T>& ga, const GridView<T>& gb, T* const* fa, T* const* fb,
                       const SourceList<T>& src, const long long* step_base, int off,
                       cudaStream_t st) {
    Fields<T> A, B;
    for (int c = 0; c < 6; c++) { A.c[c] = fa[c]; B.c[c] = fb[c]; }
    int zc = fused_zchunk(ga.Nz);
    dim3 grid((ga.Nx + 31) / 32, (ga.Ny + kFusedTY - 1) / kFusedTY, (ga.Nz + zc - 1) / zc);
    k_step_fused<T, kFusedTY><<<grid, 32 * (kFusedTY + 2), 0, st>>>(ga, gb, A, B, src, step_base,
                                                                   off, zc);
}

template void launch_step_fused<float>(const GridView<float>&, const GridView<float>&,
                                       float* const*, float* const*, const SourceList<float>&,
                                       const long long*, int, cudaStream_t);
template void launch_step_fused<double>(const GridView<double>&, const GridView<double>&,
                                        double* const*, double* const*,
                                        const SourceList<double>&, const long long*, int,
                                        cudaStream_t);

}  // namespace fdtdb
