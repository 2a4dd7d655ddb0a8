// cell.cuh -- per-cell Yee arithmetic shared by the unfused and fused
// step kernels (src/fdtd.cpp:175-310 for H, :503-669 for E).
#pragma once

#include "grid.cuh"

namespace fdtdb {

template <typename T>
struct Fields {
    T* c[6];  // Ex Ey Ez Hx Hy Hz
};

template <typename T>
__device__ __forceinline__ T ld(const T* p) {
    return __ldg(p);
}

// ------------------------------------------------------------ H arithmetic
// Everything the H update of one cell needs, given the E neighbours.
template <typename T>
struct HIn {
    T ex, ey, ez;          // E at the cell
    T ex_y, ex_z;          // Ex at j+1, i+1
    T ey_x, ey_z;          // Ey at k+1, i+1
    T ez_x, ez_y;          // Ez at k+1, j+1
};

template <typename T>
__device__ __forceinline__ void h_cell(const GridView<T>& g, int i, int j, int k, long long p,
                                       const HIn<T>& e, T& hx, T& hy, T& hz,
                                       T* const* psi_rd_x, T* const* psi_wr_x,
                                       T* const* psi_rd_y, T* const* psi_wr_y,
                                       T* const* psi_rd_z, T* const* psi_wr_z, bool write_psi) {
    T mx = g.bHarr[0] ? ld(g.bHarr[0] + p) : g.bH[0];
    T my = g.bHarr[1] ? ld(g.bHarr[1] + p) : g.bH[1];
    T mz = g.bHarr[2] ? ld(g.bHarr[2] + p) : g.bH[2];
    T dEzdy = g.ody * (e.ez_y - e.ez);
    T dEydz = g.odz * (e.ey_z - e.ey);
    T dExdz = g.odz * (e.ex_z - e.ex);
    T dEzdx = g.odx * (e.ez_x - e.ez);
    T dEydx = g.odx * (e.ey_x - e.ey);
    T dExdy = g.ody * (e.ex_y - e.ex);
    hx = hx + mx * (dEydz - dEzdy);
    hy = hy + my * (dEzdx - dExdz);
    hz = hz + mz * (dExdy - dEydx);

    const PmlAxis<T>& PX = g.pml[0];
    int l = slab_local(PX, k, false);
    if (l >= 0) {
        long long s = ((long long)i * g.Ny + j) * PX.wsum + l;
        T kinv = ld(PX.kinvH + l), b = ld(PX.bH + l), C = ld(PX.cH + l);
        T p0 = C * dEydx + b * psi_rd_x[0][s];
        T p1 = C * dEzdx + b * psi_rd_x[1][s];
        if (write_psi) { psi_wr_x[0][s] = p0; psi_wr_x[1][s] = p1; }
        hz = hz - mz * ((p0 - dEydx) + dEydx * kinv);
        hy = hy + my * ((p1 - dEzdx) + dEzdx * kinv);
    }
    const PmlAxis<T>& PY = g.pml[1];
    l = slab_local(PY, j, false);
    if (l >= 0) {
        long long s = ((long long)i * PY.wsum + l) * g.px + k;
        T kinv = ld(PY.kinvH + l), b = ld(PY.bH + l), C = ld(PY.cH + l);
        T p0 = C * dExdy + b * psi_rd_y[0][s];
        T p1 = C * dEzdy + b * psi_rd_y[1][s];
        if (write_psi) { psi_wr_y[0][s] = p0; psi_wr_y[1][s] = p1; }
        hz = hz + mz * ((p0 - dExdy) + dExdy * kinv);
        hx = hx - mx * ((p1 - dEzdy) + dEzdy * kinv);
    }
    const PmlAxis<T>& PZ = g.pml[2];
    l = slab_local(PZ, i, true);
    if (l >= 0) {
        long long s = ((long long)l * g.Ny + j) * g.px + k;
        T kinv = ld(PZ.kinvH + l), b = ld(PZ.bH + l), C = ld(PZ.cH + l);
        T p0 = C * dExdz + b * psi_rd_z[0][s];
        T p1 = C * dEydz + b * psi_rd_z[1][s];
        if (write_psi) { psi_wr_z[0][s] = p0; psi_wr_z[1][s] = p1; }
        hx = hx + mx * ((p1 - dEydz) + dEydz * kinv);
        hy = hy - my * ((p0 - dExdz) + dExdz * kinv);
    }
}

// ------------------------------------------------------------ E arithmetic
template <typename T>
struct EIn {
    T hx, hy, hz;          // H at the cell
    T hx_y, hx_z;          // Hx at j-1, i-1
    T hy_x, hy_z;          // Hy at k-1, i-1
    T hz_x, hz_y;          // Hz at k-1, j-1
};

template <typename T>
__device__ __forceinline__ void e_cell(const GridView<T>& g, int i, int j, int k, long long p,
                                       const EIn<T>& h, T& ex, T& ey, T& ez,
                                       T* const* psi_rd_x, T* const* psi_wr_x,
                                       T* const* psi_rd_y, T* const* psi_wr_y,
                                       T* const* psi_rd_z, T* const* psi_wr_z,
                                       T& bx, T& by, T& bz) {
    bx = ld(g.bE[0] + p);
    by = ld(g.bE[1] + p);
    bz = ld(g.bE[2] + p);
    T dHzdy = g.ody * (h.hz - h.hz_y);
    T dHydz = g.odz * (h.hy - h.hy_z);
    T dHxdz = g.odz * (h.hx - h.hx_z);
    T dHzdx = g.odx * (h.hz - h.hz_x);
    T dHydx = g.odx * (h.hy - h.hy_x);
    T dHxdy = g.ody * (h.hx - h.hx_y);
    if (g.aE[0]) {
        ex = ld(g.aE[0] + p) * ex + (dHzdy - dHydz) * bx;
        ey = ld(g.aE[1] + p) * ey + (dHxdz - dHzdx) * by;
        ez = ld(g.aE[2] + p) * ez + (dHydx - dHxdy) * bz;
    } else {
        ex = ex + (dHzdy - dHydz) * bx;
        ey = ey + (dHxdz - dHzdx) * by;
        ez = ez + (dHydx - dHxdy) * bz;
    }
    const PmlAxis<T>& PX = g.pml[0];
    int l = slab_local(PX, k, false);
    if (l >= 0) {
        long long s = ((long long)i * g.Ny + j) * PX.wsum + l;
        T kinv = ld(PX.kinvE + l), b = ld(PX.bE + l), C = ld(PX.cE + l);
        T p2 = C * dHydx + b * psi_rd_x[2][s];
        T p3 = C * dHzdx + b * psi_rd_x[3][s];
        psi_wr_x[2][s] = p2; psi_wr_x[3][s] = p3;
        ez = ez + ((p2 - dHydx) + dHydx * kinv) * bz;
        ey = ey - ((p3 - dHzdx) + dHzdx * kinv) * by;
    }
    const PmlAxis<T>& PY = g.pml[1];
    l = slab_local(PY, j, false);
    if (l >= 0) {
        long long s = ((long long)i * PY.wsum + l) * g.px + k;
        T kinv = ld(PY.kinvE + l), b = ld(PY.bE + l), C = ld(PY.cE + l);
        T p2 = C * dHxdy + b * psi_rd_y[2][s];
        T p3 = C * dHzdy + b * psi_rd_y[3][s];
        psi_wr_y[2][s] = p2; psi_wr_y[3][s] = p3;
        ez = ez - ((p2 - dHxdy) + dHxdy * kinv) * bz;
        ex = ex + ((p3 - dHzdy) + dHzdy * kinv) * bx;
    }
    const PmlAxis<T>& PZ = g.pml[2];
    l = slab_local(PZ, i, true);
    if (l >= 0) {
        long long s = ((long long)l * g.Ny + j) * g.px + k;
        T kinv = ld(PZ.kinvE + l), b = ld(PZ.bE + l), C = ld(PZ.cE + l);
        T p2 = C * dHxdz + b * psi_rd_z[2][s];
        T p3 = C * dHydz + b * psi_rd_z[3][s];
        psi_wr_z[2][s] = p2; psi_wr_z[3][s] = p3;
        ex = ex - ((p3 - dHydz) + dHydz * kinv) * bx;
        ey = ey + ((p2 - dHxdz) + dHxdz * kinv) * by;
    }
}

// Add the magnetic (sign +1) or electric (sign -1) currents of every source
// box containing (i,j,k); comp_base is 3 for M and 0 for J.
template <typename T>
__device__ __forceinline__ void add_sources(const SourceList<T>& src, int i, int j, int k,
                                            int comp_base, T S, T C, T& f0, T& f1, T& f2,
                                            bool subtract) {
    for (int q = 0; q < src.n; q++) {
        const DevSource<T>& s = src.s[q];
        int li = i - s.i0, lj = j - s.j0, lk = k - s.k0;
        if ((unsigned)li >= (unsigned)s.I || (unsigned)lj >= (unsigned)s.J ||
            (unsigned)lk >= (unsigned)s.K)
            continue;
        long long m = 2 * (((long long)li * s.J + lj) * s.K + lk);
        const T* c0 = s.comp[comp_base + 0];
        const T* c1 = s.comp[comp_base + 1];
        const T* c2 = s.comp[comp_base + 2];
        if (subtract) {
            if (c0) f0 = f0 - (S * c0[m] + C * c0[m + 1]);
            if (c1) f1 = f1 - (S * c1[m] + C * c1[m + 1]);
            if (c2) f2 = f2 - (S * c2[m] + C * c2[m + 1]);
        } else {
            if (c0) f0 = f0 + (S * c0[m] + C * c0[m + 1]);
            if (c1) f1 = f1 + (S * c1[m] + C * c1[m + 1]);
            if (c2) f2 = f2 + (S * c2[m] + C * c2[m + 1]);
        }
    }
}

// Value of the H ghost below the min face from the boundary rule; `first` is
// H at index 0 on that axis, `wrap` H at the last index (periodic).
template <typename T>
__device__ __forceinline__ T h_min_ghost(char bc, T first, T wrap) {
    if (bc == '0') return T(0);
    if (bc == 'E') return -first;
    if (bc == 'H') return first;
    return wrap;
}

// ------------------------------------------------------ whole-cell updates
// The H update of cell (i, j, k) in place, with its E neighbours read from the
// fields (max-face ghosts from the boundary rule, periodic wrap otherwise) and
// the magnetic currents of the step g.step_tab[*step_ctr + off].
template <typename T>
__device__ __forceinline__ void cell_update_H(const GridView<T>& g, const Fields<T>& f,
                                              const SourceList<T>& src, const long long* step_ctr,
                                              int off, int i, int j, int k) {
    const long long p = (long long)i * g.plane + (long long)j * g.px + k;
    const T *Ex = f.c[0], *Ey = f.c[1], *Ez = f.c[2];
    const bool px_ = g.bc[0] != '0' && g.bc[0] != 'E' && g.bc[0] != 'H';
    const bool py_ = g.bc[1] != '0' && g.bc[1] != 'E' && g.bc[1] != 'H';
    const bool pz_ = g.bc[2] != '0' && g.bc[2] != 'E' && g.bc[2] != 'H';
    HIn<T> e;
    e.ex = Ex[p]; e.ey = Ey[p]; e.ez = Ez[p];
    if (k + 1 < g.Nx) { e.ey_x = Ey[p + 1]; e.ez_x = Ez[p + 1]; }
    else if (px_) { e.ey_x = Ey[p - k]; e.ez_x = Ez[p - k]; }
    else { e.ey_x = T(0); e.ez_x = T(0); }
    if (j + 1 < g.Ny) { e.ex_y = Ex[p + g.px]; e.ez_y = Ez[p + g.px]; }
    else if (py_) { long long q = p - (long long)j * g.px; e.ex_y = Ex[q]; e.ez_y = Ez[q]; }
    else { e.ex_y = T(0); e.ez_y = T(0); }
    if (i + 1 < g.Nz) { e.ex_z = Ex[p + g.plane]; e.ey_z = Ey[p + g.plane]; }
    else if (pz_) { long long q = p - (long long)i * g.plane; e.ex_z = Ex[q]; e.ey_z = Ey[q]; }
    else { e.ex_z = T(0); e.ey_z = T(0); }
    T hx = f.c[3][p], hy = f.c[4][p], hz = f.c[5][p];
    h_cell<T>(g, i, j, k, p, e, hx, hy, hz, g.pml[0].psi, g.pml[0].psi, g.pml[1].psi,
              g.pml[1].psi, g.pml[2].psi, g.pml[2].psi, true);
    if (src.n) {
        double4 st = g.step_tab[*step_ctr + off];
        add_sources<T>(src, i, j, k, 3, T(st.x), T(st.y), hx, hy, hz, false);
    }
    f.c[3][p] = hx; f.c[4][p] = hy; f.c[5][p] = hz;
}

// The E update of cell (i, j, k) in place, with its H neighbours read from the
// fields (min-face ghosts from the boundary rule, periodic wrap otherwise) and
// the electric currents of the step.
template <typename T>
__device__ __forceinline__ void cell_update_E(const GridView<T>& g, const Fields<T>& f,
                                              const SourceList<T>& src, const long long* step_ctr,
                                              int off, int i, int j, int k) {
    const long long p = (long long)i * g.plane + (long long)j * g.px + k;
    const T *Hx = f.c[3], *Hy = f.c[4], *Hz = f.c[5];
    EIn<T> h;
    h.hx = Hx[p]; h.hy = Hy[p]; h.hz = Hz[p];
    if (k > 0) { h.hy_x = Hy[p - 1]; h.hz_x = Hz[p - 1]; }
    else {
        long long q = p + g.Nx - 1;
        h.hy_x = h_min_ghost<T>(g.bc[0], h.hy, Hy[q]);
        h.hz_x = h_min_ghost<T>(g.bc[0], h.hz, Hz[q]);
    }
    if (j > 0) { h.hx_y = Hx[p - g.px]; h.hz_y = Hz[p - g.px]; }
    else {
        long long q = p + (long long)(g.Ny - 1) * g.px;
        h.hx_y = h_min_ghost<T>(g.bc[1], h.hx, Hx[q]);
        h.hz_y = h_min_ghost<T>(g.bc[1], h.hz, Hz[q]);
    }
    if (i > 0) { h.hx_z = Hx[p - g.plane]; h.hy_z = Hy[p - g.plane]; }
    else {
        long long q = p + (long long)(g.Nz - 1) * g.plane;
        h.hx_z = h_min_ghost<T>(g.bc[2], h.hx, Hx[q]);
        h.hy_z = h_min_ghost<T>(g.bc[2], h.hy, Hy[q]);
    }
    T ex = f.c[0][p], ey = f.c[1][p], ez = f.c[2][p];
    T bx, by, bz;
    e_cell<T>(g, i, j, k, p, h, ex, ey, ez, g.pml[0].psi, g.pml[0].psi, g.pml[1].psi,
              g.pml[1].psi, g.pml[2].psi, g.pml[2].psi, bx, by, bz);
    if (src.n) {
        double4 st = g.step_tab[*step_ctr + off];
        add_sources<T>(src, i, j, k, 0, T(st.z), T(st.w), ex, ey, ez, true);
    }
    f.c[0][p] = ex; f.c[1][p] = ey; f.c[2][p] = ez;
}

}  // namespace fdtdb
