// zmarch_kernels.cu -- one fused time step (H half step, then E half step)
// per launch, each warp marching up a column of planes.
//
// Arithmetic per cell: src/fdtd.cpp:175-310 (H) and :503-669 (E), in the same
// association as the vector bodies (vec_body.cuh): curl scaled by R/d, CPML
// corrections in x, y, z order with psi <- c d + b psi and (psi - d) + d/kappa,
// sources after each half step, E beyond the max faces zero (PEC), the
// symmetry rule at the min faces (src/fdtd.cpp:141-173, :397-501).
//
// Work of one warp (single-warp CTA): a 60-cell segment x0 .. x0+59 of row j,
// for the planes i0 .. i1-1 of its z chunk.  Lane l holds the two cells
// c0 = x0 - 2 + 2l, c0 + 1 (one float2 / double2 per array): lanes 1..30 own
// the 60 cells; lane 0 computes H at x0 - 1 (the E update of cell x0 reads
// it) and lane 31 only supplies E at x0 + 60 (the H update of x0 + 59 reads
// it).  Per plane i the warp
//   * loads E(i+1) of rows j-1, j and j+1, H(i) of rows j-1 and j and the E
//     coefficients of row j -- E(i) of those rows and H(i-1) of row j are
//     still in registers from the previous plane;
//   * computes H(i) of row j and of row j-1 (the E update of row j reads Hx
//     and Hz there; row j-1 belongs to another warp, which stores it);
//   * computes E(i) of row j and stores H(i) and E(i) of row j.
// The first plane of a chunk also recomputes H(i0-1) of row j.  Every value a
// warp recomputes is read from the other field set, so the step reads set A
// (fields and CPML state) and writes set B: no warp waits for another.
// Each array is read from DRAM once per step; the halo rows and planes are L2
// hits.  Bodies: M = 0 for warps whose cells, halo included, lie in no CPML
// slab (no CPML code at all), M = -1 otherwise (run-time slab tests).
#include "kernels.h"
#include "vec_body.cuh"

namespace fdtdb {

namespace {

template <typename T>
struct Pair {
    T v[2];
};

template <typename T>
__device__ __forceinline__ Pair<T> pload(const T* p, bool ok) {
    Pair<T> r;
    if (ok) {
        // the read set is not written during the step: read-only cache path
        typename vecb::V16<T>::type v = __ldg(reinterpret_cast<const typename vecb::V16<T>::type*>(p));
        r.v[0] = v.x;
        r.v[1] = v.y;
    } else {
        r.v[0] = T(0);
        r.v[1] = T(0);
    }
    return r;
}

template <typename T>
__device__ __forceinline__ void pstore(T* p, T a, T b) {
    typename vecb::V16<T>::type v;
    v.x = a;
    v.y = b;
    *reinterpret_cast<typename vecb::V16<T>::type*>(p) = v;
}

// CPML slots of one cell pair: x per cell (-1: none), y per row, z per plane.
struct Slots {
    int lx[2], ly, lz;
};

template <typename T, int M>
__device__ __forceinline__ Slots slots_of(const GridView<T>& g, int i, int j, int c0, bool ok) {
    Slots s;
    s.ly = s.lz = -1;
    s.lx[0] = s.lx[1] = -1;
    if (M == 0 || !ok) return s;
    s.ly = slab_local(g.pml[1], j, false);
    s.lz = slab_local(g.pml[2], i + g.pml[2].off, true);
#pragma unroll
    for (int e = 0; e < 2; e++) {
        const int k = c0 + e;
        s.lx[e] = (k >= 0 && k < g.Nx) ? slab_local(g.pml[0], k, false) : -1;
    }
    return s;
}

// psi of the H update (q = 0, 1) or the E update (q = 2, 3) of one cell
// pair, all three axes: a[axis][q & 1][cell].
template <typename T>
struct Psi {
    T a[3][2][2];
};

template <typename T, int M>
__device__ __forceinline__ void psi_load(const GridView<T>& g, const Slots& s, int i, int j, int c0,
                                         int q0, bool need0, bool need1, Psi<T>& p) {
    if (M == 0) return;
    const int Ny = g.Ny, px = g.px;
#pragma unroll
    for (int e = 0; e < 2; e++)
        if (s.lx[e] >= 0) {
            const int o = (i * Ny + j) * g.pml[0].wsum + s.lx[e];
            if (need0) p.a[0][0][e] = ld(g.pml[0].psi[q0] + o);
            if (need1) p.a[0][1][e] = ld(g.pml[0].psi[q0 + 1] + o);
        }
    if (s.ly >= 0) {
        const int o = (i * g.pml[1].wsum + s.ly) * px + c0;
        if (need0) { Pair<T> t = pload<T>(g.pml[1].psi[q0] + o, true); p.a[1][0][0] = t.v[0]; p.a[1][0][1] = t.v[1]; }
        if (need1) { Pair<T> t = pload<T>(g.pml[1].psi[q0 + 1] + o, true); p.a[1][1][0] = t.v[0]; p.a[1][1][1] = t.v[1]; }
    }
    if (s.lz >= 0) {
        const int o = (s.lz * Ny + j) * px + c0;
        if (need0) { Pair<T> t = pload<T>(g.pml[2].psi[q0] + o, true); p.a[2][0][0] = t.v[0]; p.a[2][0][1] = t.v[1]; }
        if (need1) { Pair<T> t = pload<T>(g.pml[2].psi[q0 + 1] + o, true); p.a[2][1][0] = t.v[0]; p.a[2][1][1] = t.v[1]; }
    }
}

template <typename T, int M>
__device__ __forceinline__ void psi_store(const GridView<T>& g, const Slots& s, int i, int j, int c0,
                                          int q0, const Psi<T>& p) {
    if (M == 0) return;
    const int Ny = g.Ny, px = g.px;
#pragma unroll
    for (int e = 0; e < 2; e++)
        if (s.lx[e] >= 0) {
            const int o = (i * Ny + j) * g.pml[0].wsum + s.lx[e];
            g.pml[0].psi[q0][o] = p.a[0][0][e];
            g.pml[0].psi[q0 + 1][o] = p.a[0][1][e];
        }
    if (s.ly >= 0) {
        const int o = (i * g.pml[1].wsum + s.ly) * px + c0;
        pstore<T>(g.pml[1].psi[q0] + o, p.a[1][0][0], p.a[1][0][1]);
        pstore<T>(g.pml[1].psi[q0 + 1] + o, p.a[1][1][0], p.a[1][1][1]);
    }
    if (s.lz >= 0) {
        const int o = (s.lz * Ny + j) * px + c0;
        pstore<T>(g.pml[2].psi[q0] + o, p.a[2][0][0], p.a[2][0][1]);
        pstore<T>(g.pml[2].psi[q0 + 1] + o, p.a[2][1][0], p.a[2][1][1]);
    }
}

// E of one row of a plane: ex, ey, ez per cell of the pair.
template <typename T>
struct ERow {
    T x[2], y[2], z[2];
};

// H of one cell pair: in the old values, out the new ones.  e: E of the row,
// e_xn: Ey, Ez at c0 + 2 (first cell of the next lane), ejx/ejz: Ex, Ez of
// row j+1, eix/eiy: Ex, Ey of plane i+1, mu: dt/mu per cell.  The CPML state
// is updated in p (H slots).  Sources of row (i, j) are added when srcb.
template <typename T, int M>
__device__ __forceinline__ void h_pair(const GridView<T>& g, const SourceList<T>& src, int i, int j,
                                       int c0, const ERow<T>& e, T ey_n, T ez_n, const T (&ejx)[2],
                                       const T (&ejz)[2], const T (&eix)[2], const T (&eiy)[2],
                                       const T (&mx)[2], const T (&my)[2], const T (&mz)[2],
                                       const Slots& s, Psi<T>& p, bool srcb, T SH, T CH,
                                       T (&hx)[2], T (&hy)[2], T (&hz)[2]) {
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const T eyx = c == 0 ? e.y[1] : ey_n;
        const T ezx = c == 0 ? e.z[1] : ez_n;
        const T dEzdy = g.ody * (ejz[c] - e.z[c]);
        const T dEydz = g.odz * (eiy[c] - e.y[c]);
        const T dExdz = g.odz * (eix[c] - e.x[c]);
        const T dEzdx = g.odx * (ezx - e.z[c]);
        const T dEydx = g.odx * (eyx - e.y[c]);
        const T dExdy = g.ody * (ejx[c] - e.x[c]);
        T Hx = hx[c] + mx[c] * (dEydz - dEzdy);
        T Hy = hy[c] + my[c] * (dEzdx - dExdz);
        T Hz = hz[c] + mz[c] * (dExdy - dEydx);
        if (M != 0) {
            if (s.lx[c] >= 0) {
                const PmlAxis<T>& P = g.pml[0];
                const int l = s.lx[c];
                const T kv = ld(P.kinvH + l), bv = ld(P.bH + l), cv = ld(P.cH + l);
                p.a[0][0][c] = cv * dEydx + bv * p.a[0][0][c];
                p.a[0][1][c] = cv * dEzdx + bv * p.a[0][1][c];
                Hz = Hz - mz[c] * ((p.a[0][0][c] - dEydx) + dEydx * kv);
                Hy = Hy + my[c] * ((p.a[0][1][c] - dEzdx) + dEzdx * kv);
            }
            if (s.ly >= 0) {
                const PmlAxis<T>& P = g.pml[1];
                const T kv = ld(P.kinvH + s.ly), bv = ld(P.bH + s.ly), cv = ld(P.cH + s.ly);
                p.a[1][0][c] = cv * dExdy + bv * p.a[1][0][c];
                p.a[1][1][c] = cv * dEzdy + bv * p.a[1][1][c];
                Hz = Hz + mz[c] * ((p.a[1][0][c] - dExdy) + dExdy * kv);
                Hx = Hx - mx[c] * ((p.a[1][1][c] - dEzdy) + dEzdy * kv);
            }
            if (s.lz >= 0) {
                const PmlAxis<T>& P = g.pml[2];
                const T kv = ld(P.kinvH + s.lz), bv = ld(P.bH + s.lz), cv = ld(P.cH + s.lz);
                p.a[2][0][c] = cv * dExdz + bv * p.a[2][0][c];
                p.a[2][1][c] = cv * dEydz + bv * p.a[2][1][c];
                Hx = Hx + mx[c] * ((p.a[2][1][c] - dEydz) + dEydz * kv);
                Hy = Hy - my[c] * ((p.a[2][0][c] - dExdz) + dExdz * kv);
            }
        }
        const int k = c0 + c;
        if (srcb && k >= 0 && k < g.Nx) add_sources<T>(src, i, j, k, 3, SH, CH, Hx, Hy, Hz, false);
        hx[c] = Hx; hy[c] = Hy; hz[c] = Hz;
    }
}

// dt/mu of a cell pair (uniform mu: the scalar of each component).
template <typename T>
__device__ __forceinline__ void mu_pair(const GridView<T>& g, int o, bool ok, T (&mx)[2], T (&my)[2],
                                        T (&mz)[2]) {
    if (g.bHarr[0] != nullptr) {
        Pair<T> a = pload<T>(g.bHarr[0] + o, ok), b = pload<T>(g.bHarr[1] + o, ok),
                c = pload<T>(g.bHarr[2] + o, ok);
#pragma unroll
        for (int e = 0; e < 2; e++) { mx[e] = a.v[e]; my[e] = b.v[e]; mz[e] = c.v[e]; }
    } else {
#pragma unroll
        for (int e = 0; e < 2; e++) { mx[e] = g.bH[0]; my[e] = g.bH[1]; mz[e] = g.bH[2]; }
    }
}

template <typename T, int M>
__device__ __forceinline__ void zm_body(const GridView<T>& ga, const GridView<T>& gb,
                                        const Fields<T>& fa, const Fields<T>& fb,
                                        const SourceList<T>& src, const long long* step_ctr,
                                        int off, int x0, int j, int i0, int i1, int lane) {
    constexpr unsigned FULL = 0xffffffffu;
    const int Nx = ga.Nx, Ny = ga.Ny, Nz = ga.Nz, px = ga.px;
    const int c0 = x0 - 2 + 2 * lane;
    // a lane's pair is in the row when its first cell is (rows are padded to
    // an even pitch, so the second cell never leaves the row's storage)
    const bool ok = c0 >= 0 && c0 < Nx;
    const bool own = ok && lane >= 1 && lane <= 30;
    const bool hasj1 = j + 1 < Ny;
    const bool hasjm = j > 0;
    const long long plane = ga.plane;
    const int rj = j * px + c0;   // offset of the pair within a plane

    // step constants of the sources
    T SH = T(0), CH = T(0), SE = T(0), CE = T(0);
    if (src.n) {
        const double4 st = ga.step_tab[*step_ctr + off];
        SH = T(st.x); CH = T(st.y); SE = T(st.z); CE = T(st.w);
    }
    // sources near this warp's cells in plane i, rows [ja, jb)
    auto src_near = [&](int comp_base, int i, int ja, int jb) {
        return src.n != 0 && vecb::sources_touch<T>(src, comp_base, i, ja, jb, x0 - 2, x0 + 62);
    };

    // E(i) of rows j-1, j, j+1 (the plane below the one the loop loads next)
    ERow<T> em, e0;
    T e1x[2], e1z[2];
    auto load_erow = [&](ERow<T>& r, int i, int jj, bool row_ok) {
        const bool q = ok && row_ok && i < Nz;
        const long long o = (long long)i * plane + (long long)jj * px + c0;
        Pair<T> a = pload<T>(fa.c[0] + o, q), b = pload<T>(fa.c[1] + o, q), c = pload<T>(fa.c[2] + o, q);
        r.x[0] = a.v[0]; r.x[1] = a.v[1]; r.y[0] = b.v[0]; r.y[1] = b.v[1]; r.z[0] = c.v[0]; r.z[1] = c.v[1];
    };
    auto load_xz = [&](T (&x)[2], T (&z)[2], int i, int jj, bool row_ok) {
        const bool q = ok && row_ok && i < Nz;
        const long long o = (long long)i * plane + (long long)jj * px + c0;
        Pair<T> a = pload<T>(fa.c[0] + o, q), c = pload<T>(fa.c[2] + o, q);
        x[0] = a.v[0]; x[1] = a.v[1]; z[0] = c.v[0]; z[1] = c.v[1];
    };
    auto next_lane = [&](const ERow<T>& r, T& ey_n, T& ez_n) {
        ey_n = __shfl_down_sync(FULL, r.y[0], 1);
        ez_n = __shfl_down_sync(FULL, r.z[0], 1);
    };

    load_erow(e0, i0, j, true);
    load_erow(em, i0, j - 1, hasjm);
    load_xz(e1x, e1z, i0, j + 1, hasj1);

    // H(i0 - 1) of row j: Hx and Hy, read by the E update of plane i0
    T hpx[2], hpy[2];
    if (i0 > 0) {
        const int i = i0 - 1;
        ERow<T> e;
        T ejx[2], ejz[2], hx[2], hy[2], hz[2], mx[2], my[2], mz[2];
        load_erow(e, i, j, true);
        load_xz(ejx, ejz, i, j + 1, hasj1);
        const long long o = (long long)i * plane + rj;
        Pair<T> a = pload<T>(fa.c[3] + o, ok), b = pload<T>(fa.c[4] + o, ok);
        hx[0] = a.v[0]; hx[1] = a.v[1]; hy[0] = b.v[0]; hy[1] = b.v[1]; hz[0] = hz[1] = T(0);
        mu_pair<T>(ga, (int)o, ok, mx, my, mz);
        const Slots s = slots_of<T, M>(ga, i, j, c0, ok);
        Psi<T> p;
        psi_load<T, M>(ga, s, i, j, c0, 0, true, true, p);
        T ey_n, ez_n;
        next_lane(e, ey_n, ez_n);
        const T eix[2] = {e0.x[0], e0.x[1]}, eiy[2] = {e0.y[0], e0.y[1]};
        h_pair<T, M>(ga, src, i, j, c0, e, ey_n, ez_n, ejx, ejz, eix, eiy, mx, my, mz, s, p,
                     src_near(3, i, j, j + 1), SH, CH, hx, hy, hz);
        hpx[0] = hx[0]; hpx[1] = hx[1]; hpy[0] = hy[0]; hpy[1] = hy[1];
    } else {
        hpx[0] = hpx[1] = hpy[0] = hpy[1] = T(0);
    }

    // CPML slots that do not change along the march: x per lane, y per row
    Slots s_own = slots_of<T, M>(ga, 0, j, c0, ok);
    Slots s_hal = slots_of<T, M>(ga, 0, j - 1, c0, ok && hasjm);

    for (int i = i0; i < i1; i++) {
        // ---- loads of the plane: E(i+1) of rows j-1, j, j+1, H(i) of rows
        // j-1, j, the E coefficients, the CPML state of both rows
        ERow<T> nm, n0;
        T n1x[2], n1z[2];
        load_erow(n0, i + 1, j, true);
        load_erow(nm, i + 1, j - 1, hasjm);
        load_xz(n1x, n1z, i + 1, j + 1, hasj1);
        const long long o = (long long)i * plane + rj;
        T hx[2], hy[2], hz[2], gx[2], gz[2];
        {
            Pair<T> a = pload<T>(fa.c[3] + o, ok), b = pload<T>(fa.c[4] + o, ok),
                    c = pload<T>(fa.c[5] + o, ok);
            hx[0] = a.v[0]; hx[1] = a.v[1]; hy[0] = b.v[0]; hy[1] = b.v[1]; hz[0] = c.v[0]; hz[1] = c.v[1];
            Pair<T> d = pload<T>(fa.c[3] + o - px, ok && hasjm), f = pload<T>(fa.c[5] + o - px, ok && hasjm);
            gx[0] = d.v[0]; gx[1] = d.v[1]; gz[0] = f.v[0]; gz[1] = f.v[1];
        }
        T bx[2], by[2], bz[2];
        {
            Pair<T> a = pload<T>(ga.bE[0] + o, ok), b = pload<T>(ga.bE[1] + o, ok),
                    c = pload<T>(ga.bE[2] + o, ok);
            bx[0] = a.v[0]; bx[1] = a.v[1]; by[0] = b.v[0]; by[1] = b.v[1]; bz[0] = c.v[0]; bz[1] = c.v[1];
        }
        Slots s = s_own, sm = s_hal;
        if (M != 0) {
            const int lz = slab_local(ga.pml[2], i + ga.pml[2].off, true);
            s.lz = ok ? lz : -1;
            sm.lz = ok && hasjm ? lz : -1;
        }
        Psi<T> ph, pe, pm;
        psi_load<T, M>(ga, s, i, j, c0, 0, true, true, ph);
        psi_load<T, M>(ga, s, i, j, c0, 2, true, true, pe);
        psi_load<T, M>(ga, sm, i, j - 1, c0, 0, true, true, pm);
        T mx[2], my[2], mz[2], gmx[2], gmy[2], gmz[2];
        mu_pair<T>(ga, (int)o, ok, mx, my, mz);
        mu_pair<T>(ga, (int)(o - px), ok && hasjm, gmx, gmy, gmz);

        // ---- H(i) of row j, then of row j-1 (Hx, Hz only are used)
        T ey_n, ez_n;
        next_lane(e0, ey_n, ez_n);
        {
            const T eix[2] = {n0.x[0], n0.x[1]}, eiy[2] = {n0.y[0], n0.y[1]};
            h_pair<T, M>(ga, src, i, j, c0, e0, ey_n, ez_n, e1x, e1z, eix, eiy, mx, my, mz, s, ph,
                         src_near(3, i, j, j + 1), SH, CH, hx, hy, hz);
        }
        if (hasjm) {
            T my_ey_n, my_ez_n;
            next_lane(em, my_ey_n, my_ez_n);
            const T ejx[2] = {e0.x[0], e0.x[1]}, ejz[2] = {e0.z[0], e0.z[1]};
            const T eix[2] = {nm.x[0], nm.x[1]}, eiy[2] = {nm.y[0], nm.y[1]};
            T gy[2] = {T(0), T(0)};
            h_pair<T, M>(ga, src, i, j - 1, c0, em, my_ey_n, my_ez_n, ejx, ejz, eix, eiy, gmx, gmy,
                         gmz, sm, pm, src_near(3, i, j - 1, j), SH, CH, gx, gy, gz);
        }

        // ---- E(i) of row j
        // Hy, Hz at k - 1: the previous cell, across lanes by a shuffle
        T hy_p = __shfl_up_sync(FULL, hy[1], 1), hz_p = __shfl_up_sync(FULL, hz[1], 1);
        const bool lossy = ga.aE[0] != nullptr;
        T ax[2], ay[2], az[2];
        if (lossy) {
            Pair<T> a = pload<T>(ga.aE[0] + o, ok), b = pload<T>(ga.aE[1] + o, ok), c = pload<T>(ga.aE[2] + o, ok);
            ax[0] = a.v[0]; ax[1] = a.v[1]; ay[0] = b.v[0]; ay[1] = b.v[1]; az[0] = c.v[0]; az[1] = c.v[1];
        }
        const bool srce = src_near(0, i, j, j + 1);
        T ex[2], ey[2], ez[2];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int k = c0 + c;
            T hyx = c == 0 ? hy_p : hy[0];
            T hzx = c == 0 ? hz_p : hz[0];
            if (k == 0) { hyx = h_min_ghost<T>(ga.bc[0], hy[c], T(0)); hzx = h_min_ghost<T>(ga.bc[0], hz[c], T(0)); }
            T hxj = gx[c], hzj = gz[c];
            if (!hasjm) { hxj = h_min_ghost<T>(ga.bc[1], hx[c], T(0)); hzj = h_min_ghost<T>(ga.bc[1], hz[c], T(0)); }
            T hxi = hpx[c], hyi = hpy[c];
            if (i == 0) { hxi = h_min_ghost<T>(ga.bc[2], hx[c], T(0)); hyi = h_min_ghost<T>(ga.bc[2], hy[c], T(0)); }
            const T dHzdy = ga.ody * (hz[c] - hzj);
            const T dHydz = ga.odz * (hy[c] - hyi);
            const T dHxdz = ga.odz * (hx[c] - hxi);
            const T dHzdx = ga.odx * (hz[c] - hzx);
            const T dHydx = ga.odx * (hy[c] - hyx);
            const T dHxdy = ga.ody * (hx[c] - hxj);
            T Ex, Ey, Ez;
            if (lossy) {
                Ex = ax[c] * e0.x[c] + (dHzdy - dHydz) * bx[c];
                Ey = ay[c] * e0.y[c] + (dHxdz - dHzdx) * by[c];
                Ez = az[c] * e0.z[c] + (dHydx - dHxdy) * bz[c];
            } else {
                Ex = e0.x[c] + (dHzdy - dHydz) * bx[c];
                Ey = e0.y[c] + (dHxdz - dHzdx) * by[c];
                Ez = e0.z[c] + (dHydx - dHxdy) * bz[c];
            }
            if (M != 0) {
                if (s.lx[c] >= 0) {
                    const PmlAxis<T>& P = ga.pml[0];
                    const int l = s.lx[c];
                    const T kv = ld(P.kinvE + l), bv = ld(P.bE + l), cv = ld(P.cE + l);
                    pe.a[0][0][c] = cv * dHydx + bv * pe.a[0][0][c];
                    pe.a[0][1][c] = cv * dHzdx + bv * pe.a[0][1][c];
                    Ez = Ez + ((pe.a[0][0][c] - dHydx) + dHydx * kv) * bz[c];
                    Ey = Ey - ((pe.a[0][1][c] - dHzdx) + dHzdx * kv) * by[c];
                }
                if (s.ly >= 0) {
                    const PmlAxis<T>& P = ga.pml[1];
                    const T kv = ld(P.kinvE + s.ly), bv = ld(P.bE + s.ly), cv = ld(P.cE + s.ly);
                    pe.a[1][0][c] = cv * dHxdy + bv * pe.a[1][0][c];
                    pe.a[1][1][c] = cv * dHzdy + bv * pe.a[1][1][c];
                    Ez = Ez - ((pe.a[1][0][c] - dHxdy) + dHxdy * kv) * bz[c];
                    Ex = Ex + ((pe.a[1][1][c] - dHzdy) + dHzdy * kv) * bx[c];
                }
                if (s.lz >= 0) {
                    const PmlAxis<T>& P = ga.pml[2];
                    const T kv = ld(P.kinvE + s.lz), bv = ld(P.bE + s.lz), cv = ld(P.cE + s.lz);
                    pe.a[2][0][c] = cv * dHxdz + bv * pe.a[2][0][c];
                    pe.a[2][1][c] = cv * dHydz + bv * pe.a[2][1][c];
                    Ex = Ex - ((pe.a[2][1][c] - dHydz) + dHydz * kv) * bx[c];
                    Ey = Ey + ((pe.a[2][0][c] - dHxdz) + dHxdz * kv) * by[c];
                }
            }
            if (srce && k < Nx) add_sources<T>(src, i, j, k, 0, SE, CE, Ex, Ey, Ez, true);
            ex[c] = Ex; ey[c] = Ey; ez[c] = Ez;
        }

        // ---- stores of row j (the 60 owned cells)
        if (own) {
            pstore<T>(fb.c[3] + o, hx[0], hx[1]);
            pstore<T>(fb.c[4] + o, hy[0], hy[1]);
            pstore<T>(fb.c[5] + o, hz[0], hz[1]);
            pstore<T>(fb.c[0] + o, ex[0], ex[1]);
            pstore<T>(fb.c[1] + o, ey[0], ey[1]);
            pstore<T>(fb.c[2] + o, ez[0], ez[1]);
            psi_store<T, M>(gb, s, i, j, c0, 0, ph);
            psi_store<T, M>(gb, s, i, j, c0, 2, pe);
        }

        // ---- the next plane
        hpx[0] = hx[0]; hpx[1] = hx[1]; hpy[0] = hy[0]; hpy[1] = hy[1];
        e0 = n0;
        em = nm;
        e1x[0] = n1x[0]; e1x[1] = n1x[1]; e1z[0] = n1z[0]; e1z[1] = n1z[1];
    }
}

}  // namespace

#ifndef ZM_MINB32
#define ZM_MINB32 16
#endif
#define ZM_MINB(T) (sizeof(T) == 8 ? 0 : ZM_MINB32)

// One time step: fields and CPML state read from (ga, fa), written to (gb, fb).
// grid = (60-cell segments per row, rows, z chunks of zc planes); block = 32.
template <typename T>
__global__ void __launch_bounds__(32, ZM_MINB(T))
k_step_zmarch(GridView<T> ga, GridView<T> gb, Fields<T> fa, Fields<T> fb, SourceList<T> src,
              const long long* step_base, int off, int zc) {
    const int x0 = blockIdx.x * 60;
    const int j = blockIdx.y;
    const int i0 = blockIdx.z * zc;
    const int i1 = min(i0 + zc, ga.Nz);
    // slab-free warp: cells x0-2 .. x0+61, rows j-1 .. j, planes i0-1 .. i1-1
    const PmlAxis<T>& PX = ga.pml[0];
    const PmlAxis<T>& PY = ga.pml[1];
    const PmlAxis<T>& PZ = ga.pml[2];
    const bool xin = x0 - 2 >= PX.w0 && x0 + 61 < PX.edge_max;
    const bool yin = (j > 0 ? j - 1 : 0) >= PY.w0 && j < PY.edge_max;
    const int zlo = (i0 > 0 ? i0 - 1 : 0) + PZ.off, zhi = i1 - 1 + PZ.off;
    const bool zin = zlo >= PZ.w0 && (PZ.w1 == 0 || zhi <= PZ.edge_max);
    if (xin && yin && zin)
        zm_body<T, 0>(ga, gb, fa, fb, src, step_base, off, x0, j, i0, i1, threadIdx.x);
    else
        zm_body<T, -1>(ga, gb, fa, fb, src, step_base, off, x0, j, i0, i1, threadIdx.x);
}

template <typename T>
cudaError_t launch_step_zmarch(const GridView<T>& ga, const GridView<T>& gb, T* const* fa,
                               T* const* fb, const SourceList<T>& src, const long long* step_base,
                               int off, int zc, cudaStream_t st) {
    Fields<T> a, b;
    for (int c = 0; c < 6; c++) { a.c[c] = fa[c]; b.c[c] = fb[c]; }
    if (zc <= 0) zc = ga.Nz;
    dim3 grid((ga.Nx + 59) / 60, ga.Ny, (ga.Nz + zc - 1) / zc);
    k_step_zmarch<T><<<grid, 32, 0, st>>>(ga, gb, a, b, src, step_base, off, zc);
    return cudaGetLastError();
}

int zmarch_chunk(int Nx, int Ny, int Nz, int sms) {
    // enough single-warp CTAs for about 32 per SM, chunks of at least 4 planes
    const long long cols = (long long)((Nx + 59) / 60) * Ny;
    const long long want = 32LL * (sms > 0 ? sms : 148);
    int nchunk = (int)((want + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    int zc = (Nz + nchunk - 1) / nchunk;
    if (zc < 4) zc = 4;
    if (zc > Nz) zc = Nz;
    return zc;
}

template cudaError_t launch_step_zmarch<float>(const GridView<float>&, const GridView<float>&,
                                               float* const*, float* const*,
                                               const SourceList<float>&, const long long*, int, int,
                                               cudaStream_t);
template cudaError_t launch_step_zmarch<double>(const GridView<double>&, const GridView<double>&,
                                                double* const*, double* const*,
                                                const SourceList<double>&, const long long*, int,
                                                int, cudaStream_t);

}  // namespace fdtdb
