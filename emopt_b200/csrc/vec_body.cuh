// vec_body.cuh -- per-warp bodies of the vector H and E half-steps.
//
// The same in-place update as k_update_H / k_update_E (src/fdtd.cpp:121-367
// and :369-755).  One warp updates 32 consecutive V-vectors (V = 2 cells,
// float2 / double2) of row j of plane i, starting at vector 32 * xb; lane
// `lane` owns cells k0 .. k0+V-1 with k0 = (32 xb + lane) V.  Every field,
// coefficient and y/z-slab CPML access is one aligned vector load or store
// (rows are 128-byte aligned, px is a multiple of 32).  The x neighbour across
// the vector boundary comes from the adjacent lane with a warp shuffle; only
// the last lane (first lane for the E update) loads it separately, so all 32
// lanes must call the body together.  Each thread issues all of its loads
// before any dependent instruction; the source test is made once per warp.
// The source coefficients of the step are g.step_tab[*step_ctr + off].
// Used by the single-solve kernels (vec_kernels.cu) and the batched serving
// kernels (serve_kernels.cu).  Requires non-periodic boundaries.  Built with
// FDTD_BOUNDS_CHECK, every index a lane computes is checked against its
// array first; a lane out of range records the site (GridView::chk) and
// skips its accesses.  In a z slab
// of a distributed solve (g.zlo / g.zhi) the neighbour plane across an inner
// slab face is read through g.zhalo (the slab's halo plane, or the
// neighbouring slab's boundary plane on the same device), and the z CPML
// index is taken at the global plane i + g.pml[2].off.
#pragma once

#include "cell.cuh"

namespace fdtdb {

namespace vecb {


// Two consecutive x cells per thread: float2 (8 B) or double2 (16 B) accesses.
template <typename T>
struct V16;
template <>
struct V16<float> {
    using type = float2;
    static constexpr int N = 2;
};
template <>
struct V16<double> {
    using type = double2;
    static constexpr int N = 2;
};

template <typename T>
__device__ __forceinline__ void vload(T (&d)[V16<T>::N], const T* p) {
    typename V16<T>::type v = __ldg(reinterpret_cast<const typename V16<T>::type*>(p));
    d[0] = v.x;
    d[1] = v.y;
}

template <typename T>
__device__ __forceinline__ void vzero(T (&d)[V16<T>::N]) {
#pragma unroll
    for (int e = 0; e < V16<T>::N; e++) d[e] = T(0);
}

template <typename T>
__device__ __forceinline__ void vstore(T* p, const T (&d)[V16<T>::N]) {
    typename V16<T>::type v;
    v.x = d[0];
    v.y = d[1];
    *reinterpret_cast<typename V16<T>::type*>(p) = v;
}

// Does a source box with a non-zero component among comp_base..comp_base+2
// touch rows [j0, j1), columns [k0, k1) of plane i?
template <typename T>
__device__ __forceinline__ bool sources_touch(const SourceList<T>& src, int comp_base, int i,
                                              int j0, int j1, int k0, int k1) {
    // the box of all sources of this half step first: a few comparisons on
    // kernel parameters reject almost every warp
    const int* b = src.box[comp_base / 3];
    if (i < b[0] || i >= b[1] || j1 <= b[2] || j0 >= b[3] || k1 <= b[4] || k0 >= b[5]) return false;
    bool hit = false;
    for (int q = 0; q < src.n; q++) {
        const DevSource<T>& s = src.s[q];
        const bool drives = s.comp[comp_base] || s.comp[comp_base + 1] || s.comp[comp_base + 2];
        hit |= drives && i >= s.i0 && i < s.i0 + s.I && s.j0 < j1 && s.j0 + s.J > j0 &&
               s.k0 < k1 && s.k0 + s.K > k0;
    }
    return hit;
}

// Does the warp that updates row j of plane i, vectors 32 xb .. 32 xb + 31,
// touch no CPML slab and no source box of the half step (comp_base 3: H
// sources, 0: E sources)?  Then the body built without CPML and source code
// (GEN = false) computes the same values in the same order.
template <typename T>
__device__ __forceinline__ bool plain_warp(const GridView<T>& g, const SourceList<T>& src,
                                           int comp_base, int i, int j, int xb) {
    constexpr int V = V16<T>::N;
    if (slab_local(g.pml[2], i + g.pml[2].off, true) >= 0) return false;
    if (j < g.Ny && slab_local(g.pml[1], j, false) >= 0) return false;
    if (xb * 32 * V < g.pml[0].w0 || (xb + 1) * 32 * V - 1 >= g.pml[0].edge_max) return false;
    return !(src.n && sources_touch<T>(src, comp_base, i, j, j + 1, xb * 32 * V, (xb + 1) * 32 * V));
}

#ifdef FDTD_BOUNDS_CHECK
// Debug builds: is idx in [lo, hi)?  The first failure records its site.
template <typename T>
__device__ bool in_range(const GridView<T>& g, long long idx, long long lo, long long hi, int site) {
    if (idx >= lo && idx < hi) return true;
    if (g.chk) atomicCAS(g.chk, 0, site);
    return false;
}

// Every field vector (and scalar) the H body of this lane reads and writes.
template <typename T>
__device__ bool h_fields_ok(const GridView<T>& g, int i, int j, int k0, int lane, long long p) {
    constexpr int V = V16<T>::N;
    const long long plane = g.plane, top = (long long)g.Nz * plane;
    bool ok = in_range(g, p, 0, top - V + 1, 1);
    if (j + 1 < g.Ny) ok &= in_range(g, p + g.px, 0, top - V + 1, 2);
    if (i + 1 < g.Nz) ok &= in_range(g, p + plane, 0, top - V + 1, 3);
    else if (g.zhi) ok &= in_range(g, p - (long long)i * plane, 0, plane - V + 1, 3);
    if (lane == 31 && k0 + V < g.Nx) ok &= in_range(g, p + V, 0, top, 4);
    return ok;
}

// ... and the E body.
template <typename T>
__device__ bool e_fields_ok(const GridView<T>& g, int i, int j, int k0, int lane, long long p) {
    constexpr int V = V16<T>::N;
    const long long plane = g.plane, top = (long long)g.Nz * plane;
    bool ok = in_range(g, p, 0, top - V + 1, 11);
    if (j > 0) ok &= in_range(g, p - g.px, 0, top - V + 1, 12);
    if (i > 0) ok &= in_range(g, p - plane, 0, top - V + 1, 13);
    else if (g.zlo) ok &= in_range(g, p, 0, plane - V + 1, 13);
    if (lane == 0 && k0 > 0) ok &= in_range(g, p - 1, 0, top, 14);
    return ok;
}
#endif

}  // namespace vecb

// One warp task: the 32 vectors 32 xb .. 32 xb + 31 of row j of plane i.
// Each body is a load phase (every index, then every load the task needs,
// issued before any arithmetic) and a finish phase (the update and the
// stores) around a register set of the task (HTask / ETask).  A task writes
// only its own cells, and no array a half step writes is read by another
// task of that half step, so tasks may run in any order.
// GEN = false: the caller guarantees that the task touches no CPML slab; the
// CPML code is compiled out, and so is the source code unless SRC is set
// (default: SRC = GEN; with GEN = false the caller then also guarantees that
// no source box touches the task, vecb::plain_warp).
// SERVE: a served request's state gates the stores, and the H half step
// writes the fields it read into a snapshot set on a capture step
// (ServeGate).

template <typename T>
struct HTask {
    static constexpr int V = vecb::V16<T>::N;
    T ex[V], ey[V], ez[V], exj[V], ezj[V], exi[V], eyi[V], hx[V], hy[V], hz[V];
    T py0[V], py1[V], pz0[V], pz1[V], px0[V], px1[V];
    T mx[V], my[V], mz[V];
    T ey_n, ez_n;
    int lxs[V];
    int p, ly, lz;
    bool act;
    int sstate, scap;
};

template <typename T, bool GEN = true, bool SERVE = false>
__device__ __forceinline__ void h_load(const GridView<T>& g, const Fields<T>& f, int i, int j, int xb,
                                       int lane, const ServeGate<T>* sg, HTask<T>& t) {
    constexpr int V = vecb::V16<T>::N;
    const int m = xb * 32 + lane;
    const int k0 = m * V;
    const int Ny = g.Ny, Nz = g.Nz, px = g.px;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int lz0 = GEN ? slab_local(PZ, i + PZ.off, true) : -1;
    // lanes beyond the row still take part in the shuffles of the finish phase
    const bool act0 = j < Ny && k0 < g.Nx;
    t.p = act0 ? (i * Ny + j) * px + k0 : 0;
    const int ly0 = GEN ? slab_local(PY, j, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
    // a lane whose indices fall outside their arrays records the site and skips
    t.act = act0 && vecb::h_fields_ok(g, i, j, k0, lane, t.p);
    t.ly = (ly0 >= 0 && t.act && !vecb::in_range(g, (long long)(i * PY.wsum + ly0) * px + k0, 0,
                                                  (long long)Nz * PY.wsum * px - V + 1, 5)) ? -1 : ly0;
    t.lz = (lz0 >= 0 && t.act && !vecb::in_range(g, (long long)(lz0 * Ny + j) * px + k0, 0,
                                                  (long long)PZ.wsum * Ny * px - V + 1, 6)) ? -1 : lz0;
#else
    t.act = act0;
    t.ly = ly0;
    t.lz = lz0;
#endif
    // does any lane of the warp touch an x slab?  (the same for all lanes)
    const bool xw = GEN && (xb * 32 * V < PX.w0 || (xb + 1) * 32 * V - 1 >= PX.edge_max);

    // a served request's state and capture flag, read with the fields
    t.sstate = SERVE_RUN;
    t.scap = 0;
    if (SERVE) { t.sstate = __ldg(sg->state); t.scap = __ldg(sg->capture); }

    vecb::vzero<T>(t.ex); vecb::vzero<T>(t.ey); vecb::vzero<T>(t.ez); vecb::vzero<T>(t.exj);
    vecb::vzero<T>(t.ezj); vecb::vzero<T>(t.exi); vecb::vzero<T>(t.eyi);
    t.ey_n = T(0); t.ez_n = T(0);
    if (t.act) {
        const int q = t.p;
        vecb::vload<T>(t.ex, f.c[0] + q); vecb::vload<T>(t.ey, f.c[1] + q); vecb::vload<T>(t.ez, f.c[2] + q);
        if (j + 1 < Ny) { vecb::vload<T>(t.exj, f.c[0] + q + px); vecb::vload<T>(t.ezj, f.c[2] + q + px); }
        if (i + 1 < Nz) { vecb::vload<T>(t.exi, f.c[0] + q + Ny * px); vecb::vload<T>(t.eyi, f.c[1] + q + Ny * px); }
        else if (g.zhi) { vecb::vload<T>(t.exi, g.zhalo[0] + (q - i * Ny * px)); vecb::vload<T>(t.eyi, g.zhalo[1] + (q - i * Ny * px)); }
        vecb::vload<T>(t.hx, f.c[3] + q); vecb::vload<T>(t.hy, f.c[4] + q); vecb::vload<T>(t.hz, f.c[5] + q);
        if (lane == 31 && k0 + V < g.Nx) { t.ey_n = ld(f.c[1] + q + V); t.ez_n = ld(f.c[2] + q + V); }
        if (t.ly >= 0) {
            const int s = (i * PY.wsum + t.ly) * px + k0;
            vecb::vload<T>(t.py0, PY.psi[0] + s); vecb::vload<T>(t.py1, PY.psi[1] + s);
        }
        if (t.lz >= 0) {
            const int s = (t.lz * Ny + j) * px + k0;
            vecb::vload<T>(t.pz0, PZ.psi[0] + s); vecb::vload<T>(t.pz1, PZ.psi[1] + s);
        }
    }
#pragma unroll
    for (int e = 0; e < V; e++) t.lxs[e] = -1;
    if (xw) {
        const bool xs = t.act && (k0 < PX.w0 || k0 + V - 1 >= PX.edge_max);
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int k = k0 + e;
            t.lxs[e] = (xs && k < g.Nx) ? slab_local(PX, k, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
            if (t.lxs[e] >= 0 && !vecb::in_range(g, (long long)(i * Ny + j) * PX.wsum + t.lxs[e], 0,
                                                 (long long)Nz * Ny * PX.wsum, 7))
                t.lxs[e] = -1;
#endif
            if (t.lxs[e] >= 0) {
                const int s = (i * Ny + j) * PX.wsum + t.lxs[e];
                t.px0[e] = ld(PX.psi[0] + s); t.px1[e] = ld(PX.psi[1] + s);
            }
        }
    }
    if (g.bHarr[0] != nullptr && t.act) {
        vecb::vload<T>(t.mx, g.bHarr[0] + t.p); vecb::vload<T>(t.my, g.bHarr[1] + t.p);
        vecb::vload<T>(t.mz, g.bHarr[2] + t.p);
    } else {
#pragma unroll
        for (int e = 0; e < V; e++) { t.mx[e] = g.bH[0]; t.my[e] = g.bH[1]; t.mz[e] = g.bH[2]; }
    }
}

template <typename T, bool GEN = true, bool SERVE = false, bool SRC = GEN>
__device__ __forceinline__ void h_finish(const GridView<T>& g, const Fields<T>& f, const SourceList<T>& src,
                                         const long long* step_ctr, int off, int i, int j, int xb,
                                         int lane, const ServeGate<T>* sg, HTask<T>& t) {
    constexpr int V = vecb::V16<T>::N;
    constexpr unsigned FULL = 0xffffffffu;
    const int k0 = (xb * 32 + lane) * V;
    const int Ny = g.Ny, px = g.px;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const bool xw = GEN && (xb * 32 * V < PX.w0 || (xb + 1) * 32 * V - 1 >= PX.edge_max);
    if (SERVE) {
        // the whole warp leaves together (one state per request)
        if (!serve_running(t.sstate)) return;
        if ((t.scap == 1 || t.scap == 2) && t.act) {
            T* const* d = sg->snap[t.scap - 1];
            const int q = t.p;
            vecb::vstore<T>(d[0] + q, t.ex); vecb::vstore<T>(d[1] + q, t.ey); vecb::vstore<T>(d[2] + q, t.ez);
            vecb::vstore<T>(d[3] + q, t.hx); vecb::vstore<T>(d[4] + q, t.hy); vecb::vstore<T>(d[5] + q, t.hz);
        }
    }
    const bool srcb = SRC && src.n && vecb::sources_touch<T>(src, 3, i, j, j + 1,
                                                             xb * 32 * V, (xb + 1) * 32 * V);
    double4 st = make_double4(0, 0, 0, 0);
    if (srcb) st = g.step_tab[*step_ctr + off];

    // ---- x neighbour of the last cell: first cell of the next vector
    {
        const T a = __shfl_down_sync(FULL, t.ey[0], 1), b = __shfl_down_sync(FULL, t.ez[0], 1);
        if (lane != 31) { t.ey_n = a; t.ez_n = b; }
    }
    if (!t.act) return;
#pragma unroll
    for (int e = 0; e < V; e++) {
        const T eyx = e + 1 < V ? t.ey[e + 1] : t.ey_n;
        const T ezx = e + 1 < V ? t.ez[e + 1] : t.ez_n;
        const T dEzdy = g.ody * (t.ezj[e] - t.ez[e]);
        const T dEydz = g.odz * (t.eyi[e] - t.ey[e]);
        const T dExdz = g.odz * (t.exi[e] - t.ex[e]);
        const T dEzdx = g.odx * (ezx - t.ez[e]);
        const T dEydx = g.odx * (eyx - t.ey[e]);
        const T dExdy = g.ody * (t.exj[e] - t.ex[e]);
        T Hx = t.hx[e] + t.mx[e] * (dEydz - dEzdy);
        T Hy = t.hy[e] + t.my[e] * (dEzdx - dExdz);
        T Hz = t.hz[e] + t.mz[e] * (dExdy - dEydx);
        if (xw && t.lxs[e] >= 0) {
            const int l = t.lxs[e];
            const T kv = ld(PX.kinvH + l), bv = ld(PX.bH + l), cv = ld(PX.cH + l);
            t.px0[e] = cv * dEydx + bv * t.px0[e];
            t.px1[e] = cv * dEzdx + bv * t.px1[e];
            Hz = Hz - t.mz[e] * ((t.px0[e] - dEydx) + dEydx * kv);
            Hy = Hy + t.my[e] * ((t.px1[e] - dEzdx) + dEzdx * kv);
        }
        if (t.ly >= 0) {
            const int l = t.ly;
            const T kv = ld(PY.kinvH + l), bv = ld(PY.bH + l), cv = ld(PY.cH + l);
            t.py0[e] = cv * dExdy + bv * t.py0[e];
            t.py1[e] = cv * dEzdy + bv * t.py1[e];
            Hz = Hz + t.mz[e] * ((t.py0[e] - dExdy) + dExdy * kv);
            Hx = Hx - t.mx[e] * ((t.py1[e] - dEzdy) + dEzdy * kv);
        }
        if (t.lz >= 0) {
            const int l = t.lz;
            const T kv = ld(PZ.kinvH + l), bv = ld(PZ.bH + l), cv = ld(PZ.cH + l);
            t.pz0[e] = cv * dExdz + bv * t.pz0[e];
            t.pz1[e] = cv * dEydz + bv * t.pz1[e];
            Hx = Hx + t.mx[e] * ((t.pz1[e] - dEydz) + dEydz * kv);
            Hy = Hy - t.my[e] * ((t.pz0[e] - dExdz) + dExdz * kv);
        }
        if (srcb && k0 + e < g.Nx)
            add_sources<T>(src, i, j, k0 + e, 3, T(st.x), T(st.y), Hx, Hy, Hz, false);
        t.hx[e] = Hx; t.hy[e] = Hy; t.hz[e] = Hz;
    }
    const int q = t.p;
    vecb::vstore<T>(f.c[3] + q, t.hx); vecb::vstore<T>(f.c[4] + q, t.hy); vecb::vstore<T>(f.c[5] + q, t.hz);
    if (t.ly >= 0) {
        const int s = (i * PY.wsum + t.ly) * px + k0;
        vecb::vstore<T>(PY.psi[0] + s, t.py0); vecb::vstore<T>(PY.psi[1] + s, t.py1);
    }
    if (t.lz >= 0) {
        const int s = (t.lz * Ny + j) * px + k0;
        vecb::vstore<T>(PZ.psi[0] + s, t.pz0); vecb::vstore<T>(PZ.psi[1] + s, t.pz1);
    }
    if (xw) {
#pragma unroll
        for (int e = 0; e < V; e++)
            if (t.lxs[e] >= 0) {
                const int s = (i * Ny + j) * PX.wsum + t.lxs[e];
                PX.psi[0][s] = t.px0[e]; PX.psi[1][s] = t.px1[e];
            }
    }
}

template <typename T, bool GEN = true, bool SERVE = false, bool SRC = GEN>
__device__ __forceinline__ void vec_update_H(const GridView<T>& g, const Fields<T>& f,
                                             const SourceList<T>& src, const long long* step_ctr,
                                             int off, int i, int j, int xb, int lane,
                                             const ServeGate<T>* sg = nullptr) {
    HTask<T> t;
    h_load<T, GEN, SERVE>(g, f, i, j, xb, lane, sg, t);
    h_finish<T, GEN, SERVE, SRC>(g, f, src, step_ctr, off, i, j, xb, lane, sg, t);
}

template <typename T>
struct ETask {
    static constexpr int V = vecb::V16<T>::N;
    T hx[V], hy[V], hz[V], hxj[V], hzj[V], hxi[V], hyi[V];
    T ex[V], ey[V], ez[V], bx[V], by[V], bz[V];
    T py2[V], py3[V], pz2[V], pz3[V], px2[V], px3[V], ax[V], ay[V], az[V];
    T hy_p, hz_p;
    int lxs[V];
    int p, ly, lz;
    bool act;
    int sstate;
};

template <typename T, bool GEN = true, bool SERVE = false>
__device__ __forceinline__ void e_load(const GridView<T>& g, const Fields<T>& f, int i, int j, int xb,
                                       int lane, const ServeGate<T>* sg, ETask<T>& t) {
    constexpr int V = vecb::V16<T>::N;
    const int m = xb * 32 + lane;
    const int k0 = m * V;
    const int Ny = g.Ny, px = g.px;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int lz0 = GEN ? slab_local(PZ, i + PZ.off, true) : -1;
    const bool act0 = j < Ny && k0 < g.Nx;
    t.p = act0 ? (i * Ny + j) * px + k0 : 0;
    const int ly0 = GEN ? slab_local(PY, j, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
    t.act = act0 && vecb::e_fields_ok(g, i, j, k0, lane, t.p);
    t.ly = (ly0 >= 0 && t.act && !vecb::in_range(g, (long long)(i * PY.wsum + ly0) * px + k0, 0,
                                                  (long long)g.Nz * PY.wsum * px - V + 1, 15)) ? -1 : ly0;
    t.lz = (lz0 >= 0 && t.act && !vecb::in_range(g, (long long)(lz0 * Ny + j) * px + k0, 0,
                                                  (long long)PZ.wsum * Ny * px - V + 1, 16)) ? -1 : lz0;
#else
    t.act = act0;
    t.ly = ly0;
    t.lz = lz0;
#endif
    // does any lane of the warp touch an x slab?  (the same for all lanes)
    const bool xw = GEN && (xb * 32 * V < PX.w0 || (xb + 1) * 32 * V - 1 >= PX.edge_max);
    const bool lossy = g.aE[0] != nullptr;

    t.sstate = SERVE_RUN;
    if (SERVE) t.sstate = __ldg(sg->state);

    vecb::vzero<T>(t.hy); vecb::vzero<T>(t.hz);
    t.hy_p = T(0); t.hz_p = T(0);
    if (t.act) {
        const int q = t.p;
        vecb::vload<T>(t.hx, f.c[3] + q); vecb::vload<T>(t.hy, f.c[4] + q); vecb::vload<T>(t.hz, f.c[5] + q);
        vecb::vload<T>(t.ex, f.c[0] + q); vecb::vload<T>(t.ey, f.c[1] + q); vecb::vload<T>(t.ez, f.c[2] + q);
        vecb::vload<T>(t.bx, g.bE[0] + q); vecb::vload<T>(t.by, g.bE[1] + q); vecb::vload<T>(t.bz, g.bE[2] + q);
        if (j > 0) { vecb::vload<T>(t.hxj, f.c[3] + q - px); vecb::vload<T>(t.hzj, f.c[5] + q - px); }
        if (i > 0) { vecb::vload<T>(t.hxi, f.c[3] + q - Ny * px); vecb::vload<T>(t.hyi, f.c[4] + q - Ny * px); }
        else if (g.zlo) { vecb::vload<T>(t.hxi, g.zhalo[2] + q); vecb::vload<T>(t.hyi, g.zhalo[3] + q); }
        if (lane == 0 && k0 > 0) { t.hy_p = ld(f.c[4] + q - 1); t.hz_p = ld(f.c[5] + q - 1); }
        if (t.ly >= 0) {
            const int s = (i * PY.wsum + t.ly) * px + k0;
            vecb::vload<T>(t.py2, PY.psi[2] + s); vecb::vload<T>(t.py3, PY.psi[3] + s);
        }
        if (t.lz >= 0) {
            const int s = (t.lz * Ny + j) * px + k0;
            vecb::vload<T>(t.pz2, PZ.psi[2] + s); vecb::vload<T>(t.pz3, PZ.psi[3] + s);
        }
        if (lossy) {
            vecb::vload<T>(t.ax, g.aE[0] + q); vecb::vload<T>(t.ay, g.aE[1] + q); vecb::vload<T>(t.az, g.aE[2] + q);
        }
    }
#pragma unroll
    for (int e = 0; e < V; e++) t.lxs[e] = -1;
    if (xw) {
        const bool xs = t.act && (k0 < PX.w0 || k0 + V - 1 >= PX.edge_max);
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int k = k0 + e;
            t.lxs[e] = (xs && k < g.Nx) ? slab_local(PX, k, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
            if (t.lxs[e] >= 0 && !vecb::in_range(g, (long long)(i * Ny + j) * PX.wsum + t.lxs[e], 0,
                                                 (long long)g.Nz * Ny * PX.wsum, 17))
                t.lxs[e] = -1;
#endif
            if (t.lxs[e] >= 0) {
                const int s = (i * Ny + j) * PX.wsum + t.lxs[e];
                t.px2[e] = ld(PX.psi[2] + s); t.px3[e] = ld(PX.psi[3] + s);
            }
        }
    }
}

template <typename T, bool GEN = true, bool SERVE = false, bool SRC = GEN>
__device__ __forceinline__ void e_finish(const GridView<T>& g, const Fields<T>& f, const SourceList<T>& src,
                                         const long long* step_ctr, int off, int i, int j, int xb,
                                         int lane, ETask<T>& t) {
    constexpr int V = vecb::V16<T>::N;
    constexpr unsigned FULL = 0xffffffffu;
    const int k0 = (xb * 32 + lane) * V;
    const int Ny = g.Ny, px = g.px;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const bool xw = GEN && (xb * 32 * V < PX.w0 || (xb + 1) * 32 * V - 1 >= PX.edge_max);
    const bool lossy = g.aE[0] != nullptr;
    if (SERVE && !serve_running(t.sstate)) return;   // the whole warp leaves together
    const bool srcb = SRC && src.n && vecb::sources_touch<T>(src, 0, i, j, j + 1,
                                                             xb * 32 * V, (xb + 1) * 32 * V);
    double4 st = make_double4(0, 0, 0, 0);
    if (srcb) st = g.step_tab[*step_ctr + off];

    // ---- x neighbour of the first cell: last cell of the previous vector
    {
        const T a = __shfl_up_sync(FULL, t.hy[V - 1], 1), b = __shfl_up_sync(FULL, t.hz[V - 1], 1);
        if (lane != 0) { t.hy_p = a; t.hz_p = b; }
    }
    if (!t.act) return;
    if (k0 == 0) { t.hy_p = h_min_ghost<T>(g.bc[0], t.hy[0], T(0)); t.hz_p = h_min_ghost<T>(g.bc[0], t.hz[0], T(0)); }
    if (j == 0) {
#pragma unroll
        for (int e = 0; e < V; e++) {
            t.hxj[e] = h_min_ghost<T>(g.bc[1], t.hx[e], T(0));
            t.hzj[e] = h_min_ghost<T>(g.bc[1], t.hz[e], T(0));
        }
    }
    if (i == 0 && !g.zlo) {
#pragma unroll
        for (int e = 0; e < V; e++) {
            t.hxi[e] = h_min_ghost<T>(g.bc[2], t.hx[e], T(0));
            t.hyi[e] = h_min_ghost<T>(g.bc[2], t.hy[e], T(0));
        }
    }
#pragma unroll
    for (int e = 0; e < V; e++) {
        const T hyx = e > 0 ? t.hy[e - 1] : t.hy_p;
        const T hzx = e > 0 ? t.hz[e - 1] : t.hz_p;
        const T dHzdy = g.ody * (t.hz[e] - t.hzj[e]);
        const T dHydz = g.odz * (t.hy[e] - t.hyi[e]);
        const T dHxdz = g.odz * (t.hx[e] - t.hxi[e]);
        const T dHzdx = g.odx * (t.hz[e] - hzx);
        const T dHydx = g.odx * (t.hy[e] - hyx);
        const T dHxdy = g.ody * (t.hx[e] - t.hxj[e]);
        T Ex, Ey, Ez;
        if (lossy) {
            Ex = t.ax[e] * t.ex[e] + (dHzdy - dHydz) * t.bx[e];
            Ey = t.ay[e] * t.ey[e] + (dHxdz - dHzdx) * t.by[e];
            Ez = t.az[e] * t.ez[e] + (dHydx - dHxdy) * t.bz[e];
        } else {
            Ex = t.ex[e] + (dHzdy - dHydz) * t.bx[e];
            Ey = t.ey[e] + (dHxdz - dHzdx) * t.by[e];
            Ez = t.ez[e] + (dHydx - dHxdy) * t.bz[e];
        }
        if (xw && t.lxs[e] >= 0) {
            const int l = t.lxs[e];
            const T kv = ld(PX.kinvE + l), bv = ld(PX.bE + l), cv = ld(PX.cE + l);
            t.px2[e] = cv * dHydx + bv * t.px2[e];
            t.px3[e] = cv * dHzdx + bv * t.px3[e];
            Ez = Ez + ((t.px2[e] - dHydx) + dHydx * kv) * t.bz[e];
            Ey = Ey - ((t.px3[e] - dHzdx) + dHzdx * kv) * t.by[e];
        }
        if (t.ly >= 0) {
            const int l = t.ly;
            const T kv = ld(PY.kinvE + l), bv = ld(PY.bE + l), cv = ld(PY.cE + l);
            t.py2[e] = cv * dHxdy + bv * t.py2[e];
            t.py3[e] = cv * dHzdy + bv * t.py3[e];
            Ez = Ez - ((t.py2[e] - dHxdy) + dHxdy * kv) * t.bz[e];
            Ex = Ex + ((t.py3[e] - dHzdy) + dHzdy * kv) * t.bx[e];
        }
        if (t.lz >= 0) {
            const int l = t.lz;
            const T kv = ld(PZ.kinvE + l), bv = ld(PZ.bE + l), cv = ld(PZ.cE + l);
            t.pz2[e] = cv * dHxdz + bv * t.pz2[e];
            t.pz3[e] = cv * dHydz + bv * t.pz3[e];
            Ex = Ex - ((t.pz3[e] - dHydz) + dHydz * kv) * t.bx[e];
            Ey = Ey + ((t.pz2[e] - dHxdz) + dHxdz * kv) * t.by[e];
        }
        if (srcb && k0 + e < g.Nx)
            add_sources<T>(src, i, j, k0 + e, 0, T(st.z), T(st.w), Ex, Ey, Ez, true);
        t.ex[e] = Ex; t.ey[e] = Ey; t.ez[e] = Ez;
    }
    const int q = t.p;
    vecb::vstore<T>(f.c[0] + q, t.ex); vecb::vstore<T>(f.c[1] + q, t.ey); vecb::vstore<T>(f.c[2] + q, t.ez);
    if (t.ly >= 0) {
        const int s = (i * PY.wsum + t.ly) * px + k0;
        vecb::vstore<T>(PY.psi[2] + s, t.py2); vecb::vstore<T>(PY.psi[3] + s, t.py3);
    }
    if (t.lz >= 0) {
        const int s = (t.lz * Ny + j) * px + k0;
        vecb::vstore<T>(PZ.psi[2] + s, t.pz2); vecb::vstore<T>(PZ.psi[3] + s, t.pz3);
    }
    if (xw) {
#pragma unroll
        for (int e = 0; e < V; e++)
            if (t.lxs[e] >= 0) {
                const int s = (i * Ny + j) * PX.wsum + t.lxs[e];
                PX.psi[2][s] = t.px2[e]; PX.psi[3][s] = t.px3[e];
            }
    }
}

template <typename T, bool GEN = true, bool SERVE = false, bool SRC = GEN>
__device__ __forceinline__ void vec_update_E(const GridView<T>& g, const Fields<T>& f,
                                             const SourceList<T>& src, const long long* step_ctr,
                                             int off, int i, int j, int xb, int lane,
                                             const ServeGate<T>* sg = nullptr) {
    ETask<T> t;
    e_load<T, GEN, SERVE>(g, f, i, j, xb, lane, sg, t);
    e_finish<T, GEN, SERVE, SRC>(g, f, src, step_ctr, off, i, j, xb, lane, t);
}

}  // namespace fdtdb
