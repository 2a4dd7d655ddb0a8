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

// L2 prefetch (GridView::pf planes ahead, 0: none).  The warp that updates
// row j of plane i asks L2 for the same 64-cell segment of plane i + pf of
// the arrays it streams, so that the warp which later updates that plane
// finds them in L2 (fp32 MMI block: 119.4 instead of 121.0 us per step at
// distance 2, fp64 199 instead of 205; distance 4 and 8 and one bulk request
// per array gained less).  The host enables it only when the prefetched
// planes fit in L2 beside the planes being updated (make_view).

// p: first cell of the warp's segment; `room` cells of the row's pitch remain
// from there, so no request leaves the row.
template <typename T>
__device__ __forceinline__ void l2_prefetch(const T* p, int lane, int room) {
    if (2 * lane < room) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p + 2 * lane));
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

// Does the warp that updates rows j0 .. j0+NR-1 of plane i, vectors 32 xb ..
// 32 xb + 31, touch no CPML slab and no source box of the half step
// (comp_base 3: H sources, 0: E sources)?  Then the body built without CPML
// and source code (GEN = false) computes the same values in the same order.
template <typename T, int NR>
__device__ __forceinline__ bool plain_warp(const GridView<T>& g, const SourceList<T>& src,
                                           int comp_base, int i, int j0, int xb) {
    constexpr int V = V16<T>::N;
    if (slab_local(g.pml[2], i + g.pml[2].off, true) >= 0) return false;
#pragma unroll
    for (int r = 0; r < NR; r++)
        if (j0 + r < g.Ny && slab_local(g.pml[1], j0 + r, false) >= 0) return false;
    if (xb * 32 * V < g.pml[0].w0 || (xb + 1) * 32 * V - 1 >= g.pml[0].edge_max) return false;
    return !(src.n && sources_touch<T>(src, comp_base, i, j0, j0 + NR, xb * 32 * V, (xb + 1) * 32 * V));
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

// Rows per warp: a warp updates the same 32 vectors of NR consecutive rows
// j0 .. j0+NR-1 of plane i.  Every load of all rows is issued before any
// arithmetic, so NR = 2 keeps twice the bytes of one warp in flight; the rows
// share the loads they have in common (the H update of row j reads E of row
// j+1, the E update of row j reads H of row j-1).
template <typename T, int NR = 1, bool GEN = true, bool SERVE = false>
__device__ __forceinline__ void vec_update_H(const GridView<T>& g, const Fields<T>& f,
                                     const SourceList<T>& src, const long long* step_ctr,
                                     int off, int i, int j0, int xb, int lane,
                                     const ServeGate<T>* sg = nullptr) {
    constexpr int V = vecb::V16<T>::N;
    constexpr unsigned FULL = 0xffffffffu;
    const int m = xb * 32 + lane;
    const int k0 = m * V;
    const int Ny = g.Ny, Nz = g.Nz, px = g.px;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int lz0 = GEN ? slab_local(PZ, i + PZ.off, true) : -1;   // same for every row of the warp
    bool act[NR];
    int p[NR], ly[NR], lz[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const int j = j0 + r;
        // lanes beyond the row still take part in the shuffles below
        const bool act0 = j < Ny && k0 < g.Nx;
        p[r] = act0 ? (i * Ny + j) * px + k0 : 0;
        const int ly0 = GEN ? slab_local(PY, j, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
        // a lane whose indices fall outside their arrays records the site and skips
        act[r] = act0 && vecb::h_fields_ok(g, i, j, k0, lane, p[r]);
        ly[r] = (ly0 >= 0 && act[r] && !vecb::in_range(g, (long long)(i * PY.wsum + ly0) * px + k0, 0,
                                                       (long long)Nz * PY.wsum * px - V + 1, 5)) ? -1 : ly0;
        lz[r] = (lz0 >= 0 && act[r] && !vecb::in_range(g, (long long)(lz0 * Ny + j) * px + k0, 0,
                                                       (long long)PZ.wsum * Ny * px - V + 1, 6)) ? -1 : lz0;
#else
        act[r] = act0;
        ly[r] = ly0;
        lz[r] = lz0;
#endif
    }
    // does any lane of the warp touch an x slab?  (the same for all lanes)
    const bool xw = GEN && (xb * 32 * V < PX.w0 || (xb + 1) * 32 * V - 1 >= PX.edge_max);

    if (g.pf > 0 && i + g.pf < Nz && xb * 32 * V < g.Nx) {
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (j0 + r < Ny) {
                const long long q = (long long)(i + g.pf) * g.plane + (long long)(j0 + r) * px + xb * 32 * V;
#pragma unroll
                for (int c = 0; c < 6; c++) vecb::l2_prefetch<T>(f.c[c] + q, lane, px - xb * 32 * V);
            }
    }

    // a served request's state and capture flag, read with the fields
    int sstate = SERVE_RUN, scap = 0;
    if (SERVE) { sstate = __ldg(sg->state); scap = __ldg(sg->capture); }

    // ---- every load of the thread first
    T ex[NR][V], ey[NR][V], ez[NR][V], exj[NR][V], ezj[NR][V], exi[NR][V], eyi[NR][V];
    T hx[NR][V], hy[NR][V], hz[NR][V];
    T py0[NR][V], py1[NR][V], pz0[NR][V], pz1[NR][V], px0[NR][V], px1[NR][V];
    T ey_n[NR], ez_n[NR];
    int lxs[NR][V];
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const int j = j0 + r;
        vecb::vzero<T>(ex[r]); vecb::vzero<T>(ey[r]); vecb::vzero<T>(ez[r]); vecb::vzero<T>(exj[r]);
        vecb::vzero<T>(ezj[r]); vecb::vzero<T>(exi[r]); vecb::vzero<T>(eyi[r]);
        ey_n[r] = T(0); ez_n[r] = T(0);
        if (act[r]) {
            const int q = p[r];
            vecb::vload<T>(ex[r], f.c[0] + q); vecb::vload<T>(ey[r], f.c[1] + q); vecb::vload<T>(ez[r], f.c[2] + q);
            // E of row j+1: the next row's own load, or a load of its own for the last row
            if (r + 1 == NR && j + 1 < Ny) { vecb::vload<T>(exj[r], f.c[0] + q + px); vecb::vload<T>(ezj[r], f.c[2] + q + px); }
            if (i + 1 < Nz) { vecb::vload<T>(exi[r], f.c[0] + q + Ny * px); vecb::vload<T>(eyi[r], f.c[1] + q + Ny * px); }
            else if (g.zhi) { vecb::vload<T>(exi[r], g.zhalo[0] + (q - i * Ny * px)); vecb::vload<T>(eyi[r], g.zhalo[1] + (q - i * Ny * px)); }
            vecb::vload<T>(hx[r], f.c[3] + q); vecb::vload<T>(hy[r], f.c[4] + q); vecb::vload<T>(hz[r], f.c[5] + q);
            if (lane == 31 && k0 + V < g.Nx) { ey_n[r] = ld(f.c[1] + q + V); ez_n[r] = ld(f.c[2] + q + V); }
            if (ly[r] >= 0) {
                const int s = (i * PY.wsum + ly[r]) * px + k0;
                vecb::vload<T>(py0[r], PY.psi[0] + s); vecb::vload<T>(py1[r], PY.psi[1] + s);
            }
            if (lz[r] >= 0) {
                const int s = (lz[r] * Ny + j) * px + k0;
                vecb::vload<T>(pz0[r], PZ.psi[0] + s); vecb::vload<T>(pz1[r], PZ.psi[1] + s);
            }
        }
#pragma unroll
        for (int e = 0; e < V; e++) lxs[r][e] = -1;
        if (xw) {
            const bool xs = act[r] && (k0 < PX.w0 || k0 + V - 1 >= PX.edge_max);
#pragma unroll
            for (int e = 0; e < V; e++) {
                const int k = k0 + e;
                lxs[r][e] = (xs && k < g.Nx) ? slab_local(PX, k, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
                if (lxs[r][e] >= 0 && !vecb::in_range(g, (long long)(i * Ny + j) * PX.wsum + lxs[r][e], 0,
                                                      (long long)Nz * Ny * PX.wsum, 7))
                    lxs[r][e] = -1;
#endif
                if (lxs[r][e] >= 0) {
                    const int s = (i * Ny + j) * PX.wsum + lxs[r][e];
                    px0[r][e] = ld(PX.psi[0] + s); px1[r][e] = ld(PX.psi[1] + s);
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r + 1 < NR; r++)
        if (act[r] && j0 + r + 1 < Ny) {
#pragma unroll
            for (int e = 0; e < V; e++) { exj[r][e] = ex[r + 1][e]; ezj[r][e] = ez[r + 1][e]; }
        }
    T mx[NR][V], my[NR][V], mz[NR][V];
    const bool mu_arr = g.bHarr[0] != nullptr;
#pragma unroll
    for (int r = 0; r < NR; r++) {
        if (mu_arr && act[r]) {
            vecb::vload<T>(mx[r], g.bHarr[0] + p[r]); vecb::vload<T>(my[r], g.bHarr[1] + p[r]);
            vecb::vload<T>(mz[r], g.bHarr[2] + p[r]);
        } else {
#pragma unroll
            for (int e = 0; e < V; e++) { mx[r][e] = g.bH[0]; my[r][e] = g.bH[1]; mz[r][e] = g.bH[2]; }
        }
    }
    if (SERVE) {
        // the whole warp leaves together (one state per request)
        if (!serve_running(sstate)) return;
        if (scap == 1 || scap == 2) {
            T* const* d = sg->snap[scap - 1];
#pragma unroll
            for (int r = 0; r < NR; r++)
                if (act[r]) {
                    const int q = p[r];
                    vecb::vstore<T>(d[0] + q, ex[r]); vecb::vstore<T>(d[1] + q, ey[r]); vecb::vstore<T>(d[2] + q, ez[r]);
                    vecb::vstore<T>(d[3] + q, hx[r]); vecb::vstore<T>(d[4] + q, hy[r]); vecb::vstore<T>(d[5] + q, hz[r]);
                }
        }
    }
    const bool srcb = GEN && src.n && vecb::sources_touch<T>(src, 3, i, j0, j0 + NR,
                                                xb * 32 * V, (xb + 1) * 32 * V);
    double4 st = make_double4(0, 0, 0, 0);
    if (srcb) st = g.step_tab[*step_ctr + off];

#pragma unroll
    for (int r = 0; r < NR; r++) {
        const int j = j0 + r;
        // ---- x neighbour of the last cell: first cell of the next vector
        {
            const T a = __shfl_down_sync(FULL, ey[r][0], 1), b = __shfl_down_sync(FULL, ez[r][0], 1);
            if (lane != 31) { ey_n[r] = a; ez_n[r] = b; }
        }
        if (!act[r]) continue;
#pragma unroll
        for (int e = 0; e < V; e++) {
            const T eyx = e + 1 < V ? ey[r][e + 1] : ey_n[r];
            const T ezx = e + 1 < V ? ez[r][e + 1] : ez_n[r];
            const T dEzdy = g.ody * (ezj[r][e] - ez[r][e]);
            const T dEydz = g.odz * (eyi[r][e] - ey[r][e]);
            const T dExdz = g.odz * (exi[r][e] - ex[r][e]);
            const T dEzdx = g.odx * (ezx - ez[r][e]);
            const T dEydx = g.odx * (eyx - ey[r][e]);
            const T dExdy = g.ody * (exj[r][e] - ex[r][e]);
            T Hx = hx[r][e] + mx[r][e] * (dEydz - dEzdy);
            T Hy = hy[r][e] + my[r][e] * (dEzdx - dExdz);
            T Hz = hz[r][e] + mz[r][e] * (dExdy - dEydx);
            if (xw && lxs[r][e] >= 0) {
                const int l = lxs[r][e];
                const T kv = ld(PX.kinvH + l), bv = ld(PX.bH + l), cv = ld(PX.cH + l);
                px0[r][e] = cv * dEydx + bv * px0[r][e];
                px1[r][e] = cv * dEzdx + bv * px1[r][e];
                Hz = Hz - mz[r][e] * ((px0[r][e] - dEydx) + dEydx * kv);
                Hy = Hy + my[r][e] * ((px1[r][e] - dEzdx) + dEzdx * kv);
            }
            if (ly[r] >= 0) {
                const int l = ly[r];
                const T kv = ld(PY.kinvH + l), bv = ld(PY.bH + l), cv = ld(PY.cH + l);
                py0[r][e] = cv * dExdy + bv * py0[r][e];
                py1[r][e] = cv * dEzdy + bv * py1[r][e];
                Hz = Hz + mz[r][e] * ((py0[r][e] - dExdy) + dExdy * kv);
                Hx = Hx - mx[r][e] * ((py1[r][e] - dEzdy) + dEzdy * kv);
            }
            if (lz[r] >= 0) {
                const int l = lz[r];
                const T kv = ld(PZ.kinvH + l), bv = ld(PZ.bH + l), cv = ld(PZ.cH + l);
                pz0[r][e] = cv * dExdz + bv * pz0[r][e];
                pz1[r][e] = cv * dEydz + bv * pz1[r][e];
                Hx = Hx + mx[r][e] * ((pz1[r][e] - dEydz) + dEydz * kv);
                Hy = Hy - my[r][e] * ((pz0[r][e] - dExdz) + dExdz * kv);
            }
            if (srcb && k0 + e < g.Nx)
                add_sources<T>(src, i, j, k0 + e, 3, T(st.x), T(st.y), Hx, Hy, Hz, false);
            hx[r][e] = Hx; hy[r][e] = Hy; hz[r][e] = Hz;
        }
        const int q = p[r];
        vecb::vstore<T>(f.c[3] + q, hx[r]); vecb::vstore<T>(f.c[4] + q, hy[r]); vecb::vstore<T>(f.c[5] + q, hz[r]);
        if (ly[r] >= 0) {
            const int s = (i * PY.wsum + ly[r]) * px + k0;
            vecb::vstore<T>(PY.psi[0] + s, py0[r]); vecb::vstore<T>(PY.psi[1] + s, py1[r]);
        }
        if (lz[r] >= 0) {
            const int s = (lz[r] * Ny + j) * px + k0;
            vecb::vstore<T>(PZ.psi[0] + s, pz0[r]); vecb::vstore<T>(PZ.psi[1] + s, pz1[r]);
        }
        if (xw) {
#pragma unroll
            for (int e = 0; e < V; e++)
                if (lxs[r][e] >= 0) {
                    const int s = (i * Ny + j) * PX.wsum + lxs[r][e];
                    PX.psi[0][s] = px0[r][e]; PX.psi[1][s] = px1[r][e];
                }
        }
    }
}

template <typename T, int NR = 1, bool GEN = true, bool SERVE = false>
__device__ __forceinline__ void vec_update_E(const GridView<T>& g, const Fields<T>& f,
                                     const SourceList<T>& src, const long long* step_ctr,
                                     int off, int i, int j0, int xb, int lane,
                                     const ServeGate<T>* sg = nullptr) {
    constexpr int V = vecb::V16<T>::N;
    constexpr unsigned FULL = 0xffffffffu;
    const int m = xb * 32 + lane;
    const int k0 = m * V;
    const int Ny = g.Ny, px = g.px;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int lz0 = GEN ? slab_local(PZ, i + PZ.off, true) : -1;   // same for every row of the warp
    bool act[NR];
    int p[NR], ly[NR], lz[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const int j = j0 + r;
        const bool act0 = j < Ny && k0 < g.Nx;
        p[r] = act0 ? (i * Ny + j) * px + k0 : 0;
        const int ly0 = GEN ? slab_local(PY, j, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
        act[r] = act0 && vecb::e_fields_ok(g, i, j, k0, lane, p[r]);
        ly[r] = (ly0 >= 0 && act[r] && !vecb::in_range(g, (long long)(i * PY.wsum + ly0) * px + k0, 0,
                                                       (long long)g.Nz * PY.wsum * px - V + 1, 15)) ? -1 : ly0;
        lz[r] = (lz0 >= 0 && act[r] && !vecb::in_range(g, (long long)(lz0 * Ny + j) * px + k0, 0,
                                                       (long long)PZ.wsum * Ny * px - V + 1, 16)) ? -1 : lz0;
#else
        act[r] = act0;
        ly[r] = ly0;
        lz[r] = lz0;
#endif
    }
    // does any lane of the warp touch an x slab?  (the same for all lanes)
    const bool xw = GEN && (xb * 32 * V < PX.w0 || (xb + 1) * 32 * V - 1 >= PX.edge_max);
    const bool lossy = g.aE[0] != nullptr;

    if (g.pf > 0 && i + g.pf < g.Nz && xb * 32 * V < g.Nx) {
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (j0 + r < Ny) {
                const long long q = (long long)(i + g.pf) * g.plane + (long long)(j0 + r) * px + xb * 32 * V;
#pragma unroll
                for (int c = 0; c < 6; c++) vecb::l2_prefetch<T>(f.c[c] + q, lane, px - xb * 32 * V);
#pragma unroll
                for (int c = 0; c < 3; c++) vecb::l2_prefetch<T>(g.bE[c] + q, lane, px - xb * 32 * V);
            }
    }

    int sstate = SERVE_RUN;
    if (SERVE) sstate = __ldg(sg->state);

    // ---- every load of the thread first
    T hx[NR][V], hy[NR][V], hz[NR][V], hxj[NR][V], hzj[NR][V], hxi[NR][V], hyi[NR][V];
    T ex[NR][V], ey[NR][V], ez[NR][V], bx[NR][V], by[NR][V], bz[NR][V];
    T py2[NR][V], py3[NR][V], pz2[NR][V], pz3[NR][V], px2[NR][V], px3[NR][V], ax[NR][V], ay[NR][V], az[NR][V];
    T hy_p[NR], hz_p[NR];
    int lxs[NR][V];
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const int j = j0 + r;
        vecb::vzero<T>(hy[r]); vecb::vzero<T>(hz[r]);
        hy_p[r] = T(0); hz_p[r] = T(0);
        if (act[r]) {
            const int q = p[r];
            vecb::vload<T>(hx[r], f.c[3] + q); vecb::vload<T>(hy[r], f.c[4] + q); vecb::vload<T>(hz[r], f.c[5] + q);
            vecb::vload<T>(ex[r], f.c[0] + q); vecb::vload<T>(ey[r], f.c[1] + q); vecb::vload<T>(ez[r], f.c[2] + q);
            vecb::vload<T>(bx[r], g.bE[0] + q); vecb::vload<T>(by[r], g.bE[1] + q); vecb::vload<T>(bz[r], g.bE[2] + q);
            // H of row j-1: the previous row's own load, or a load of its own for the first row
            if (r == 0 && j > 0) { vecb::vload<T>(hxj[r], f.c[3] + q - px); vecb::vload<T>(hzj[r], f.c[5] + q - px); }
            if (i > 0) { vecb::vload<T>(hxi[r], f.c[3] + q - Ny * px); vecb::vload<T>(hyi[r], f.c[4] + q - Ny * px); }
            else if (g.zlo) { vecb::vload<T>(hxi[r], g.zhalo[2] + q); vecb::vload<T>(hyi[r], g.zhalo[3] + q); }
            if (lane == 0 && k0 > 0) { hy_p[r] = ld(f.c[4] + q - 1); hz_p[r] = ld(f.c[5] + q - 1); }
            if (ly[r] >= 0) {
                const int s = (i * PY.wsum + ly[r]) * px + k0;
                vecb::vload<T>(py2[r], PY.psi[2] + s); vecb::vload<T>(py3[r], PY.psi[3] + s);
            }
            if (lz[r] >= 0) {
                const int s = (lz[r] * Ny + j) * px + k0;
                vecb::vload<T>(pz2[r], PZ.psi[2] + s); vecb::vload<T>(pz3[r], PZ.psi[3] + s);
            }
            if (lossy) {
                vecb::vload<T>(ax[r], g.aE[0] + q); vecb::vload<T>(ay[r], g.aE[1] + q); vecb::vload<T>(az[r], g.aE[2] + q);
            }
        }
#pragma unroll
        for (int e = 0; e < V; e++) lxs[r][e] = -1;
        if (xw) {
            const bool xs = act[r] && (k0 < PX.w0 || k0 + V - 1 >= PX.edge_max);
#pragma unroll
            for (int e = 0; e < V; e++) {
                const int k = k0 + e;
                lxs[r][e] = (xs && k < g.Nx) ? slab_local(PX, k, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
                if (lxs[r][e] >= 0 && !vecb::in_range(g, (long long)(i * Ny + j) * PX.wsum + lxs[r][e], 0,
                                                      (long long)g.Nz * Ny * PX.wsum, 17))
                    lxs[r][e] = -1;
#endif
                if (lxs[r][e] >= 0) {
                    const int s = (i * Ny + j) * PX.wsum + lxs[r][e];
                    px2[r][e] = ld(PX.psi[2] + s); px3[r][e] = ld(PX.psi[3] + s);
                }
            }
        }
    }
#pragma unroll
    for (int r = 1; r < NR; r++)
        if (act[r]) {
#pragma unroll
            for (int e = 0; e < V; e++) { hxj[r][e] = hx[r - 1][e]; hzj[r][e] = hz[r - 1][e]; }
        }
    if (SERVE && !serve_running(sstate)) return;   // the whole warp leaves together
    const bool srcb = GEN && src.n && vecb::sources_touch<T>(src, 0, i, j0, j0 + NR,
                                                xb * 32 * V, (xb + 1) * 32 * V);
    double4 st = make_double4(0, 0, 0, 0);
    if (srcb) st = g.step_tab[*step_ctr + off];

#pragma unroll
    for (int r = 0; r < NR; r++) {
        const int j = j0 + r;
        // ---- x neighbour of the first cell: last cell of the previous vector
        {
            const T a = __shfl_up_sync(FULL, hy[r][V - 1], 1), b = __shfl_up_sync(FULL, hz[r][V - 1], 1);
            if (lane != 0) { hy_p[r] = a; hz_p[r] = b; }
        }
        if (!act[r]) continue;
        if (k0 == 0) { hy_p[r] = h_min_ghost<T>(g.bc[0], hy[r][0], T(0)); hz_p[r] = h_min_ghost<T>(g.bc[0], hz[r][0], T(0)); }
        if (j == 0) {
#pragma unroll
            for (int e = 0; e < V; e++) {
                hxj[r][e] = h_min_ghost<T>(g.bc[1], hx[r][e], T(0));
                hzj[r][e] = h_min_ghost<T>(g.bc[1], hz[r][e], T(0));
            }
        }
        if (i == 0 && !g.zlo) {
#pragma unroll
            for (int e = 0; e < V; e++) {
                hxi[r][e] = h_min_ghost<T>(g.bc[2], hx[r][e], T(0));
                hyi[r][e] = h_min_ghost<T>(g.bc[2], hy[r][e], T(0));
            }
        }
#pragma unroll
        for (int e = 0; e < V; e++) {
            const T hyx = e > 0 ? hy[r][e - 1] : hy_p[r];
            const T hzx = e > 0 ? hz[r][e - 1] : hz_p[r];
            const T dHzdy = g.ody * (hz[r][e] - hzj[r][e]);
            const T dHydz = g.odz * (hy[r][e] - hyi[r][e]);
            const T dHxdz = g.odz * (hx[r][e] - hxi[r][e]);
            const T dHzdx = g.odx * (hz[r][e] - hzx);
            const T dHydx = g.odx * (hy[r][e] - hyx);
            const T dHxdy = g.ody * (hx[r][e] - hxj[r][e]);
            T Ex, Ey, Ez;
            if (lossy) {
                Ex = ax[r][e] * ex[r][e] + (dHzdy - dHydz) * bx[r][e];
                Ey = ay[r][e] * ey[r][e] + (dHxdz - dHzdx) * by[r][e];
                Ez = az[r][e] * ez[r][e] + (dHydx - dHxdy) * bz[r][e];
            } else {
                Ex = ex[r][e] + (dHzdy - dHydz) * bx[r][e];
                Ey = ey[r][e] + (dHxdz - dHzdx) * by[r][e];
                Ez = ez[r][e] + (dHydx - dHxdy) * bz[r][e];
            }
            if (xw && lxs[r][e] >= 0) {
                const int l = lxs[r][e];
                const T kv = ld(PX.kinvE + l), bv = ld(PX.bE + l), cv = ld(PX.cE + l);
                px2[r][e] = cv * dHydx + bv * px2[r][e];
                px3[r][e] = cv * dHzdx + bv * px3[r][e];
                Ez = Ez + ((px2[r][e] - dHydx) + dHydx * kv) * bz[r][e];
                Ey = Ey - ((px3[r][e] - dHzdx) + dHzdx * kv) * by[r][e];
            }
            if (ly[r] >= 0) {
                const int l = ly[r];
                const T kv = ld(PY.kinvE + l), bv = ld(PY.bE + l), cv = ld(PY.cE + l);
                py2[r][e] = cv * dHxdy + bv * py2[r][e];
                py3[r][e] = cv * dHzdy + bv * py3[r][e];
                Ez = Ez - ((py2[r][e] - dHxdy) + dHxdy * kv) * bz[r][e];
                Ex = Ex + ((py3[r][e] - dHzdy) + dHzdy * kv) * bx[r][e];
            }
            if (lz[r] >= 0) {
                const int l = lz[r];
                const T kv = ld(PZ.kinvE + l), bv = ld(PZ.bE + l), cv = ld(PZ.cE + l);
                pz2[r][e] = cv * dHxdz + bv * pz2[r][e];
                pz3[r][e] = cv * dHydz + bv * pz3[r][e];
                Ex = Ex - ((pz3[r][e] - dHydz) + dHydz * kv) * bx[r][e];
                Ey = Ey + ((pz2[r][e] - dHxdz) + dHxdz * kv) * by[r][e];
            }
            if (srcb && k0 + e < g.Nx)
                add_sources<T>(src, i, j, k0 + e, 0, T(st.z), T(st.w), Ex, Ey, Ez, true);
            ex[r][e] = Ex; ey[r][e] = Ey; ez[r][e] = Ez;
        }
        const int q = p[r];
        vecb::vstore<T>(f.c[0] + q, ex[r]); vecb::vstore<T>(f.c[1] + q, ey[r]); vecb::vstore<T>(f.c[2] + q, ez[r]);
        if (ly[r] >= 0) {
            const int s = (i * PY.wsum + ly[r]) * px + k0;
            vecb::vstore<T>(PY.psi[2] + s, py2[r]); vecb::vstore<T>(PY.psi[3] + s, py3[r]);
        }
        if (lz[r] >= 0) {
            const int s = (lz[r] * Ny + j) * px + k0;
            vecb::vstore<T>(PZ.psi[2] + s, pz2[r]); vecb::vstore<T>(PZ.psi[3] + s, pz3[r]);
        }
        if (xw) {
#pragma unroll
            for (int e = 0; e < V; e++)
                if (lxs[r][e] >= 0) {
                    const int s = (i * Ny + j) * PX.wsum + lxs[r][e];
                    PX.psi[2][s] = px2[r][e]; PX.psi[3][s] = px3[r][e];
                }
        }
    }
}

}  // namespace fdtdb
