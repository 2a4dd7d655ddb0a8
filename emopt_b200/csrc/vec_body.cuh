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
// slab face is read from the halo plane of the field arrays, and the z CPML
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

// L2 prefetch distance in planes (0: none).  The warp that updates row j of
// plane i asks L2 for the same 64-cell segment of plane i + VEC_PREFETCH of
// the arrays it streams, so that the warp which later updates that plane
// finds them in L2 (fp32 MMI block: 119.4 instead of 121.0 us per step at
// distance 2, fp64 199 instead of 205; distance 4 and 8 and one bulk request
// per array gained less).
#ifndef VEC_PREFETCH
#define VEC_PREFETCH 2
#endif

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
    const long long fhi = ((long long)g.Nz + (g.zhi ? 1 : 0)) * plane;
    bool ok = in_range(g, p, 0, top - V + 1, 1);
    if (j + 1 < g.Ny) ok &= in_range(g, p + g.px, 0, top - V + 1, 2);
    if (i + 1 < g.Nz || g.zhi) ok &= in_range(g, p + plane, 0, fhi - V + 1, 3);
    if (lane == 31 && k0 + V < g.Nx) ok &= in_range(g, p + V, 0, top, 4);
    return ok;
}

// ... and the E body.
template <typename T>
__device__ bool e_fields_ok(const GridView<T>& g, int i, int j, int k0, int lane, long long p) {
    constexpr int V = V16<T>::N;
    const long long plane = g.plane, top = (long long)g.Nz * plane;
    const long long flo = g.zlo ? -plane : 0;
    bool ok = in_range(g, p, 0, top - V + 1, 11);
    if (j > 0) ok &= in_range(g, p - g.px, 0, top - V + 1, 12);
    if (i > 0 || g.zlo) ok &= in_range(g, p - plane, flo, top - V + 1, 13);
    if (lane == 0 && k0 > 0) ok &= in_range(g, p - 1, 0, top, 14);
    return ok;
}
#endif

}  // namespace vecb

template <typename T>
__device__ __forceinline__ void vec_update_H(const GridView<T>& g, const Fields<T>& f,
                                     const SourceList<T>& src, const long long* step_ctr,
                                     int off, int i, int j, int xb, int lane) {
    constexpr int V = vecb::V16<T>::N;
    constexpr unsigned FULL = 0xffffffffu;
    const int m = xb * 32 + lane;
    const int k0 = m * V;
    // Lanes beyond the row still take part in the shuffle below.
    const bool act0 = j < g.Ny && k0 < g.Nx;
    const int Ny = g.Ny, Nz = g.Nz, px = g.px;
    const int p = act0 ? (i * Ny + j) * px + k0 : 0;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int ly0 = slab_local(PY, j, false);   // same for the whole warp
    const int lz0 = slab_local(PZ, i + PZ.off, true);
#ifdef FDTD_BOUNDS_CHECK
    // a lane whose indices fall outside their arrays records the site and skips
    const bool act = act0 && vecb::h_fields_ok(g, i, j, k0, lane, p);
    const int ly = (ly0 >= 0 && act && !vecb::in_range(g, (long long)(i * PY.wsum + ly0) * px + k0, 0,
                                                      (long long)Nz * PY.wsum * px - V + 1, 5)) ? -1 : ly0;
    const int lz = (lz0 >= 0 && act && !vecb::in_range(g, (long long)(lz0 * Ny + j) * px + k0, 0,
                                                      (long long)PZ.wsum * Ny * px - V + 1, 6)) ? -1 : lz0;
#else
    const bool act = act0;
    const int ly = ly0, lz = lz0;
#endif
    // does any lane of the warp touch an x slab?  (the same for all lanes)
    const bool xw = xb * 32 * V < PX.w0 || (xb + 1) * 32 * V - 1 >= PX.edge_max;
    const bool xs = xw && act && (k0 < PX.w0 || k0 + V - 1 >= PX.edge_max);

    if (VEC_PREFETCH > 0 && i + VEC_PREFETCH < Nz && j < Ny && xb * 32 * V < g.Nx) {
        const long long q = (long long)(i + VEC_PREFETCH) * g.plane + (long long)j * px + xb * 32 * V;
#pragma unroll
        for (int c = 0; c < 6; c++) vecb::l2_prefetch<T>(f.c[c] + q, lane, px - xb * 32 * V);
    }

    // ---- every load of the thread first
    T ex[V], ey[V], ez[V], exj[V], ezj[V], exi[V], eyi[V], hx[V], hy[V], hz[V];
    T py0[V], py1[V], pz0[V], pz1[V], px0[V], px1[V];
    int lxs[V];
    vecb::vzero<T>(ex); vecb::vzero<T>(ey); vecb::vzero<T>(ez); vecb::vzero<T>(exj); vecb::vzero<T>(ezj);
    vecb::vzero<T>(exi); vecb::vzero<T>(eyi);
    T ey_n = T(0), ez_n = T(0);
    if (act) {
        vecb::vload<T>(ex, f.c[0] + p); vecb::vload<T>(ey, f.c[1] + p); vecb::vload<T>(ez, f.c[2] + p);
        if (j + 1 < Ny) { vecb::vload<T>(exj, f.c[0] + p + px); vecb::vload<T>(ezj, f.c[2] + p + px); }
        if (i + 1 < Nz || g.zhi) { vecb::vload<T>(exi, f.c[0] + p + Ny * px); vecb::vload<T>(eyi, f.c[1] + p + Ny * px); }
        vecb::vload<T>(hx, f.c[3] + p); vecb::vload<T>(hy, f.c[4] + p); vecb::vload<T>(hz, f.c[5] + p);
        if (lane == 31 && k0 + V < g.Nx) { ey_n = ld(f.c[1] + p + V); ez_n = ld(f.c[2] + p + V); }
        if (ly >= 0) {
            const int s = (i * PY.wsum + ly) * px + k0;
            vecb::vload<T>(py0, PY.psi[0] + s); vecb::vload<T>(py1, PY.psi[1] + s);
        }
        if (lz >= 0) {
            const int s = (lz * Ny + j) * px + k0;
            vecb::vload<T>(pz0, PZ.psi[0] + s); vecb::vload<T>(pz1, PZ.psi[1] + s);
        }
    }
#pragma unroll
    for (int e = 0; e < V; e++) lxs[e] = -1;
    if (xw) {
#pragma unroll
    for (int e = 0; e < V; e++) {
        const int k = k0 + e;
        lxs[e] = (xs && k < g.Nx) ? slab_local(PX, k, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
        if (lxs[e] >= 0 && !vecb::in_range(g, (long long)(i * Ny + j) * PX.wsum + lxs[e], 0,
                                           (long long)Nz * Ny * PX.wsum, 7))
            lxs[e] = -1;
#endif
        if (lxs[e] >= 0) {
            const int s = (i * Ny + j) * PX.wsum + lxs[e];
            px0[e] = ld(PX.psi[0] + s); px1[e] = ld(PX.psi[1] + s);
        }
    }
    }
    T mx[V], my[V], mz[V];
    const bool mu_arr = g.bHarr[0] != nullptr;
    if (mu_arr && act) { vecb::vload<T>(mx, g.bHarr[0] + p); vecb::vload<T>(my, g.bHarr[1] + p); vecb::vload<T>(mz, g.bHarr[2] + p); }
    const bool srcb = src.n && vecb::sources_touch<T>(src, 3, i, j, j + 1,
                                                xb * 32 * V, (xb + 1) * 32 * V);
    double4 st = make_double4(0, 0, 0, 0);
    if (srcb) st = g.step_tab[*step_ctr + off];

    // ---- x neighbour of the last cell: first cell of the next vector
    {
        const T a = __shfl_down_sync(FULL, ey[0], 1), b = __shfl_down_sync(FULL, ez[0], 1);
        if (lane != 31) { ey_n = a; ez_n = b; }
    }
    if (!act) return;
    if (!mu_arr) {
#pragma unroll
        for (int e = 0; e < V; e++) { mx[e] = g.bH[0]; my[e] = g.bH[1]; mz[e] = g.bH[2]; }
    }

#pragma unroll
    for (int e = 0; e < V; e++) {
        const T eyx = e + 1 < V ? ey[e + 1] : ey_n;
        const T ezx = e + 1 < V ? ez[e + 1] : ez_n;
        const T dEzdy = g.ody * (ezj[e] - ez[e]);
        const T dEydz = g.odz * (eyi[e] - ey[e]);
        const T dExdz = g.odz * (exi[e] - ex[e]);
        const T dEzdx = g.odx * (ezx - ez[e]);
        const T dEydx = g.odx * (eyx - ey[e]);
        const T dExdy = g.ody * (exj[e] - ex[e]);
        T Hx = hx[e] + mx[e] * (dEydz - dEzdy);
        T Hy = hy[e] + my[e] * (dEzdx - dExdz);
        T Hz = hz[e] + mz[e] * (dExdy - dEydx);
        if (xw && lxs[e] >= 0) {
            const int l = lxs[e];
            const T kv = ld(PX.kinvH + l), bv = ld(PX.bH + l), cv = ld(PX.cH + l);
            px0[e] = cv * dEydx + bv * px0[e];
            px1[e] = cv * dEzdx + bv * px1[e];
            Hz = Hz - mz[e] * ((px0[e] - dEydx) + dEydx * kv);
            Hy = Hy + my[e] * ((px1[e] - dEzdx) + dEzdx * kv);
        }
        if (ly >= 0) {
            const T kv = ld(PY.kinvH + ly), bv = ld(PY.bH + ly), cv = ld(PY.cH + ly);
            py0[e] = cv * dExdy + bv * py0[e];
            py1[e] = cv * dEzdy + bv * py1[e];
            Hz = Hz + mz[e] * ((py0[e] - dExdy) + dExdy * kv);
            Hx = Hx - mx[e] * ((py1[e] - dEzdy) + dEzdy * kv);
        }
        if (lz >= 0) {
            const T kv = ld(PZ.kinvH + lz), bv = ld(PZ.bH + lz), cv = ld(PZ.cH + lz);
            pz0[e] = cv * dExdz + bv * pz0[e];
            pz1[e] = cv * dEydz + bv * pz1[e];
            Hx = Hx + mx[e] * ((pz1[e] - dEydz) + dEydz * kv);
            Hy = Hy - my[e] * ((pz0[e] - dExdz) + dExdz * kv);
        }
        if (srcb && k0 + e < g.Nx)
            add_sources<T>(src, i, j, k0 + e, 3, T(st.x), T(st.y), Hx, Hy, Hz, false);
        hx[e] = Hx; hy[e] = Hy; hz[e] = Hz;
    }
    vecb::vstore<T>(f.c[3] + p, hx); vecb::vstore<T>(f.c[4] + p, hy); vecb::vstore<T>(f.c[5] + p, hz);
    if (ly >= 0) {
        const int s = (i * PY.wsum + ly) * px + k0;
        vecb::vstore<T>(PY.psi[0] + s, py0); vecb::vstore<T>(PY.psi[1] + s, py1);
    }
    if (lz >= 0) {
        const int s = (lz * Ny + j) * px + k0;
        vecb::vstore<T>(PZ.psi[0] + s, pz0); vecb::vstore<T>(PZ.psi[1] + s, pz1);
    }
    if (xw) {
#pragma unroll
        for (int e = 0; e < V; e++)
            if (lxs[e] >= 0) {
                const int s = (i * Ny + j) * PX.wsum + lxs[e];
                PX.psi[0][s] = px0[e]; PX.psi[1][s] = px1[e];
            }
    }
}

template <typename T>
__device__ __forceinline__ void vec_update_E(const GridView<T>& g, const Fields<T>& f,
                                     const SourceList<T>& src, const long long* step_ctr,
                                     int off, int i, int j, int xb, int lane) {
    constexpr int V = vecb::V16<T>::N;
    constexpr unsigned FULL = 0xffffffffu;
    const int m = xb * 32 + lane;
    const int k0 = m * V;
    const bool act0 = j < g.Ny && k0 < g.Nx;
    const int Ny = g.Ny, px = g.px;
    const int p = act0 ? (i * Ny + j) * px + k0 : 0;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int ly0 = slab_local(PY, j, false);   // same for the whole warp
    const int lz0 = slab_local(PZ, i + PZ.off, true);
#ifdef FDTD_BOUNDS_CHECK
    const bool act = act0 && vecb::e_fields_ok(g, i, j, k0, lane, p);
    const int ly = (ly0 >= 0 && act && !vecb::in_range(g, (long long)(i * PY.wsum + ly0) * px + k0, 0,
                                                      (long long)g.Nz * PY.wsum * px - V + 1, 15)) ? -1 : ly0;
    const int lz = (lz0 >= 0 && act && !vecb::in_range(g, (long long)(lz0 * Ny + j) * px + k0, 0,
                                                      (long long)PZ.wsum * Ny * px - V + 1, 16)) ? -1 : lz0;
#else
    const bool act = act0;
    const int ly = ly0, lz = lz0;
#endif
    // does any lane of the warp touch an x slab?  (the same for all lanes)
    const bool xw = xb * 32 * V < PX.w0 || (xb + 1) * 32 * V - 1 >= PX.edge_max;
    const bool xs = xw && act && (k0 < PX.w0 || k0 + V - 1 >= PX.edge_max);
    const bool lossy = g.aE[0] != nullptr;

    if (VEC_PREFETCH > 0 && i + VEC_PREFETCH < g.Nz && j < Ny && xb * 32 * V < g.Nx) {
        const long long q = (long long)(i + VEC_PREFETCH) * g.plane + (long long)j * px + xb * 32 * V;
#pragma unroll
        for (int c = 0; c < 6; c++) vecb::l2_prefetch<T>(f.c[c] + q, lane, px - xb * 32 * V);
#pragma unroll
        for (int c = 0; c < 3; c++) vecb::l2_prefetch<T>(g.bE[c] + q, lane, px - xb * 32 * V);
    }

    // ---- every load of the thread first
    T hx[V], hy[V], hz[V], hxj[V], hzj[V], hxi[V], hyi[V], ex[V], ey[V], ez[V], bx[V], by[V], bz[V];
    T py2[V], py3[V], pz2[V], pz3[V], px2[V], px3[V], ax[V], ay[V], az[V];
    int lxs[V];
    vecb::vzero<T>(hy); vecb::vzero<T>(hz);
    T hy_p = T(0), hz_p = T(0);
    if (act) {
        vecb::vload<T>(hx, f.c[3] + p); vecb::vload<T>(hy, f.c[4] + p); vecb::vload<T>(hz, f.c[5] + p);
        vecb::vload<T>(ex, f.c[0] + p); vecb::vload<T>(ey, f.c[1] + p); vecb::vload<T>(ez, f.c[2] + p);
        vecb::vload<T>(bx, g.bE[0] + p); vecb::vload<T>(by, g.bE[1] + p); vecb::vload<T>(bz, g.bE[2] + p);
        if (j > 0) { vecb::vload<T>(hxj, f.c[3] + p - px); vecb::vload<T>(hzj, f.c[5] + p - px); }
        if (i > 0 || g.zlo) { vecb::vload<T>(hxi, f.c[3] + p - Ny * px); vecb::vload<T>(hyi, f.c[4] + p - Ny * px); }
        if (lane == 0 && k0 > 0) { hy_p = ld(f.c[4] + p - 1); hz_p = ld(f.c[5] + p - 1); }
        if (ly >= 0) {
            const int s = (i * PY.wsum + ly) * px + k0;
            vecb::vload<T>(py2, PY.psi[2] + s); vecb::vload<T>(py3, PY.psi[3] + s);
        }
        if (lz >= 0) {
            const int s = (lz * Ny + j) * px + k0;
            vecb::vload<T>(pz2, PZ.psi[2] + s); vecb::vload<T>(pz3, PZ.psi[3] + s);
        }
        if (lossy) { vecb::vload<T>(ax, g.aE[0] + p); vecb::vload<T>(ay, g.aE[1] + p); vecb::vload<T>(az, g.aE[2] + p); }
    }
#pragma unroll
    for (int e = 0; e < V; e++) lxs[e] = -1;
    if (xw) {
#pragma unroll
    for (int e = 0; e < V; e++) {
        const int k = k0 + e;
        lxs[e] = (xs && k < g.Nx) ? slab_local(PX, k, false) : -1;
#ifdef FDTD_BOUNDS_CHECK
        if (lxs[e] >= 0 && !vecb::in_range(g, (long long)(i * Ny + j) * PX.wsum + lxs[e], 0,
                                           (long long)g.Nz * Ny * PX.wsum, 17))
            lxs[e] = -1;
#endif
        if (lxs[e] >= 0) {
            const int s = (i * Ny + j) * PX.wsum + lxs[e];
            px2[e] = ld(PX.psi[2] + s); px3[e] = ld(PX.psi[3] + s);
        }
    }
    }
    const bool srcb = src.n && vecb::sources_touch<T>(src, 0, i, j, j + 1,
                                                xb * 32 * V, (xb + 1) * 32 * V);
    double4 st = make_double4(0, 0, 0, 0);
    if (srcb) st = g.step_tab[*step_ctr + off];

    // ---- x neighbour of the first cell: last cell of the previous vector
    {
        const T a = __shfl_up_sync(FULL, hy[V - 1], 1), b = __shfl_up_sync(FULL, hz[V - 1], 1);
        if (lane != 0) { hy_p = a; hz_p = b; }
    }
    if (!act) return;
    if (k0 == 0) { hy_p = h_min_ghost<T>(g.bc[0], hy[0], T(0)); hz_p = h_min_ghost<T>(g.bc[0], hz[0], T(0)); }
    if (j == 0) {
#pragma unroll
        for (int e = 0; e < V; e++) { hxj[e] = h_min_ghost<T>(g.bc[1], hx[e], T(0)); hzj[e] = h_min_ghost<T>(g.bc[1], hz[e], T(0)); }
    }
    if (i == 0 && !g.zlo) {
#pragma unroll
        for (int e = 0; e < V; e++) { hxi[e] = h_min_ghost<T>(g.bc[2], hx[e], T(0)); hyi[e] = h_min_ghost<T>(g.bc[2], hy[e], T(0)); }
    }

#pragma unroll
    for (int e = 0; e < V; e++) {
        const T hyx = e > 0 ? hy[e - 1] : hy_p;
        const T hzx = e > 0 ? hz[e - 1] : hz_p;
        const T dHzdy = g.ody * (hz[e] - hzj[e]);
        const T dHydz = g.odz * (hy[e] - hyi[e]);
        const T dHxdz = g.odz * (hx[e] - hxi[e]);
        const T dHzdx = g.odx * (hz[e] - hzx);
        const T dHydx = g.odx * (hy[e] - hyx);
        const T dHxdy = g.ody * (hx[e] - hxj[e]);
        T Ex, Ey, Ez;
        if (lossy) {
            Ex = ax[e] * ex[e] + (dHzdy - dHydz) * bx[e];
            Ey = ay[e] * ey[e] + (dHxdz - dHzdx) * by[e];
            Ez = az[e] * ez[e] + (dHydx - dHxdy) * bz[e];
        } else {
            Ex = ex[e] + (dHzdy - dHydz) * bx[e];
            Ey = ey[e] + (dHxdz - dHzdx) * by[e];
            Ez = ez[e] + (dHydx - dHxdy) * bz[e];
        }
        if (xw && lxs[e] >= 0) {
            const int l = lxs[e];
            const T kv = ld(PX.kinvE + l), bv = ld(PX.bE + l), cv = ld(PX.cE + l);
            px2[e] = cv * dHydx + bv * px2[e];
            px3[e] = cv * dHzdx + bv * px3[e];
            Ez = Ez + ((px2[e] - dHydx) + dHydx * kv) * bz[e];
            Ey = Ey - ((px3[e] - dHzdx) + dHzdx * kv) * by[e];
        }
        if (ly >= 0) {
            const T kv = ld(PY.kinvE + ly), bv = ld(PY.bE + ly), cv = ld(PY.cE + ly);
            py2[e] = cv * dHxdy + bv * py2[e];
            py3[e] = cv * dHzdy + bv * py3[e];
            Ez = Ez - ((py2[e] - dHxdy) + dHxdy * kv) * bz[e];
            Ex = Ex + ((py3[e] - dHzdy) + dHzdy * kv) * bx[e];
        }
        if (lz >= 0) {
            const T kv = ld(PZ.kinvE + lz), bv = ld(PZ.bE + lz), cv = ld(PZ.cE + lz);
            pz2[e] = cv * dHxdz + bv * pz2[e];
            pz3[e] = cv * dHydz + bv * pz3[e];
            Ex = Ex - ((pz3[e] - dHydz) + dHydz * kv) * bx[e];
            Ey = Ey + ((pz2[e] - dHxdz) + dHxdz * kv) * by[e];
        }
        if (srcb && k0 + e < g.Nx)
            add_sources<T>(src, i, j, k0 + e, 0, T(st.z), T(st.w), Ex, Ey, Ez, true);
        ex[e] = Ex; ey[e] = Ey; ez[e] = Ez;
    }
    vecb::vstore<T>(f.c[0] + p, ex); vecb::vstore<T>(f.c[1] + p, ey); vecb::vstore<T>(f.c[2] + p, ez);
    if (ly >= 0) {
        const int s = (i * PY.wsum + ly) * px + k0;
        vecb::vstore<T>(PY.psi[2] + s, py2); vecb::vstore<T>(PY.psi[3] + s, py3);
    }
    if (lz >= 0) {
        const int s = (lz * Ny + j) * px + k0;
        vecb::vstore<T>(PZ.psi[2] + s, pz2); vecb::vstore<T>(PZ.psi[3] + s, pz3);
    }
    if (xw) {
#pragma unroll
        for (int e = 0; e < V; e++)
            if (lxs[e] >= 0) {
                const int s = (i * Ny + j) * PX.wsum + lxs[e];
                PX.psi[2][s] = px2[e]; PX.psi[3][s] = px3[e];
            }
    }
}

}  // namespace fdtdb
