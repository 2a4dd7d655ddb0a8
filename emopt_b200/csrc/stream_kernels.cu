// stream_kernels.cu -- H and E half-steps as persistent kernels that stream
// row tiles through a shared-memory ring filled by bulk async copies.
//
// The same in-place update as k_update_H / k_update_E (src/fdtd.cpp:121-367
// and :369-755).  The unit of work is a tile: R consecutive rows of one plane,
// all x.  Because rows are contiguous in the [Nz][Ny][px] layout, the part of
// each array a tile needs is one contiguous range of memory, so thread 0 of
// a CTA fetches a whole tile with one 1-D bulk copy per array
// (cp.async.bulk ... mbarrier::complete_tx) into one stage of an S-stage ring
// and keeps S-1 tiles in flight ahead of the computation; no register is held
// by an outstanding load.  For the H update a tile carries E at rows j0..j0+R
// (one row of y halo) and at plane i+1, and H, plus the y- and z-slab CPML
// accumulators of its rows; for the E update H at rows j0-1..j0+R-1 and at
// plane i-1, E, the three coefficients b = dt/eps and the CPML accumulators.
// The x-slab accumulators (a narrow band per row), per-cell dt/mu and the
// lossy coefficients are read with ordinary loads.
//
// Each thread computes one 16-byte vector of x cells (4 floats / 2 doubles)
// per pass from shared memory and stores the result straight to global
// memory.  CPML and source handling are chosen once per tile, so tiles
// outside the slabs run code without CPML terms.  Grid: persistent CTAs
// (SM count x occupancy), CTA c takes tiles c, c + G, c + 2G, ... in plane
// order, so all CTAs sweep the grid together and halo rows are served from
// L2.  Every mbarrier wait is bounded; a wait that runs out sets *err, the
// CTA drains its outstanding copies (again bounded) and stops.
#include <cstring>

#include "async.cuh"
#include "cell.cuh"
#include "kernels.h"

namespace fdtdb {

namespace {

template <typename T>
struct SVec;
template <>
struct SVec<float> {
    using type = float4;
    static constexpr int N = 4;
};
template <>
struct SVec<double> {
    using type = double2;
    static constexpr int N = 2;
};

template <typename T, int V>
__device__ __forceinline__ void vget(T (&d)[V], const T* p) {   // shared or global, 16 B aligned
    using VT = typename SVec<T>::type;
    const VT v = *reinterpret_cast<const VT*>(p);
    if constexpr (V == 4) {
        d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    } else {
        d[0] = v.x; d[1] = v.y;
    }
}

template <typename T, int V>
__device__ __forceinline__ void vput(T* p, const T (&d)[V]) {
    using VT = typename SVec<T>::type;
    VT v;
    if constexpr (V == 4) {
        v.x = d[0]; v.y = d[1]; v.z = d[2]; v.w = d[3];
    } else {
        v.x = d[0]; v.y = d[1];
    }
    *reinterpret_cast<VT*>(p) = v;
}

template <typename T, int V>
__device__ __forceinline__ void vset(T (&d)[V], T x) {
#pragma unroll
    for (int e = 0; e < V; e++) d[e] = x;
}

// Slots of a stage (see StreamPlan::slot).
enum HSlot { HS_EX, HS_EY, HS_EZ, HS_EXN, HS_EYN, HS_HX, HS_HY, HS_HZ, HS_Y0, HS_Y1, HS_Z0, HS_Z1 };
enum ESlot {
    ES_HX, ES_HY, ES_HZ, ES_HXP, ES_HYP, ES_EX, ES_EY, ES_EZ, ES_BX, ES_BY, ES_BZ,
    ES_Y2, ES_Y3, ES_Z2, ES_Z3
};

struct TileGeo {
    int i, j0, rows;
};

__device__ __forceinline__ TileGeo tile_geo(const StreamPlan& P, int Ny, int n) {
    TileGeo t;
    t.i = n / P.nty;
    t.j0 = (n - t.i * P.nty) * P.R;
    t.rows = min(P.R, Ny - t.j0);
    return t;
}

// Calls emit(slot, dst_row, src, nrows) for every y-slab row run of the tile:
// rows of a run are consecutive in the y accumulator layout (i*wy + l)*px.
template <typename T, typename F>
__device__ __forceinline__ void y_runs(const PmlAxis<T>& PY, const TileGeo& t, F&& emit) {
    int r = 0;
    while (r < t.rows) {
        const int l0 = slab_local(PY, t.j0 + r, false);
        if (l0 < 0) { r++; continue; }
        int n = 1;
        while (r + n < t.rows && slab_local(PY, t.j0 + r + n, false) == l0 + n) n++;
        emit(r, l0, n);
        r += n;
    }
}

// Thread 0: issue every copy of tile n into stage s (expected bytes first).
template <typename T>
__device__ void issue_h(const GridView<T>& g, const Fields<T>& f, const StreamPlan& P, int n,
                        unsigned char* stage, uint64_t* bar) {
    const TileGeo t = tile_geo(P, g.Ny, n);
    const int px = g.px, Ny = g.Ny;
    const size_t rb = sizeof(T) * (size_t)px;
    const long long base = ((long long)t.i * Ny + t.j0) * px;
    const bool yhalo = t.j0 + t.rows < Ny, znext = t.i + 1 < g.Nz;
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int lz = slab_local(PZ, t.i, true);
    auto copies = [&](auto&& cp) {
        cp(HS_EX, 0, f.c[0] + base, t.rows + yhalo);
        cp(HS_EY, 0, f.c[1] + base, t.rows);
        cp(HS_EZ, 0, f.c[2] + base, t.rows + yhalo);
        if (znext) {
            cp(HS_EXN, 0, f.c[0] + base + (long long)Ny * px, t.rows);
            cp(HS_EYN, 0, f.c[1] + base + (long long)Ny * px, t.rows);
        }
        cp(HS_HX, 0, f.c[3] + base, t.rows);
        cp(HS_HY, 0, f.c[4] + base, t.rows);
        cp(HS_HZ, 0, f.c[5] + base, t.rows);
        y_runs<T>(PY, t, [&](int r, int l0, int nr) {
            const long long s = ((long long)t.i * PY.wsum + l0) * px;
            cp(HS_Y0, r, PY.psi[0] + s, nr);
            cp(HS_Y1, r, PY.psi[1] + s, nr);
        });
        if (lz >= 0) {
            const long long s = ((long long)lz * Ny + t.j0) * px;
            cp(HS_Z0, 0, PZ.psi[0] + s, t.rows);
            cp(HS_Z1, 0, PZ.psi[1] + s, t.rows);
        }
    };
    uint32_t total = 0;
    copies([&](int, int, const T*, int nr) { total += (uint32_t)(rb * nr); });
    fence_proxy_async();
    mbar_expect_tx(bar, total);
    copies([&](int slot, int r, const T* src, int nr) {
        bulk_load(stage + P.slot[slot] + rb * r, src, (uint32_t)(rb * nr), bar);
    });
}

template <typename T>
__device__ void issue_e(const GridView<T>& g, const Fields<T>& f, const StreamPlan& P, int n,
                        unsigned char* stage, uint64_t* bar) {
    const TileGeo t = tile_geo(P, g.Ny, n);
    const int px = g.px, Ny = g.Ny;
    const size_t rb = sizeof(T) * (size_t)px;
    const long long base = ((long long)t.i * Ny + t.j0) * px;
    const bool ylow = t.j0 > 0, zprev = t.i > 0;
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int lz = slab_local(PZ, t.i, true);
    auto copies = [&](auto&& cp) {
        // slot row 0 of Hx / Hz is row j0 - 1
        cp(ES_HX, ylow ? 0 : 1, f.c[3] + base - (ylow ? px : 0), t.rows + ylow);
        cp(ES_HY, 0, f.c[4] + base, t.rows);
        cp(ES_HZ, ylow ? 0 : 1, f.c[5] + base - (ylow ? px : 0), t.rows + ylow);
        if (zprev) {
            cp(ES_HXP, 0, f.c[3] + base - (long long)Ny * px, t.rows);
            cp(ES_HYP, 0, f.c[4] + base - (long long)Ny * px, t.rows);
        }
        cp(ES_EX, 0, f.c[0] + base, t.rows);
        cp(ES_EY, 0, f.c[1] + base, t.rows);
        cp(ES_EZ, 0, f.c[2] + base, t.rows);
        cp(ES_BX, 0, g.bE[0] + base, t.rows);
        cp(ES_BY, 0, g.bE[1] + base, t.rows);
        cp(ES_BZ, 0, g.bE[2] + base, t.rows);
        y_runs<T>(PY, t, [&](int r, int l0, int nr) {
            const long long s = ((long long)t.i * PY.wsum + l0) * px;
            cp(ES_Y2, r, PY.psi[2] + s, nr);
            cp(ES_Y3, r, PY.psi[3] + s, nr);
        });
        if (lz >= 0) {
            const long long s = ((long long)lz * Ny + t.j0) * px;
            cp(ES_Z2, 0, PZ.psi[2] + s, t.rows);
            cp(ES_Z3, 0, PZ.psi[3] + s, t.rows);
        }
    };
    uint32_t total = 0;
    copies([&](int, int, const T*, int nr) { total += (uint32_t)(rb * nr); });
    fence_proxy_async();
    mbar_expect_tx(bar, total);
    copies([&](int slot, int r, const T* src, int nr) {
        bulk_load(stage + P.slot[slot] + rb * r, src, (uint32_t)(rb * nr), bar);
    });
}

__device__ __forceinline__ bool box_hit(const int* box, const TileGeo& t) {
    return t.i >= box[0] && t.i < box[1] && t.j0 < box[3] && t.j0 + t.rows > box[2];
}

// H update of one vector (cells k0..k0+V-1 of row j = j0 + r).
template <typename T, int V, bool PMLY, bool PMLZ>
__device__ __forceinline__ void h_vec(const GridView<T>& g, const Fields<T>& f,
                                      const SourceList<T>& src, const StreamPlan& P,
                                      const unsigned char* stage, const TileGeo& t, int r, int v,
                                      int lz, bool srcb, T SH, T CH) {
    const int px = g.px, Ny = g.Ny;
    const int j = t.j0 + r, k0 = v * V;
    const long long p = ((long long)t.i * Ny + j) * px + k0;
    auto row = [&](int slot, int rr) {
        return reinterpret_cast<const T*>(stage + P.slot[slot]) + (size_t)rr * px + k0;
    };
    T ex[V], ey[V], ez[V], exj[V], ezj[V], exi[V], eyi[V], hx[V], hy[V], hz[V];
    vget<T, V>(ex, row(HS_EX, r));
    vget<T, V>(ey, row(HS_EY, r));
    vget<T, V>(ez, row(HS_EZ, r));
    if (j + 1 < Ny) { vget<T, V>(exj, row(HS_EX, r + 1)); vget<T, V>(ezj, row(HS_EZ, r + 1)); }
    else { vset<T, V>(exj, T(0)); vset<T, V>(ezj, T(0)); }
    if (t.i + 1 < g.Nz) { vget<T, V>(exi, row(HS_EXN, r)); vget<T, V>(eyi, row(HS_EYN, r)); }
    else { vset<T, V>(exi, T(0)); vset<T, V>(eyi, T(0)); }
    vget<T, V>(hx, row(HS_HX, r));
    vget<T, V>(hy, row(HS_HY, r));
    vget<T, V>(hz, row(HS_HZ, r));
    const bool nxt = v + 1 < P.nvr;
    const T ey_n = nxt ? row(HS_EY, r)[V] : T(0);
    const T ez_n = nxt ? row(HS_EZ, r)[V] : T(0);
    T mx[V], my[V], mz[V];
    if (g.bHarr[0]) {
        vget<T, V>(mx, g.bHarr[0] + p); vget<T, V>(my, g.bHarr[1] + p); vget<T, V>(mz, g.bHarr[2] + p);
    } else {
        vset<T, V>(mx, g.bH[0]); vset<T, V>(my, g.bH[1]); vset<T, V>(mz, g.bH[2]);
    }
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int ly = PMLY ? slab_local(PY, j, false) : -1;
    T py0[V], py1[V], pz0[V], pz1[V];
    T kyv = T(0), byv = T(0), cyv = T(0), kzv = T(0), bzv = T(0), czv = T(0);
    if (PMLY && ly >= 0) {
        vget<T, V>(py0, row(HS_Y0, r)); vget<T, V>(py1, row(HS_Y1, r));
        kyv = ld(PY.kinvH + ly); byv = ld(PY.bH + ly); cyv = ld(PY.cH + ly);
    }
    if (PMLZ) {
        vget<T, V>(pz0, row(HS_Z0, r)); vget<T, V>(pz1, row(HS_Z1, r));
        kzv = ld(PZ.kinvH + lz); bzv = ld(PZ.bH + lz); czv = ld(PZ.cH + lz);
    }
    const bool xs = k0 < PX.w0 || k0 + V - 1 >= PX.edge_max;

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
        if (xs) {
            const int k = k0 + e;
            const int lx = k < g.Nx ? slab_local(PX, k, false) : -1;
            if (lx >= 0) {
                const long long s = ((long long)t.i * Ny + j) * PX.wsum + lx;
                const T kv = ld(PX.kinvH + lx), bv = ld(PX.bH + lx), cv = ld(PX.cH + lx);
                const T q0 = cv * dEydx + bv * ld(PX.psi[0] + s);
                const T q1 = cv * dEzdx + bv * ld(PX.psi[1] + s);
                PX.psi[0][s] = q0; PX.psi[1][s] = q1;
                Hz = Hz - mz[e] * ((q0 - dEydx) + dEydx * kv);
                Hy = Hy + my[e] * ((q1 - dEzdx) + dEzdx * kv);
            }
        }
        if (PMLY && ly >= 0) {
            py0[e] = cyv * dExdy + byv * py0[e];
            py1[e] = cyv * dEzdy + byv * py1[e];
            Hz = Hz + mz[e] * ((py0[e] - dExdy) + dExdy * kyv);
            Hx = Hx - mx[e] * ((py1[e] - dEzdy) + dEzdy * kyv);
        }
        if (PMLZ) {
            pz0[e] = czv * dExdz + bzv * pz0[e];
            pz1[e] = czv * dEydz + bzv * pz1[e];
            Hx = Hx + mx[e] * ((pz1[e] - dEydz) + dEydz * kzv);
            Hy = Hy - my[e] * ((pz0[e] - dExdz) + dExdz * kzv);
        }
        if (srcb && k0 + e < g.Nx) add_sources<T>(src, t.i, j, k0 + e, 3, SH, CH, Hx, Hy, Hz, false);
        hx[e] = Hx; hy[e] = Hy; hz[e] = Hz;
    }
    vput<T, V>(f.c[3] + p, hx); vput<T, V>(f.c[4] + p, hy); vput<T, V>(f.c[5] + p, hz);
    if (PMLY && ly >= 0) {
        const long long s = ((long long)t.i * PY.wsum + ly) * px + k0;
        vput<T, V>(PY.psi[0] + s, py0); vput<T, V>(PY.psi[1] + s, py1);
    }
    if (PMLZ) {
        const long long s = ((long long)lz * Ny + j) * px + k0;
        vput<T, V>(PZ.psi[0] + s, pz0); vput<T, V>(PZ.psi[1] + s, pz1);
    }
}

// E update of one vector (cells k0..k0+V-1 of row j = j0 + r).
template <typename T, int V, bool PMLY, bool PMLZ>
__device__ __forceinline__ void e_vec(const GridView<T>& g, const Fields<T>& f,
                                      const SourceList<T>& src, const StreamPlan& P,
                                      const unsigned char* stage, const TileGeo& t, int r, int v,
                                      int lz, bool srcb, T SE, T CE) {
    const int px = g.px, Ny = g.Ny;
    const int j = t.j0 + r, k0 = v * V;
    const long long p = ((long long)t.i * Ny + j) * px + k0;
    auto row = [&](int slot, int rr) {
        return reinterpret_cast<const T*>(stage + P.slot[slot]) + (size_t)rr * px + k0;
    };
    T hx[V], hy[V], hz[V], hxj[V], hzj[V], hxi[V], hyi[V], ex[V], ey[V], ez[V], bx[V], by[V], bz[V];
    vget<T, V>(hx, row(ES_HX, r + 1));
    vget<T, V>(hy, row(ES_HY, r));
    vget<T, V>(hz, row(ES_HZ, r + 1));
    if (j > 0) { vget<T, V>(hxj, row(ES_HX, r)); vget<T, V>(hzj, row(ES_HZ, r)); }
    else {
#pragma unroll
        for (int e = 0; e < V; e++) {
            hxj[e] = h_min_ghost<T>(g.bc[1], hx[e], T(0));
            hzj[e] = h_min_ghost<T>(g.bc[1], hz[e], T(0));
        }
    }
    if (t.i > 0) { vget<T, V>(hxi, row(ES_HXP, r)); vget<T, V>(hyi, row(ES_HYP, r)); }
    else {
#pragma unroll
        for (int e = 0; e < V; e++) {
            hxi[e] = h_min_ghost<T>(g.bc[2], hx[e], T(0));
            hyi[e] = h_min_ghost<T>(g.bc[2], hy[e], T(0));
        }
    }
    vget<T, V>(ex, row(ES_EX, r));
    vget<T, V>(ey, row(ES_EY, r));
    vget<T, V>(ez, row(ES_EZ, r));
    vget<T, V>(bx, row(ES_BX, r));
    vget<T, V>(by, row(ES_BY, r));
    vget<T, V>(bz, row(ES_BZ, r));
    T hy_p, hz_p;
    if (v > 0) {
        hy_p = row(ES_HY, r)[-1];
        hz_p = row(ES_HZ, r + 1)[-1];
    } else {
        hy_p = h_min_ghost<T>(g.bc[0], hy[0], T(0));
        hz_p = h_min_ghost<T>(g.bc[0], hz[0], T(0));
    }
    const bool lossy = g.aE[0] != nullptr;
    T ax[V], ay[V], az[V];
    if (lossy) { vget<T, V>(ax, g.aE[0] + p); vget<T, V>(ay, g.aE[1] + p); vget<T, V>(az, g.aE[2] + p); }
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int ly = PMLY ? slab_local(PY, j, false) : -1;
    T py2[V], py3[V], pz2[V], pz3[V];
    T kyv = T(0), byv = T(0), cyv = T(0), kzv = T(0), bzv = T(0), czv = T(0);
    if (PMLY && ly >= 0) {
        vget<T, V>(py2, row(ES_Y2, r)); vget<T, V>(py3, row(ES_Y3, r));
        kyv = ld(PY.kinvE + ly); byv = ld(PY.bE + ly); cyv = ld(PY.cE + ly);
    }
    if (PMLZ) {
        vget<T, V>(pz2, row(ES_Z2, r)); vget<T, V>(pz3, row(ES_Z3, r));
        kzv = ld(PZ.kinvE + lz); bzv = ld(PZ.bE + lz); czv = ld(PZ.cE + lz);
    }
    const bool xs = k0 < PX.w0 || k0 + V - 1 >= PX.edge_max;

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
        if (xs) {
            const int k = k0 + e;
            const int lx = k < g.Nx ? slab_local(PX, k, false) : -1;
            if (lx >= 0) {
                const long long s = ((long long)t.i * Ny + j) * PX.wsum + lx;
                const T kv = ld(PX.kinvE + lx), bv = ld(PX.bE + lx), cv = ld(PX.cE + lx);
                const T q2 = cv * dHydx + bv * ld(PX.psi[2] + s);
                const T q3 = cv * dHzdx + bv * ld(PX.psi[3] + s);
                PX.psi[2][s] = q2; PX.psi[3][s] = q3;
                Ez = Ez + ((q2 - dHydx) + dHydx * kv) * bz[e];
                Ey = Ey - ((q3 - dHzdx) + dHzdx * kv) * by[e];
            }
        }
        if (PMLY && ly >= 0) {
            py2[e] = cyv * dHxdy + byv * py2[e];
            py3[e] = cyv * dHzdy + byv * py3[e];
            Ez = Ez - ((py2[e] - dHxdy) + dHxdy * kyv) * bz[e];
            Ex = Ex + ((py3[e] - dHzdy) + dHzdy * kyv) * bx[e];
        }
        if (PMLZ) {
            pz2[e] = czv * dHxdz + bzv * pz2[e];
            pz3[e] = czv * dHydz + bzv * pz3[e];
            Ex = Ex - ((pz3[e] - dHydz) + dHydz * kzv) * bx[e];
            Ey = Ey + ((pz2[e] - dHxdz) + dHxdz * kzv) * by[e];
        }
        if (srcb && k0 + e < g.Nx) add_sources<T>(src, t.i, j, k0 + e, 0, SE, CE, Ex, Ey, Ez, true);
        ex[e] = Ex; ey[e] = Ey; ez[e] = Ez;
    }
    vput<T, V>(f.c[0] + p, ex); vput<T, V>(f.c[1] + p, ey); vput<T, V>(f.c[2] + p, ez);
    if (PMLY && ly >= 0) {
        const long long s = ((long long)t.i * PY.wsum + ly) * px + k0;
        vput<T, V>(PY.psi[2] + s, py2); vput<T, V>(PY.psi[3] + s, py3);
    }
    if (PMLZ) {
        const long long s = ((long long)lz * Ny + j) * px + k0;
        vput<T, V>(PZ.psi[2] + s, pz2); vput<T, V>(PZ.psi[3] + s, pz3);
    }
}

// One tile: every thread takes vectors q = tid, tid + blockDim, ... of the
// tile's rows x nvr vectors, with the CPML variant chosen per tile.
template <typename T, bool IS_E>
__device__ __forceinline__ void tile_compute(const GridView<T>& g, const Fields<T>& f,
                                             const SourceList<T>& src, const StreamPlan& P,
                                             const unsigned char* stage, const TileGeo& t, T S,
                                             T C) {
    constexpr int V = SVec<T>::N;
    const PmlAxis<T>& PY = g.pml[1];
    const int lz = slab_local(g.pml[2], t.i, true);
    const bool ty = t.j0 < PY.w0 || t.j0 + t.rows - 1 >= PY.edge_max;
    const bool tz = lz >= 0;
    const bool srcb = box_hit(IS_E ? P.ebox : P.hbox, t);
    const int nq = t.rows * P.nvr;
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int r = (int)__umulhi((unsigned)q, P.magic);
        const int v = q - r * P.nvr;
        if (IS_E) {
            if (ty && tz) e_vec<T, V, true, true>(g, f, src, P, stage, t, r, v, lz, srcb, S, C);
            else if (ty) e_vec<T, V, true, false>(g, f, src, P, stage, t, r, v, lz, srcb, S, C);
            else if (tz) e_vec<T, V, false, true>(g, f, src, P, stage, t, r, v, lz, srcb, S, C);
            else e_vec<T, V, false, false>(g, f, src, P, stage, t, r, v, lz, srcb, S, C);
        } else {
            if (ty && tz) h_vec<T, V, true, true>(g, f, src, P, stage, t, r, v, lz, srcb, S, C);
            else if (ty) h_vec<T, V, true, false>(g, f, src, P, stage, t, r, v, lz, srcb, S, C);
            else if (tz) h_vec<T, V, false, true>(g, f, src, P, stage, t, r, v, lz, srcb, S, C);
            else h_vec<T, V, false, false>(g, f, src, P, stage, t, r, v, lz, srcb, S, C);
        }
    }
}

}  // namespace

template <typename T, bool IS_E>
__global__ void __launch_bounds__(256) k_stream(const __grid_constant__ GridView<T> g, Fields<T> f,
                                                const __grid_constant__ SourceList<T> src,
                                                const __grid_constant__ StreamPlan P,
                                                const long long* __restrict__ step_base, int off,
                                                int* err) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((128 - (smem_addr(smem_raw) & 127)) & 127);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)P.S * P.stage_bytes);
    const int G = gridDim.x, c = blockIdx.x;

    if (threadIdx.x == 0) {
        for (int s = 0; s < P.S; s++) mbar_init(&bars[s], 1);
        fence_mbar_init();
        for (int u = 0; u < P.S && c + u * G < P.ntiles; u++) {
            if (IS_E) issue_e<T>(g, f, P, c + u * G, smem + (size_t)u * P.stage_bytes, &bars[u]);
            else issue_h<T>(g, f, P, c + u * G, smem + (size_t)u * P.stage_bytes, &bars[u]);
        }
    }
    __syncthreads();

    T S = T(0), C = T(0);
    const int* box = IS_E ? P.ebox : P.hbox;
    if (box[0] < box[1]) {
        const double4 st = g.step_tab[*step_base + off];
        S = T(IS_E ? st.z : st.x);
        C = T(IS_E ? st.w : st.y);
    }

    int u = 0;
    bool failed = false;
    for (;; u++) {
        const int n = c + u * G;
        if (n >= P.ntiles) break;
        const int s = u % P.S;
        const bool ok = mbar_wait(&bars[s], (uint32_t)((u / P.S) & 1), err);
        if (__syncthreads_or(!ok)) { failed = true; break; }
        const TileGeo t = tile_geo(P, g.Ny, n);
        tile_compute<T, IS_E>(g, f, src, P, smem + (size_t)s * P.stage_bytes, t, S, C);
        __syncthreads();
        const int n2 = n + P.S * G;
        if (threadIdx.x == 0 && n2 < P.ntiles) {
            if (IS_E) issue_e<T>(g, f, P, n2, smem + (size_t)s * P.stage_bytes, &bars[s]);
            else issue_h<T>(g, f, P, n2, smem + (size_t)s * P.stage_bytes, &bars[s]);
        }
    }
    if (failed && threadIdx.x == 0) {
        // copies of tiles u .. u+S-1 may still be in flight into the ring
        for (int w = u; w < u + P.S && c + w * G < P.ntiles; w++)
            mbar_wait(&bars[w % P.S], (uint32_t)((w / P.S) & 1), err);
    }
}

// ------------------------------------------------------------------ host
namespace {

template <typename T>
int stage_layout(int R, int px, bool is_e, int* slot) {
    const int rb = (int)sizeof(T) * px;   // a multiple of 128
    const int nslots = is_e ? 15 : 12;
    int off = 0;
    for (int q = 0; q < 16; q++) slot[q] = 0;
    for (int q = 0; q < nslots; q++) {
        const bool halo = is_e ? (q == ES_HX || q == ES_HZ) : (q == HS_EX || q == HS_EZ);
        slot[q] = off;
        off += rb * (R + (halo ? 1 : 0));
    }
    return off;
}

constexpr int kSmemMax = 227 * 1024;
constexpr int kSmemPad = 128 + 64;   // alignment slack + barriers

// Planes [b0, b1) and rows [b2, b3) touched by the sources that drive E
// (side 0: Jx, Jy, Jz) or H (side 1: Mx, My, Mz); empty when b0 >= b1.
template <typename T>
void source_box(const SourceList<T>& src, int side, int* b) {
    b[0] = 1 << 30; b[1] = -1; b[2] = 1 << 30; b[3] = -1;
    for (int q = 0; q < src.n; q++) {
        const DevSource<T>& s = src.s[q];
        const bool drives = s.comp[3 * side] || s.comp[3 * side + 1] || s.comp[3 * side + 2];
        if (!drives || s.I <= 0 || s.J <= 0 || s.K <= 0) continue;
        if (s.i0 < b[0]) b[0] = s.i0;
        if (s.i0 + s.I > b[1]) b[1] = s.i0 + s.I;
        if (s.j0 < b[2]) b[2] = s.j0;
        if (s.j0 + s.J > b[3]) b[3] = s.j0 + s.J;
    }
}

}  // namespace

template <typename T>
cudaError_t stream_plan(const GridView<T>& g, int rows_hint, StreamPlan* P) {
    constexpr int V = SVec<T>::N;
    memset(P, 0, sizeof(*P));
    const int nvr = (g.Nx + V - 1) / V;
    if (nvr < 2 || g.Ny <= 0 || g.Nz <= 0) return cudaErrorInvalidValue;
    // R rows per tile, S stages: the largest R (<= 4, or the hint) that leaves
    // room for 3-4 stages of the larger (E) stage; else R = 1 with 2 stages.
    int R = 0, S = 0;
    int hs[16], es[16];
    for (int r = (rows_hint > 0 ? rows_hint : 4); r >= 1 && !R; r--) {
        const int eb = stage_layout<T>(r, g.px, true, es);
        for (int s = 4; s >= 3; s--)
            if (s * eb + kSmemPad <= kSmemMax) { R = r; S = s; break; }
    }
    if (!R) {
        const int eb = stage_layout<T>(1, g.px, true, es);
        if (2 * eb + kSmemPad > kSmemMax) return cudaErrorInvalidValue;
        R = 1; S = 2;
    }
    P->R = R;
    P->S = S;
    P->nty = (g.Ny + R - 1) / R;
    P->ntiles = P->nty * g.Nz;
    P->nvr = nvr;
    const int nq = R * nvr;
    P->threads = nq >= 256 ? 256 : ((nq + 31) / 32 * 32 < 128 ? 128 : (nq + 31) / 32 * 32);
    const unsigned long long two32 = 1ull << 32;
    const unsigned long long magic = (two32 + nvr - 1) / nvr;
    const unsigned long long errm = magic * (unsigned long long)nvr - two32;
    if (errm * (unsigned long long)(nq + P->threads) >= two32) return cudaErrorInvalidValue;
    P->magic = (unsigned)magic;
    const int hb = stage_layout<T>(R, g.px, false, hs);
    const int eb = stage_layout<T>(R, g.px, true, es);
    P->stage_bytes = eb > hb ? eb : hb;
    P->smem = S * P->stage_bytes + kSmemPad;
    for (int q = 0; q < 16; q++) { P->hslot[q] = hs[q]; P->eslot[q] = es[q]; }

    int dev = 0, nsm = 0, occ_h = 0, occ_e = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_stream<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  P->smem)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_stream<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  P->smem)) != cudaSuccess)
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, k_stream<T, false>, P->threads,
                                                           P->smem)) != cudaSuccess)
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_e, k_stream<T, true>, P->threads,
                                                           P->smem)) != cudaSuccess)
        return e;
    int occ = occ_h < occ_e ? occ_h : occ_e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    long long grid = (long long)nsm * occ;
    P->grid = (int)(grid < P->ntiles ? grid : P->ntiles);
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_step_stream(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                               const long long* step_base, int off, const StreamPlan& plan,
                               int* err, cudaStream_t st) {
    StreamPlan ph = plan, pe = plan;
    for (int q = 0; q < 16; q++) { ph.slot[q] = plan.hslot[q]; pe.slot[q] = plan.eslot[q]; }
    source_box<T>(src, 1, ph.hbox);
    source_box<T>(src, 0, ph.ebox);
    for (int q = 0; q < 4; q++) { pe.hbox[q] = ph.hbox[q]; pe.ebox[q] = ph.ebox[q]; }
    Fields<T> f;
    for (int c = 0; c < 6; c++) f.c[c] = fields[c];
    k_stream<T, false><<<plan.grid, plan.threads, plan.smem, st>>>(g, f, src, ph, step_base, off, err);
    k_stream<T, true><<<plan.grid, plan.threads, plan.smem, st>>>(g, f, src, pe, step_base, off, err);
    return cudaGetLastError();
}

template cudaError_t stream_plan<float>(const GridView<float>&, int, StreamPlan*);
template cudaError_t stream_plan<double>(const GridView<double>&, int, StreamPlan*);
template cudaError_t launch_step_stream<float>(const GridView<float>&, float* const*,
                                               const SourceList<float>&, const long long*, int,
                                               const StreamPlan&, int*, cudaStream_t);
template cudaError_t launch_step_stream<double>(const GridView<double>&, double* const*,
                                                const SourceList<double>&, const long long*, int,
                                                const StreamPlan&, int*, cudaStream_t);

}  // namespace fdtdb
