// vec4_kernels.cu -- H and E half-steps, one 16-byte vector of x cells per
// thread, threads laid over flattened (row, vector) pairs of a plane.
//
// The same in-place update as k_update_H / k_update_E (src/fdtd.cpp:121-367
// and :369-755).  A thread owns V consecutive x cells of one row: V = 4 floats
// (float4) or V = 2 doubles (double2), so every field, coefficient and y/z-slab
// CPML access is one aligned 16-byte load or store (rows start on 128-byte
// boundaries, px is a multiple of 32).  The threads of a block cover
// consecutive vectors of the plane's Ny x nvec (row, vector) pairs, so no lane
// idles at the end of a row; a warp may span two rows.  The x neighbour across
// the vector boundary comes from the adjacent lane by shuffle when that lane
// holds the same row, by one scalar load at the warp edge, and from the
// boundary rule at the row ends.  Every load of a thread -- fields, CPML
// state and the CPML coefficients of its slab positions -- is issued before
// the first dependent instruction.
//
// Padding cells (k >= Nx) rely on one invariant: the E coefficients b = dt/eps
// are zero there, so E stays zero in the padding and serves as the x-max PEC
// ghost of src/fdtd.cpp:142-151; H in the padding then stays zero as well.
#include "cell.cuh"
#include "kernels.h"

// Threads per block: single warps free their slot as soon as they finish
// (139 us per step against 200 us with 256-thread blocks, 321 x 161 x 101
// MMI block, fp32).
#ifndef V16_BLOCK
#define V16_BLOCK 32
#endif

namespace fdtdb {

namespace {

template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int N = 4;
};
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int N = 2;
};

template <typename T, int V>
__device__ __forceinline__ void vld(T (&d)[V], const T* p) {
    using VT = typename Vec16<T>::type;
    const VT v = __ldg(reinterpret_cast<const VT*>(p));
    if constexpr (V == 4) {
        d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    } else {
        d[0] = v.x; d[1] = v.y;
    }
}

template <typename T, int V>
__device__ __forceinline__ void vst(T* p, const T (&d)[V]) {
    using VT = typename Vec16<T>::type;
    VT v;
    if constexpr (V == 4) {
        v.x = d[0]; v.y = d[1]; v.z = d[2]; v.w = d[3];
    } else {
        v.x = d[0]; v.y = d[1];
    }
    *reinterpret_cast<VT*>(p) = v;
}

template <typename T, int V>
__device__ __forceinline__ void vzero(T (&d)[V]) {
#pragma unroll
    for (int e = 0; e < V; e++) d[e] = T(0);
}

// Does a source box with a non-zero component among comp_base..comp_base+2
// touch rows [j0, j1] of plane i?
template <typename T>
__device__ __forceinline__ bool sources_touch_rows(const SourceList<T>& src, int comp_base, int i,
                                                   int j0, int j1) {
    bool hit = false;
    for (int q = 0; q < src.n; q++) {
        const DevSource<T>& s = src.s[q];
        const bool drives = s.comp[comp_base] || s.comp[comp_base + 1] || s.comp[comp_base + 2];
        hit |= drives && i >= s.i0 && i < s.i0 + s.I && s.j0 <= j1 && s.j0 + s.J > j0;
    }
    return hit;
}

// CPML coefficients of one slab position (1/kappa, b, c).
template <typename T>
struct Coef3 {
    T kinv, b, c;
};

template <typename T>
__device__ __forceinline__ Coef3<T> coef(const T* kinv, const T* b, const T* c, int l) {
    Coef3<T> r;
    r.kinv = ld(kinv + l);
    r.b = ld(b + l);
    r.c = ld(c + l);
    return r;
}

}  // namespace

template <typename T>
__global__ void __launch_bounds__(V16_BLOCK) k_update_H_v16(GridView<T> g, Fields<T> f, SourceList<T> src,
                                                      const long long* step_base, int off,
                                                      int nvec, unsigned magic) {
    constexpr int V = Vec16<T>::N;
    constexpr unsigned FULL = 0xffffffffu;
    const int Ny = g.Ny, Nz = g.Nz, px = g.px;
    const int i = blockIdx.y;
    const unsigned t = blockIdx.x * (unsigned)V16_BLOCK + threadIdx.x;
    const int j = (int)__umulhi(t, magic);
    const int v = (int)t - j * nvec;
    const int k0 = v * V;
    const int lane = threadIdx.x & 31;
    const bool act = j < Ny;
    const int p = act ? (i * Ny + j) * px + k0 : 0;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int ly = act ? slab_local(PY, j, false) : -1;
    const int lz = slab_local(PZ, i, true);
    const bool xs = act && (k0 < PX.w0 || k0 + V - 1 >= PX.edge_max);

    // ---- every load of the thread first
    T ex[V], ey[V], ez[V], exj[V], ezj[V], exi[V], eyi[V], hx[V], hy[V], hz[V];
    T py0[V], py1[V], pz0[V], pz1[V], px0[V], px1[V];
    int lxs[V];
    Coef3<T> cx[V], cy, cz;
    vzero<T, V>(ey); vzero<T, V>(ez); vzero<T, V>(exj); vzero<T, V>(ezj);
    vzero<T, V>(exi); vzero<T, V>(eyi);
    T ey_n = T(0), ez_n = T(0);
    if (act) {
        vld<T, V>(ex, f.c[0] + p); vld<T, V>(ey, f.c[1] + p); vld<T, V>(ez, f.c[2] + p);
        if (j + 1 < Ny) { vld<T, V>(exj, f.c[0] + p + px); vld<T, V>(ezj, f.c[2] + p + px); }
        if (i + 1 < Nz) { vld<T, V>(exi, f.c[0] + p + Ny * px); vld<T, V>(eyi, f.c[1] + p + Ny * px); }
        vld<T, V>(hx, f.c[3] + p); vld<T, V>(hy, f.c[4] + p); vld<T, V>(hz, f.c[5] + p);
        if (lane == 31 && v + 1 < nvec) { ey_n = ld(f.c[1] + p + V); ez_n = ld(f.c[2] + p + V); }
        if (ly >= 0) {
            const int s = (i * PY.wsum + ly) * px + k0;
            vld<T, V>(py0, PY.psi[0] + s); vld<T, V>(py1, PY.psi[1] + s);
            cy = coef<T>(PY.kinvH, PY.bH, PY.cH, ly);
        }
        if (lz >= 0) {
            const int s = (lz * Ny + j) * px + k0;
            vld<T, V>(pz0, PZ.psi[0] + s); vld<T, V>(pz1, PZ.psi[1] + s);
            cz = coef<T>(PZ.kinvH, PZ.bH, PZ.cH, lz);
        }
    }
#pragma unroll
    for (int e = 0; e < V; e++) {
        const int k = k0 + e;
        lxs[e] = (xs && k < g.Nx) ? slab_local(PX, k, false) : -1;
        if (lxs[e] >= 0) {
            const int s = (i * Ny + j) * PX.wsum + lxs[e];
            px0[e] = ld(PX.psi[0] + s); px1[e] = ld(PX.psi[1] + s);
            cx[e] = coef<T>(PX.kinvH, PX.bH, PX.cH, lxs[e]);
        }
    }
    T mx[V], my[V], mz[V];
    const bool mu_arr = g.bHarr[0] != nullptr;
    if (mu_arr && act) { vld<T, V>(mx, g.bHarr[0] + p); vld<T, V>(my, g.bHarr[1] + p); vld<T, V>(mz, g.bHarr[2] + p); }
    const int jb0 = (int)__umulhi(blockIdx.x * (unsigned)V16_BLOCK, magic);
    const bool srcb = src.n && sources_touch_rows<T>(src, 3, i, jb0, jb0 + V16_BLOCK / nvec + 1);
    double4 st = make_double4(0, 0, 0, 0);
    if (srcb) st = g.step_tab[*step_base + off];

    // ---- x neighbour of the last cell: first cell of the next vector of the row
    {
        const T a = __shfl_down_sync(FULL, ey[0], 1), b = __shfl_down_sync(FULL, ez[0], 1);
        if (lane != 31) { ey_n = a; ez_n = b; }
        if (v + 1 >= nvec) { ey_n = T(0); ez_n = T(0); }
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
        if (lxs[e] >= 0) {
            const Coef3<T> c = cx[e];
            px0[e] = c.c * dEydx + c.b * px0[e];
            px1[e] = c.c * dEzdx + c.b * px1[e];
            Hz = Hz - mz[e] * ((px0[e] - dEydx) + dEydx * c.kinv);
            Hy = Hy + my[e] * ((px1[e] - dEzdx) + dEzdx * c.kinv);
        }
        if (ly >= 0) {
            py0[e] = cy.c * dExdy + cy.b * py0[e];
            py1[e] = cy.c * dEzdy + cy.b * py1[e];
            Hz = Hz + mz[e] * ((py0[e] - dExdy) + dExdy * cy.kinv);
            Hx = Hx - mx[e] * ((py1[e] - dEzdy) + dEzdy * cy.kinv);
        }
        if (lz >= 0) {
            pz0[e] = cz.c * dExdz + cz.b * pz0[e];
            pz1[e] = cz.c * dEydz + cz.b * pz1[e];
            Hx = Hx + mx[e] * ((pz1[e] - dEydz) + dEydz * cz.kinv);
            Hy = Hy - my[e] * ((pz0[e] - dExdz) + dExdz * cz.kinv);
        }
        if (srcb && k0 + e < g.Nx)
            add_sources<T>(src, i, j, k0 + e, 3, T(st.x), T(st.y), Hx, Hy, Hz, false);
        hx[e] = Hx; hy[e] = Hy; hz[e] = Hz;
    }
    vst<T, V>(f.c[3] + p, hx); vst<T, V>(f.c[4] + p, hy); vst<T, V>(f.c[5] + p, hz);
    if (ly >= 0) {
        const int s = (i * PY.wsum + ly) * px + k0;
        vst<T, V>(PY.psi[0] + s, py0); vst<T, V>(PY.psi[1] + s, py1);
    }
    if (lz >= 0) {
        const int s = (lz * Ny + j) * px + k0;
        vst<T, V>(PZ.psi[0] + s, pz0); vst<T, V>(PZ.psi[1] + s, pz1);
    }
#pragma unroll
    for (int e = 0; e < V; e++)
        if (lxs[e] >= 0) {
            const int s = (i * Ny + j) * PX.wsum + lxs[e];
            PX.psi[0][s] = px0[e]; PX.psi[1][s] = px1[e];
        }
}

template <typename T>
__global__ void __launch_bounds__(V16_BLOCK) k_update_E_v16(GridView<T> g, Fields<T> f, SourceList<T> src,
                                                      const long long* step_base, int off,
                                                      int nvec, unsigned magic) {
    constexpr int V = Vec16<T>::N;
    constexpr unsigned FULL = 0xffffffffu;
    const int Ny = g.Ny, px = g.px;
    const int i = blockIdx.y;
    const unsigned t = blockIdx.x * (unsigned)V16_BLOCK + threadIdx.x;
    const int j = (int)__umulhi(t, magic);
    const int v = (int)t - j * nvec;
    const int k0 = v * V;
    const int lane = threadIdx.x & 31;
    const bool act = j < Ny;
    const int p = act ? (i * Ny + j) * px + k0 : 0;
    const PmlAxis<T>& PX = g.pml[0];
    const PmlAxis<T>& PY = g.pml[1];
    const PmlAxis<T>& PZ = g.pml[2];
    const int ly = act ? slab_local(PY, j, false) : -1;
    const int lz = slab_local(PZ, i, true);
    const bool xs = act && (k0 < PX.w0 || k0 + V - 1 >= PX.edge_max);
    const bool lossy = g.aE[0] != nullptr;

    // ---- every load of the thread first
    T hx[V], hy[V], hz[V], hxj[V], hzj[V], hxi[V], hyi[V], ex[V], ey[V], ez[V], bx[V], by[V], bz[V];
    T py2[V], py3[V], pz2[V], pz3[V], px2[V], px3[V], ax[V], ay[V], az[V];
    int lxs[V];
    Coef3<T> cx[V], cy, cz;
    vzero<T, V>(hy); vzero<T, V>(hz);
    T hy_p = T(0), hz_p = T(0);
    if (act) {
        vld<T, V>(hx, f.c[3] + p); vld<T, V>(hy, f.c[4] + p); vld<T, V>(hz, f.c[5] + p);
        vld<T, V>(ex, f.c[0] + p); vld<T, V>(ey, f.c[1] + p); vld<T, V>(ez, f.c[2] + p);
        vld<T, V>(bx, g.bE[0] + p); vld<T, V>(by, g.bE[1] + p); vld<T, V>(bz, g.bE[2] + p);
        if (j > 0) { vld<T, V>(hxj, f.c[3] + p - px); vld<T, V>(hzj, f.c[5] + p - px); }
        if (i > 0) { vld<T, V>(hxi, f.c[3] + p - Ny * px); vld<T, V>(hyi, f.c[4] + p - Ny * px); }
        if (lane == 0 && v > 0) { hy_p = ld(f.c[4] + p - 1); hz_p = ld(f.c[5] + p - 1); }
        if (ly >= 0) {
            const int s = (i * PY.wsum + ly) * px + k0;
            vld<T, V>(py2, PY.psi[2] + s); vld<T, V>(py3, PY.psi[3] + s);
            cy = coef<T>(PY.kinvE, PY.bE, PY.cE, ly);
        }
        if (lz >= 0) {
            const int s = (lz * Ny + j) * px + k0;
            vld<T, V>(pz2, PZ.psi[2] + s); vld<T, V>(pz3, PZ.psi[3] + s);
            cz = coef<T>(PZ.kinvE, PZ.bE, PZ.cE, lz);
        }
        if (lossy) { vld<T, V>(ax, g.aE[0] + p); vld<T, V>(ay, g.aE[1] + p); vld<T, V>(az, g.aE[2] + p); }
    }
#pragma unroll
    for (int e = 0; e < V; e++) {
        const int k = k0 + e;
        lxs[e] = (xs && k < g.Nx) ? slab_local(PX, k, false) : -1;
        if (lxs[e] >= 0) {
            const int s = (i * Ny + j) * PX.wsum + lxs[e];
            px2[e] = ld(PX.psi[2] + s); px3[e] = ld(PX.psi[3] + s);
            cx[e] = coef<T>(PX.kinvE, PX.bE, PX.cE, lxs[e]);
        }
    }
    const int jb0 = (int)__umulhi(blockIdx.x * (unsigned)V16_BLOCK, magic);
    const bool srcb = src.n && sources_touch_rows<T>(src, 0, i, jb0, jb0 + V16_BLOCK / nvec + 1);
    double4 st = make_double4(0, 0, 0, 0);
    if (srcb) st = g.step_tab[*step_base + off];

    // ---- x neighbour of the first cell: last cell of the previous vector of the row
    {
        const T a = __shfl_up_sync(FULL, hy[V - 1], 1), b = __shfl_up_sync(FULL, hz[V - 1], 1);
        if (lane != 0) { hy_p = a; hz_p = b; }
    }
    if (!act) return;
    if (v == 0) { hy_p = h_min_ghost<T>(g.bc[0], hy[0], T(0)); hz_p = h_min_ghost<T>(g.bc[0], hz[0], T(0)); }
    if (j == 0) {
#pragma unroll
        for (int e = 0; e < V; e++) { hxj[e] = h_min_ghost<T>(g.bc[1], hx[e], T(0)); hzj[e] = h_min_ghost<T>(g.bc[1], hz[e], T(0)); }
    }
    if (i == 0) {
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
        if (lxs[e] >= 0) {
            const Coef3<T> c = cx[e];
            px2[e] = c.c * dHydx + c.b * px2[e];
            px3[e] = c.c * dHzdx + c.b * px3[e];
            Ez = Ez + ((px2[e] - dHydx) + dHydx * c.kinv) * bz[e];
            Ey = Ey - ((px3[e] - dHzdx) + dHzdx * c.kinv) * by[e];
        }
        if (ly >= 0) {
            py2[e] = cy.c * dHxdy + cy.b * py2[e];
            py3[e] = cy.c * dHzdy + cy.b * py3[e];
            Ez = Ez - ((py2[e] - dHxdy) + dHxdy * cy.kinv) * bz[e];
            Ex = Ex + ((py3[e] - dHzdy) + dHzdy * cy.kinv) * bx[e];
        }
        if (lz >= 0) {
            pz2[e] = cz.c * dHxdz + cz.b * pz2[e];
            pz3[e] = cz.c * dHydz + cz.b * pz3[e];
            Ex = Ex - ((pz3[e] - dHydz) + dHydz * cz.kinv) * bx[e];
            Ey = Ey + ((pz2[e] - dHxdz) + dHxdz * cz.kinv) * by[e];
        }
        if (srcb && k0 + e < g.Nx)
            add_sources<T>(src, i, j, k0 + e, 0, T(st.z), T(st.w), Ex, Ey, Ez, true);
        ex[e] = Ex; ey[e] = Ey; ez[e] = Ez;
    }
    vst<T, V>(f.c[0] + p, ex); vst<T, V>(f.c[1] + p, ey); vst<T, V>(f.c[2] + p, ez);
    if (ly >= 0) {
        const int s = (i * PY.wsum + ly) * px + k0;
        vst<T, V>(PY.psi[2] + s, py2); vst<T, V>(PY.psi[3] + s, py3);
    }
    if (lz >= 0) {
        const int s = (lz * Ny + j) * px + k0;
        vst<T, V>(PZ.psi[2] + s, pz2); vst<T, V>(PZ.psi[3] + s, pz3);
    }
#pragma unroll
    for (int e = 0; e < V; e++)
        if (lxs[e] >= 0) {
            const int s = (i * Ny + j) * PX.wsum + lxs[e];
            PX.psi[2][s] = px2[e]; PX.psi[3][s] = px3[e];
        }
}

// Row split of the flattened index: j = umulhi(t, magic) must equal t / nvec
// for every t < Ny * nvec.  magic = ceil(2^32 / nvec) has error e = magic*nvec
// - 2^32 < nvec, and the quotient is exact while t * e < 2^32.
bool v16_magic(int Nx, int Ny, int V, int* nvec_out, unsigned* magic_out) {
    const long long nvec = (Nx + V - 1) / V;
    if (nvec <= 0 || Ny <= 0) return false;
    const unsigned long long two32 = 1ull << 32;
    const unsigned long long magic = (two32 + nvec - 1) / nvec;
    if (magic >= two32) {   // nvec == 1
        return false;
    }
    const unsigned long long err = magic * nvec - two32;
    const unsigned long long tmax = (unsigned long long)Ny * nvec + V16_BLOCK;   // incl. the block tail
    if (err * tmax >= two32) return false;
    *nvec_out = (int)nvec;
    *magic_out = (unsigned)magic;
    return true;
}

template <typename T>
cudaError_t launch_step_v16(const GridView<T>& g, T* const* fields, const SourceList<T>& src,
                            const long long* step_base, int off, cudaStream_t st) {
    constexpr int V = Vec16<T>::N;
    int nvec;
    unsigned magic;
    if (!v16_magic(g.Nx, g.Ny, V, &nvec, &magic)) return cudaErrorInvalidValue;
    Fields<T> f;
    for (int c = 0; c < 6; c++) f.c[c] = fields[c];
    const long long per_plane = (long long)g.Ny * nvec;
    dim3 grid((unsigned)((per_plane + V16_BLOCK - 1) / V16_BLOCK), g.Nz);
    k_update_H_v16<T><<<grid, V16_BLOCK, 0, st>>>(g, f, src, step_base, off, nvec, magic);
    k_update_E_v16<T><<<grid, V16_BLOCK, 0, st>>>(g, f, src, step_base, off, nvec, magic);
    return cudaGetLastError();
}

template cudaError_t launch_step_v16<float>(const GridView<float>&, float* const*,
                                            const SourceList<float>&, const long long*, int,
                                            cudaStream_t);
template cudaError_t launch_step_v16<double>(const GridView<double>&, double* const*,
                                             const SourceList<double>&, const long long*, int,
                                             cudaStream_t);

}  // namespace fdtdb
