// grid.cuh -- device-resident layout of one CW-FDTD solve.
//
// Field components are stored as dense [Nz][Ny][px] arrays (x fastest) with
// the row pitch px rounded up to a multiple of 32 elements, so every row
// starts on a 128-byte boundary (fp32) / 256-byte boundary (fp64).  There are
// no ghost cells: the boundary conditions that the reference materialises in
// its ghost layer (src/fdtd.cpp:141-173 and 397-501) are applied as
// predicates on the neighbour index.
//
// CPML state lives in one array group per axis that covers both the min and
// the max slab of that axis ("local" slab index l in [0, w0 + w1)):
//     x: slot = (i*Ny + j)*wx + l          y: slot = (i*wy + l)*px + k
//     z: slot = (l*Ny + j)*px + k
// Slots 0,1 of an axis hold the E-derivative accumulators used by the H
// update, slots 2,3 the H-derivative accumulators used by the E update (the
// same pairing as src/fdtd.cpp:223-305 and 583-665).
#pragma once

#include "common.cuh"

namespace fdtdb {

constexpr int kMaxSources = 16;

// One current source box; comp[c] points at interleaved (a_c, a_s) pairs for
// component c in (Jx, Jy, Jz, Mx, My, Mz), already multiplied by the update
// coefficient of the cell, or is null when that component is zero everywhere.
template <typename T>
struct DevSource {
    int i0, j0, k0, I, J, K;
    const T* comp[6];
};

template <typename T>
struct SourceList {
    int n;
    // bounding boxes of the sources that drive E (0: a J component is
    // non-zero) and H (1: an M component), as i0, i1, j0, j1, k0, k1 (half
    // open); empty (i0 >= i1) when no source drives that half step
    int box[2][6];
    DevSource<T> s[kMaxSources];
};

// Per-axis CPML tables indexed by the local slab index.
template <typename T>
struct PmlAxis {
    int w0, w1, wsum;      // min width, max width, total
    int edge_max;          // first index of the max slab (strict > for z)
    int off;               // global index of local coordinate 0 (z slab of a
                           // distributed solve; 0 otherwise)
    T* psi[4];
    const T* kinvH;        // 1/kappa, b, c for the H update
    const T* bH;
    const T* cH;
    const T* kinvE;        // 1/kappa, b, c for the E update
    const T* bE;
    const T* cE;
};

template <typename T>
struct GridView {
    int Nx, Ny, Nz, px;
    long long plane;               // Ny * px
    T odx, ody, odz;
    const T* bE[3];                // E update: b = dt/eps (or the lossy form)
    const T* aE[3];                // lossy E update: a (null when lossless)
    const T* bHarr[3];             // H update: dt/mu per cell (null when uniform)
    T bH[3];                       // uniform dt/mu
    char bc[3];
    // a neighbouring z slab holds the plane below local index 0 (zlo) or above
    // Nz - 1 (zhi): the field arrays then have a halo plane there, filled by
    // the exchange, which is read instead of applying the boundary rule
    char zlo, zhi;
    // where those neighbour planes are read (zlo / zhi set): Ex, Ey of the
    // plane above (zhalo[0], [1]) and Hx, Hy of the plane below ([2], [3]),
    // each Ny x px with the rows of a plane -- the slab's own halo planes, or
    // the neighbouring slab's boundary planes when it lives on this device
    const T* zhalo[4];
    int* chk;                      // builds with FDTD_BOUNDS_CHECK: first failed index check (else unused)
    PmlAxis<T> pml[3];
    const double4* step_tab;       // per step: (S_H, C_H, S_E, C_E)
};

// Loop state of one request in the batched stepping (serve_kernels.cu).
enum ServeState { SERVE_FREE = 0, SERVE_RUN = 1, SERVE_TAIL = 2, SERVE_EXTRACT = 3, SERVE_DONE = 4 };

// What a half step of one served request reads besides its grid: the
// request's loop state and capture flag (device memory, written by the
// events kernel between steps) and its two snapshot sets.  The half step
// stores only while the state is RUN, TAIL or EXTRACT; with capture = 1 or 2
// the H half step also writes the six fields it read (the state after the
// previous step) into snap[capture - 1].
template <typename T>
struct ServeGate {
    const int* state;
    const int* capture;
    T* snap[2][6];
};

__device__ __forceinline__ bool serve_running(int state) {
    return state == SERVE_RUN || state == SERVE_TAIL || state == SERVE_EXTRACT;
}

// Local CPML slab index of coordinate c on axis a, or -1.
template <typename T>
__device__ __forceinline__ int slab_local(const PmlAxis<T>& P, int c, bool strict_max) {
    if (c < P.w0) return c;
    if (strict_max ? (c > P.edge_max) : (c >= P.edge_max)) return P.w0 + (c - P.edge_max);
    return -1;
}

}  // namespace fdtdb
