// structured.cu -- layered materials of rectangles and polygons on the GPU.
//
// The material model of the reference's StructuredMaterial3D
// (src/Grid.cpp:610-874) with Rectangle (src/Grid.cpp:203-300), Polygon
// (src/Grid.cpp:300-395) and Circle (src/Grid.cpp:141-201) primitives: the z
// axis is cut into layers at the
// primitives' z1/z2; inside a layer the value of a Yee cell is the
// area-weighted average of StructuredMaterial2D (src/Grid.cpp:460-525); along
// z the value of a cell is the length-weighted average of the layers it spans,
// with 1.0 below, above and between them (src/Grid.cpp:737-826).
//
// Area weighting in a layer, per cell (xd, yd) = (x dx, y dy), cell
// [xd - dx/2, xd + dx/2] x [yd - dy/2, yd + dy/2], primitives in priority
// order (lower layer number first):
//   * a primitive with all four cell corners strictly inside while nothing of
//     the cell has been claimed yet gives the cell its material outright;
//   * a primitive with at least one corner strictly inside claims the part of
//     the still-unclaimed region it covers, weighted by that area over the
//     cell area; a primitive with no corner inside is skipped even if it cuts
//     the cell (the reference's test, kept);
//   * the walk stops once nothing is unclaimed; what is left takes 1.0;
//   * a layer with no primitive at all (a gap between z ranges) is 0.
// A primitive arrives as convex parts (a rectangle or convex polygon as
// itself, any other simple polygon as the triangles of an ear-clipping
// triangulation, made on the host) plus its outline for the corner test.  The
// unclaimed region is kept as at most kMaxPieces convex pieces of at most
// kMaxVerts vertices: removing a convex part from a convex piece leaves the
// pieces cut off by each of the part's edges in turn (disjoint, convex), and
// what remains after the last edge is the claimed piece.  Pieces smaller than
// 1e-14 of the cell area are dropped.  Overflow of either limit is reported.
//
// One thread per output element; all arithmetic in float64.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/emopt_fdtd.h"
#include "common.cuh"

namespace fdtdb {
namespace {

constexpr int kMaxPieces = 16;
constexpr int kMaxVerts = 12;

struct Poly {
    int n;
    double x[kMaxVerts], y[kMaxVerts];
};

struct Tables {
    const double* zs;        // nz layer boundaries, ascending
    int nz;
    const int* start;        // primitives of layer l: prims[start[l] .. start[l+1])
    const int* prims;
    const int* pinfo;        // per primitive: outline start, outline count, part start, part count
    const double* pval;      // per primitive: Re, Im, xmin, xmax, ymin, ymax (bounding box)
    const int* parts;        // per convex part: vertex start, vertex count (counter-clockwise)
    const double* verts;     // x, y of outline and part vertices
};

__device__ __forceinline__ double poly_area(const Poly& p) {
    double a = 0.0;
    for (int q = 0; q < p.n; q++) {
        const int r = q + 1 == p.n ? 0 : q + 1;
        a += p.x[q] * p.y[r] - p.x[r] * p.y[q];
    }
    return fabs(a) * 0.5;
}

// Part of `in` on the left of the directed edge a -> b (keep_left) or on the
// right; false on vertex overflow.
__device__ bool clip_half(const Poly& in, double ax, double ay, double bx, double by, bool keep_left,
                          Poly& out) {
    out.n = 0;
    const double ex = bx - ax, ey = by - ay;
    for (int q = 0; q < in.n; q++) {
        const int r = q + 1 == in.n ? 0 : q + 1;
        double sp = ex * (in.y[q] - ay) - ey * (in.x[q] - ax);
        double sq = ex * (in.y[r] - ay) - ey * (in.x[r] - ax);
        if (!keep_left) { sp = -sp; sq = -sq; }
        if (sp >= 0.0) {
            if (out.n == kMaxVerts) return false;
            out.x[out.n] = in.x[q];
            out.y[out.n] = in.y[q];
            out.n++;
        }
        if ((sp > 0.0 && sq < 0.0) || (sp < 0.0 && sq > 0.0)) {
            if (out.n == kMaxVerts) return false;
            const double t = sp / (sp - sq);
            out.x[out.n] = in.x[q] + (in.x[r] - in.x[q]) * t;
            out.y[out.n] = in.y[q] + (in.y[r] - in.y[q]) * t;
            out.n++;
        }
    }
    if (out.n < 3) out.n = 0;
    return true;
}

// Strictly inside the outline (a point on an edge is not; src/Grid.cpp:362-381).
__device__ bool outline_contains(const Tables& t, int pr, double px, double py) {
    const double* v = t.pval + 6 * pr;
    if (!(px > v[2] && px < v[3] && py > v[4] && py < v[5])) return false;
    const int s = t.pinfo[4 * pr], n = t.pinfo[4 * pr + 1];
    bool in = false;
    for (int q = 0; q < n; q++) {
        const int r = q + 1 == n ? 0 : q + 1;
        const double ax = t.verts[2 * (s + q)], ay = t.verts[2 * (s + q) + 1];
        const double bx = t.verts[2 * (s + r)], by = t.verts[2 * (s + r) + 1];
        const double cross = (bx - ax) * (py - ay) - (by - ay) * (px - ax);
        if (cross == 0.0 && px >= fmin(ax, bx) && px <= fmax(ax, bx) && py >= fmin(ay, by) &&
            py <= fmax(ay, by))
            return false;
        if ((ay > py) != (by > py) && px < (bx - ax) * (py - ay) / (by - ay) + ax) in = !in;
    }
    return in;
}

// A circle (outline count -1): centre and radius in its two outline vertex
// slots.  Strictly inside when dx^2 + dy^2 < r^2 (src/Grid.cpp:144-149).
__device__ __forceinline__ bool circle_contains(const Tables& t, int pr, double px, double py) {
    const int s = t.pinfo[4 * pr];
    const double dx = px - t.verts[2 * s], dy = py - t.verts[2 * s + 1], r = t.verts[2 * s + 2];
    return dx * dx + dy * dy < r * r;
}

__device__ __forceinline__ bool prim_contains(const Tables& t, int pr, double px, double py) {
    return t.pinfo[4 * pr + 1] < 0 ? circle_contains(t, pr, px, py) : outline_contains(t, pr, px, py);
}

// Value of layer l at the cell centred on (xd, yd) (src/Grid.cpp:460-525).
// A circle gives its value to a cell it holds entirely while nothing of the
// cell is claimed, and otherwise claims nothing: the reference's circle cell
// overlap is 0 (src/Grid.cpp:167-171).
__device__ void layer_value(const Tables& t, int l, double xd, double yd, double dx, double dy,
                            double& vr, double& vi, int* err) {
    vr = 0.0;
    vi = 0.0;
    // a layer without primitives (a gap between z ranges) is 0, not 1.0: the
    // reference reports an empty primitive list and returns 0
    if (t.start[l] == t.start[l + 1]) return;
    const double xmin = xd - dx / 2.0, xmax = xd + dx / 2.0;
    const double ymin = yd - dy / 2.0, ymax = yd + dy / 2.0;
    Poly pieces[kMaxPieces], next[kMaxPieces];
    int n = 1;
    pieces[0].n = 4;
    pieces[0].x[0] = xmin; pieces[0].y[0] = ymin;
    pieces[0].x[1] = xmax; pieces[0].y[1] = ymin;
    pieces[0].x[2] = xmax; pieces[0].y[2] = ymax;
    pieces[0].x[3] = xmin; pieces[0].y[3] = ymax;
    const double max_area = poly_area(pieces[0]);
    const double tiny = 1e-14 * max_area;
    double area = max_area;
    bool ok = true;
    for (int q = t.start[l]; q < t.start[l + 1]; q++) {
        const int pr = t.prims[q];
        const double* v = t.pval + 6 * pr;
        const bool c1 = prim_contains(t, pr, xmin, ymin), c2 = prim_contains(t, pr, xmax, ymin);
        const bool c3 = prim_contains(t, pr, xmax, ymax), c4 = prim_contains(t, pr, xmin, ymax);
        if (c1 && c2 && c3 && c4 && area / max_area == 1.0) {
            vr = v[0];
            vi = v[1];
            return;
        }
        if ((c1 || c2 || c3 || c4) && t.pinfo[4 * pr + 1] < 0) {
            // circle: overlap 0, nothing claimed
            vr += 0.0 * v[0];
            vi += 0.0 * v[1];
        } else if (c1 || c2 || c3 || c4) {
            // the unclaimed pieces minus every convex part of the primitive
            const int p0 = t.pinfo[4 * pr + 2], pn = t.pinfo[4 * pr + 3];
            for (int part = p0; part < p0 + pn; part++) {
                const int vs = t.parts[2 * part], vn = t.parts[2 * part + 1];
                int m = 0;
                for (int k = 0; k < n; k++) {
                    Poly cur = pieces[k], cut, inner;
                    for (int e = 0; e < vn && cur.n > 0; e++) {
                        const int f = e + 1 == vn ? 0 : e + 1;
                        const double ax = t.verts[2 * (vs + e)], ay = t.verts[2 * (vs + e) + 1];
                        const double bx = t.verts[2 * (vs + f)], by = t.verts[2 * (vs + f) + 1];
                        ok &= clip_half(cur, ax, ay, bx, by, false, cut);
                        if (cut.n > 0 && poly_area(cut) > tiny) {
                            if (m < kMaxPieces) next[m++] = cut;
                            else ok = false;
                        }
                        ok &= clip_half(cur, ax, ay, bx, by, true, inner);
                        cur = inner;
                    }
                }
                n = m;
                for (int k = 0; k < n; k++) pieces[k] = next[k];
            }
            double new_area = 0.0;
            for (int k = 0; k < n; k++) new_area += poly_area(pieces[k]);
            const double overlap = (area - new_area) / max_area;
            vr += overlap * v[0];
            vi += overlap * v[1];
            area = new_area;
        }
        if (area / max_area == 0.0) break;
    }
    if (!ok) atomicOr(err, 1);
    if (area / max_area > 0.0) vr += area / max_area * 1.0;
}

// Value at fractional indices (x, y, z) (src/Grid.cpp:737-826).
__device__ void material_value(const Tables& t, double x, double y, double z, double dx,
                               double dy, double dz, double& vr, double& vi, int* err) {
    vr = 0.0;
    vi = 0.0;
    if (t.nz < 2) {
        vr = 1.0;
        return;
    }
    double zmin = (z - 0.5) * dz, zmax = (z + 0.5) * dz;
    const double xd = x * dx, yd = y * dy;
    if (zmax <= t.zs[0]) {
        vr = 1.0;
        return;
    }
    if (zmax > t.zs[0] && zmin < t.zs[0]) {
        vr = (t.zs[0] - zmin) / dz * 1.0;
        zmin = t.zs[0];
    }
    for (int l = 0; l + 1 < t.nz; l++) {
        const double za = t.zs[l], zb = t.zs[l + 1];
        if (zmin >= za && zmax <= zb) {
            double lr, li;
            layer_value(t, l, xd, yd, dx, dy, lr, li, err);
            vr += (zmax - zmin) / dz * lr;
            vi += (zmax - zmin) / dz * li;
            return;
        } else if (zmin >= za && zmin < zb && zmax > zb) {
            double lr, li;
            layer_value(t, l, xd, yd, dx, dy, lr, li, err);
            vr += (zb - zmin) / dz * lr;
            vi += (zb - zmin) / dz * li;
            zmin = zb;
        }
    }
    vr += (zmax - zmin) / dz * 1.0;
}

__global__ void __launch_bounds__(128) k_structured(Tables t, double dx, double dy, double dz, int k1,
                                                    int Nx, int j1, int Ny, int i1, long long n,
                                                    double sx, double sy, double sz, c128* out,
                                                    int* err) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const long long row = q / Nx;
    const int k = k1 + (int)(q - row * Nx);
    const int j = j1 + (int)(row % Ny);
    const int i = i1 + (int)(row / Ny);
    double vr, vi;
    material_value(t, k + sx, j + sy, i + sz, dx, dy, dz, vr, vi, err);
    out[q].real = vr;
    out[q].imag = vi;
}

}  // namespace
}  // namespace fdtdb

extern "C" int FDTD_structured_values(int device, void* stream, const double* zs, int nzs,
                                      const int* layer_start, const int* layer_prims,
                                      const int* prim_info, const double* prim_vals, int nprims,
                                      const int* parts, int nparts, const double* verts, int nverts,
                                      double dx, double dy, double dz, int k1, int k2, int j1,
                                      int j2, int i1, int i2, double sx, double sy, double sz,
                                      fdtd_complex128* out, char* msg, int msglen) {
    auto fail = [&](int code, const char* what) {
        if (msg && msglen > 0) snprintf(msg, (size_t)msglen, "FDTD_structured_values: %s", what);
        return code;
    };
    if (nzs < 0 || nprims < 0 || nparts < 0 || nverts < 0 || (nzs > 0 && (!zs || !layer_start)) ||
        (nprims > 0 && (!prim_info || !prim_vals)) || (nparts > 0 && !parts) ||
        (nverts > 0 && !verts) || !out || k2 < k1 || j2 < j1 || i2 < i1 || dx <= 0 || dy <= 0 || dz <= 0)
        return fail(FDTD_ERR_ARG, "bad arguments");
    const int nlayers = nzs > 1 ? nzs - 1 : 0;
    const int nref = nlayers > 0 ? layer_start[nlayers] : 0;
    if (nref < 0 || (nref > 0 && !layer_prims)) return fail(FDTD_ERR_ARG, "bad layer table");
    for (int l = 0; l < nlayers; l++)
        if (layer_start[l] > layer_start[l + 1] || layer_start[l] < 0) return fail(FDTD_ERR_ARG, "bad layer table");
    for (int q = 0; q < nref; q++)
        if (layer_prims[q] < 0 || layer_prims[q] >= nprims) return fail(FDTD_ERR_ARG, "primitive index out of range");
    for (int l = 0; l + 1 < nzs; l++)
        if (!(zs[l] <= zs[l + 1])) return fail(FDTD_ERR_ARG, "layer boundaries must ascend");
    for (int q = 0; q < nprims; q++) {
        const int* pi = prim_info + 4 * q;
        // a circle: outline count -1, centre and radius in two vertex slots, no parts
        const bool circle = pi[1] == -1;
        const int nv = circle ? 2 : pi[1];
        if (pi[0] < 0 || (!circle && nv < 3) || pi[0] + nv > nverts || pi[2] < 0 ||
            (circle ? pi[3] != 0 : pi[3] < 1) || pi[2] + pi[3] > nparts)
            return fail(FDTD_ERR_ARG, "bad primitive table");
        if (circle && !(verts[2 * pi[0] + 2] >= 0.0)) return fail(FDTD_ERR_ARG, "bad circle radius");
    }
    for (int q = 0; q < nparts; q++)
        if (parts[2 * q] < 0 || parts[2 * q + 1] < 3 || parts[2 * q] + parts[2 * q + 1] > nverts)
            return fail(FDTD_ERR_ARG, "bad part table");
    const long long Nx = k2 - k1, Ny = j2 - j1, Nz = i2 - i1, n = Nx * Ny * Nz;
    if (n == 0) return FDTD_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(FDTD_ERR_NODEVICE, "no CUDA device is visible");
    }
    if (device < 0 || device >= ndev) return fail(FDTD_ERR_ARG, "device out of range");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaSetDevice(device);
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t bz = sizeof(double) * (size_t)(nzs > 0 ? nzs : 1);
    const size_t bs = sizeof(int) * (size_t)(nlayers + 1);
    const size_t bp = sizeof(int) * (size_t)(nref > 0 ? nref : 1);
    const size_t bi = sizeof(int) * 4 * (size_t)(nprims > 0 ? nprims : 1);
    const size_t bv = sizeof(double) * 6 * (size_t)(nprims > 0 ? nprims : 1);
    const size_t bq = sizeof(int) * 2 * (size_t)(nparts > 0 ? nparts : 1);
    const size_t bx = sizeof(double) * 2 * (size_t)(nverts > 0 ? nverts : 1);
    const size_t total = up(bz) + up(bs) + up(bp) + up(bi) + up(bv) + up(bq) + up(bx) + 256;
    unsigned char* d = nullptr;
    fdtdb::c128* dout = nullptr;
    bool out_dev = false;
    if (e == cudaSuccess) {
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, out) == cudaSuccess)
            out_dev = pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged;
        else
            cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMalloc(&d, total);
    if (e == cudaSuccess && !out_dev) e = cudaMalloc(&dout, sizeof(fdtdb::c128) * (size_t)n);
    unsigned char* pz = d;
    unsigned char* ps = pz + up(bz);
    unsigned char* pp = ps + up(bs);
    unsigned char* pi = pp + up(bp);
    unsigned char* pv = pi + up(bi);
    unsigned char* pq = pv + up(bv);
    unsigned char* px = pq + up(bq);
    int* perr = reinterpret_cast<int*>(px + up(bx));
    auto put = [&](void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes > 0 && src) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st);
    };
    put(pz, zs, sizeof(double) * (size_t)nzs);
    if (nlayers > 0) put(ps, layer_start, bs);
    put(pp, layer_prims, sizeof(int) * (size_t)nref);
    put(pi, prim_info, sizeof(int) * 4 * (size_t)nprims);
    put(pv, prim_vals, sizeof(double) * 6 * (size_t)nprims);
    put(pq, parts, sizeof(int) * 2 * (size_t)nparts);
    put(px, verts, sizeof(double) * 2 * (size_t)nverts);
    if (e == cudaSuccess) e = cudaMemsetAsync(perr, 0, sizeof(int), st);
    int herr = 0;
    if (e == cudaSuccess) {
        fdtdb::Tables t;
        t.zs = reinterpret_cast<const double*>(pz);
        t.nz = nzs;
        t.start = reinterpret_cast<const int*>(ps);
        t.prims = reinterpret_cast<const int*>(pp);
        t.pinfo = reinterpret_cast<const int*>(pi);
        t.pval = reinterpret_cast<const double*>(pv);
        t.parts = reinterpret_cast<const int*>(pq);
        t.verts = reinterpret_cast<const double*>(px);
        fdtdb::c128* o = out_dev ? reinterpret_cast<fdtdb::c128*>(out) : dout;
        const unsigned grid = (unsigned)((n + 127) / 128);
        fdtdb::k_structured<<<grid, 128, 0, st>>>(t, dx, dy, dz, k1, (int)Nx, j1, (int)Ny, i1, n, sx,
                                                  sy, sz, o, perr);
        e = cudaGetLastError();
        if (e == cudaSuccess && !out_dev)
            e = cudaMemcpyAsync(out, dout, sizeof(fdtdb::c128) * (size_t)n, cudaMemcpyDefault, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, perr, sizeof(int), cudaMemcpyDefault, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (d) cudaFree(d);
    if (dout) cudaFree(dout);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
    }
    if (herr) return fail(FDTD_ERR_ARG, "a cell needs more than 16 unclaimed pieces or 12 vertices per piece");
    return FDTD_OK;
}
