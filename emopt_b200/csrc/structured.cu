// structured.cu -- layered materials of rectangles evaluated on the GPU.
//
// The material model of the reference's StructuredMaterial3D
// (src/Grid.cpp:610-874) for Rectangle primitives (src/Grid.cpp:203-300):
// the z axis is cut into layers at the primitives' z1/z2; inside a layer the
// value of a Yee cell is the area-weighted average of StructuredMaterial2D
// (src/Grid.cpp:460-525); along z the value of a cell is the length-weighted
// average of the layers it spans, with 1.0 below, above and between them
// (src/Grid.cpp:737-826).
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
// The unclaimed region stays a union of disjoint rectangles (a difference of
// rectangles), at most kMaxPieces of them per cell.
//
// One thread per output element; all arithmetic in float64.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/emopt_fdtd.h"
#include "common.cuh"

namespace fdtdb {
namespace {

constexpr int kMaxPieces = 32;

struct Box2 {
    double x0, x1, y0, y1;   // xmin, xmax, ymin, ymax
};

struct LayerTables {
    const double* zs;        // nz layer boundaries, ascending
    int nz;
    const int* start;        // primitives of layer l: prims[start[l] .. start[l+1])
    const int* prims;
    const double* rects;     // per primitive: xmin, xmax, ymin, ymax, re, im
};

__device__ __forceinline__ bool inside(const double* r, double x, double y) {
    return x > r[0] && x < r[1] && y > r[2] && y < r[3];
}

__device__ __forceinline__ double box_area(const Box2& b) { return (b.x1 - b.x0) * (b.y1 - b.y0); }

// Value of layer l at the cell centred on (xd, yd) (src/Grid.cpp:460-525).
__device__ void layer_value(const LayerTables& t, int l, double xd, double yd, double dx, double dy,
                            double& vr, double& vi, int* err) {
    const double xmin = xd - dx / 2.0, xmax = xd + dx / 2.0;
    const double ymin = yd - dy / 2.0, ymax = yd + dy / 2.0;
    Box2 pieces[kMaxPieces];
    int n = 1;
    pieces[0] = Box2{xmin, xmax, ymin, ymax};
    const double max_area = fabs(box_area(pieces[0]));
    double area = max_area;
    vr = 0.0;
    vi = 0.0;
    // a layer without primitives (a gap between z ranges) is 0, not 1.0: the
    // reference reports an empty primitive list and returns 0
    if (t.start[l] == t.start[l + 1]) return;
    for (int q = t.start[l]; q < t.start[l + 1]; q++) {
        const double* r = t.rects + 6 * t.prims[q];
        const bool c1 = inside(r, xmin, ymin), c2 = inside(r, xmax, ymin);
        const bool c3 = inside(r, xmax, ymax), c4 = inside(r, xmin, ymax);
        if (c1 && c2 && c3 && c4 && area / max_area == 1.0) {
            vr = r[4];
            vi = r[5];
            return;
        }
        if (c1 || c2 || c3 || c4) {
            // unclaimed region minus the rectangle
            Box2 next[kMaxPieces];
            int m = 0;
            bool overflow = false;
            for (int p = 0; p < n; p++) {
                const Box2 b = pieces[p];
                if (r[1] <= b.x0 || r[0] >= b.x1 || r[3] <= b.y0 || r[2] >= b.y1) {
                    if (m < kMaxPieces) next[m++] = b; else overflow = true;
                    continue;
                }
                const double cx0 = fmax(b.x0, r[0]), cx1 = fmin(b.x1, r[1]);
                Box2 part[4];
                int k = 0;
                if (r[0] > b.x0) part[k++] = Box2{b.x0, cx0, b.y0, b.y1};
                if (r[1] < b.x1) part[k++] = Box2{cx1, b.x1, b.y0, b.y1};
                if (r[2] > b.y0) part[k++] = Box2{cx0, cx1, b.y0, fmax(b.y0, r[2])};
                if (r[3] < b.y1) part[k++] = Box2{cx0, cx1, fmin(b.y1, r[3]), b.y1};
                for (int e = 0; e < k; e++) {
                    if (m < kMaxPieces) next[m++] = part[e]; else overflow = true;
                }
            }
            if (overflow) atomicOr(err, 1);
            double new_area = 0.0;
            for (int p = 0; p < m; p++) {
                pieces[p] = next[p];
                new_area += fabs(box_area(next[p]));
            }
            n = m;
            const double overlap = (area - new_area) / max_area;
            vr += overlap * r[4];
            vi += overlap * r[5];
            area = new_area;
        }
        if (area / max_area == 0.0) break;
    }
    if (area / max_area > 0.0) vr += area / max_area * 1.0;
}

// Value at fractional indices (x, y, z) (src/Grid.cpp:737-826).
__device__ void material_value(const LayerTables& t, double x, double y, double z, double dx,
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

__global__ void __launch_bounds__(256) k_structured(LayerTables t, double dx, double dy, double dz,
                                                    int k1, int Nx, int j1, int Ny, int i1, long long n,
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
                                      const double* rects, int nrects, double dx, double dy,
                                      double dz, int k1, int k2, int j1, int j2, int i1, int i2,
                                      double sx, double sy, double sz, fdtd_complex128* out,
                                      char* msg, int msglen) {
    auto fail = [&](int code, const char* what) {
        if (msg && msglen > 0) snprintf(msg, (size_t)msglen, "FDTD_structured_values: %s", what);
        return code;
    };
    if (nzs < 0 || nrects < 0 || (nzs > 0 && (!zs || !layer_start)) || (nrects > 0 && !rects) || !out ||
        k2 < k1 || j2 < j1 || i2 < i1 || dx <= 0 || dy <= 0 || dz <= 0)
        return fail(FDTD_ERR_ARG, "bad arguments");
    const int nlayers = nzs > 1 ? nzs - 1 : 0;
    const int nref = nlayers > 0 ? layer_start[nlayers] : 0;
    if (nref < 0 || (nref > 0 && !layer_prims)) return fail(FDTD_ERR_ARG, "bad layer table");
    for (int l = 0; l < nlayers; l++)
        if (layer_start[l] > layer_start[l + 1] || layer_start[l] < 0) return fail(FDTD_ERR_ARG, "bad layer table");
    for (int q = 0; q < nref; q++)
        if (layer_prims[q] < 0 || layer_prims[q] >= nrects) return fail(FDTD_ERR_ARG, "primitive index out of range");
    for (int l = 0; l + 1 < nzs; l++)
        if (!(zs[l] <= zs[l + 1])) return fail(FDTD_ERR_ARG, "layer boundaries must ascend");
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
    // tables: zs | start | prims | rects | err, one device block
    const size_t bz = sizeof(double) * (size_t)(nzs > 0 ? nzs : 1);
    const size_t bs = sizeof(int) * (size_t)(nlayers + 1);
    const size_t bp = sizeof(int) * (size_t)(nref > 0 ? nref : 1);
    const size_t br = sizeof(double) * 6 * (size_t)(nrects > 0 ? nrects : 1);
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t total = up(bz) + up(bs) + up(bp) + up(br) + 256;
    unsigned char* d = nullptr;
    fdtdb::c128* dout = nullptr;
    cudaPointerAttributes pa;
    bool out_dev = false;
    if (e == cudaSuccess) {
        e = cudaPointerGetAttributes(&pa, out);
        if (e == cudaSuccess) out_dev = pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged;
        else { cudaGetLastError(); e = cudaSuccess; }
    }
    if (e == cudaSuccess) e = cudaMalloc(&d, total);
    if (e == cudaSuccess && !out_dev) e = cudaMalloc(&dout, sizeof(fdtdb::c128) * (size_t)n);
    unsigned char* pz = d;
    unsigned char* ps = pz + up(bz);
    unsigned char* pp = ps + up(bs);
    unsigned char* pr = pp + up(bp);
    int* perr = reinterpret_cast<int*>(pr + up(br));
    if (e == cudaSuccess && nzs > 0) e = cudaMemcpyAsync(pz, zs, sizeof(double) * nzs, cudaMemcpyDefault, st);
    if (e == cudaSuccess && nlayers > 0) e = cudaMemcpyAsync(ps, layer_start, bs, cudaMemcpyDefault, st);
    if (e == cudaSuccess && nref > 0) e = cudaMemcpyAsync(pp, layer_prims, sizeof(int) * nref, cudaMemcpyDefault, st);
    if (e == cudaSuccess && nrects > 0) e = cudaMemcpyAsync(pr, rects, sizeof(double) * 6 * nrects, cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(perr, 0, sizeof(int), st);
    int herr = 0;
    if (e == cudaSuccess) {
        fdtdb::LayerTables t;
        t.zs = reinterpret_cast<const double*>(pz);
        t.nz = nzs;
        t.start = reinterpret_cast<const int*>(ps);
        t.prims = reinterpret_cast<const int*>(pp);
        t.rects = reinterpret_cast<const double*>(pr);
        fdtdb::c128* o = out_dev ? reinterpret_cast<fdtdb::c128*>(out) : dout;
        const unsigned grid = (unsigned)((n + 255) / 256);
        fdtdb::k_structured<<<grid, 256, 0, st>>>(t, dx, dy, dz, k1, (int)Nx, j1, (int)Ny, i1, n, sx,
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
    if (herr) return fail(FDTD_ERR_ARG, "more than 32 unclaimed pieces in one cell");
    return FDTD_OK;
}
