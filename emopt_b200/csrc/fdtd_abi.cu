// fdtd_abi.cu -- the exported C ABI (include/emopt_fdtd.h).
//
// FDTDHandle mirrors the state of the reference class fdtd::FDTD
// (src/fdtd.hpp:163-229): parameters set through the setters, caller-owned
// arrays retained by pointer, the CPML coefficient tables and the source list.
// Every computation runs on the GPU:
//   * the per-call reference entry points (update_H/E, capture, extraction,
//     add_source's amplitude/phase conversion) copy the caller's arrays to
//     device mirrors, run the padded-layout kernels of legacy_kernels.cu and
//     copy the results back, so a caller that drives the loop itself sees
//     exactly the reference's array semantics;
//   * FDTD_solve_cw keeps everything resident and runs the whole time loop.
// The scalar fit functions (FDTD_calc_phase_3T, ...) and FDTD_src_func_t are
// pure functions of their arguments; they evaluate the same __host__ __device__
// code as the kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/emopt_fdtd.h"
#include "kernels.h"

using fdtdb::c128;

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool owned = true;      // false: a view into another DevBuf (never freed here)
    cudaError_t ensure(size_t n) {
        if (n == 0) n = 16;
        if (p && bytes >= n) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) { p = nullptr; return e; }
        bytes = n;
        owned = true;
        return cudaSuccess;
    }
    void release() {
        if (p && owned) cudaFree(p);
        p = nullptr;
        bytes = 0;
        owned = true;
    }
};

template <typename T>
T* dptr(const DevBuf& b) { return reinterpret_cast<T*>(b.p); }

struct HostSource {
    c128* comp[6];
    int i0, j0, k0, I, J, K;
};

// Device state of the resident solve for one precision.
template <typename T>
struct Resident {
    int Nx = 0, Ny = 0, Nz = 0, px = 0;
    DevBuf F[2][6];          // fields Ex Ey Ez Hx Hy Hz; set 1: the fused step's second set
    DevBuf bE[3], aE[3], bH[3];
    bool mu_uniform[3] = {true, true, true};
    double mu_value[3] = {1, 1, 1};
    bool lossy = false;
    bool coeffs_valid = false;
    DevBuf psi[2][3][4];     // CPML accumulators per set and axis
    DevBuf tab[3][6];
    DevBuf snap[2][6];
    DevBuf stage;            // complex128 staging (one component)
    std::vector<DevBuf> src_ap;    // per source: 6 comps of amp/phase (complex128)
    std::vector<DevBuf> src_coef;  // per source: 6 comps of (a_c, a_s)
    DevBuf steptab, stepbase, flag, err;
    DevBuf pwin, pA, pphi, ptimes, pout, pmap;
    int halo = 0;            // planes of halo below and above the fields (z slabs)
    DevBuf psamp;            // z slab: probe samples of all slabs [3][npoints]

    void release_all() {
        for (auto& s : F) for (auto& b : s) b.release();
        for (int c = 0; c < 3; c++) { bE[c].release(); aE[c].release(); bH[c].release(); }
        for (auto& s : psi) for (auto& a : s) for (auto& b : a) b.release();
        for (auto& a : tab) for (auto& b : a) b.release();
        for (auto& s : snap) for (auto& b : s) b.release();
        stage.release();
        for (auto& b : src_ap) b.release();
        for (auto& b : src_coef) b.release();
        src_ap.clear(); src_coef.clear();
        steptab.release(); stepbase.release(); flag.release(); err.release();
        pwin.release(); pA.release(); pphi.release(); ptimes.release(); pout.release(); pmap.release();
        psamp.release();
        coeffs_valid = false;
        Nx = Ny = Nz = px = 0;
        halo = 0;
    }
};

}  // namespace

struct FDTDHandle {
    // ---- reference parameters (src/fdtd.hpp:163-229)
    int Nx = 0, Ny = 0, Nz = 0;
    int I = 0, J = 0, K = 0, i0 = 0, j0 = 0, k0 = 0;
    double X = 0, Y = 0, Z = 0, dx = 1, dy = 1, dz = 1;
    double wavelength = 1, R = 1, dt = 1, odt = 1;
    double src_T = 0, src_min = 1e-4, src_k = 1;
    bool lossy = false;
    double* hE[3] = {nullptr, nullptr, nullptr};
    double* hH[3] = {nullptr, nullptr, nullptr};
    c128* heps[3] = {nullptr, nullptr, nullptr};
    c128* hmu[3] = {nullptr, nullptr, nullptr};
    c128* ht0[6] = {nullptr};
    c128* ht1[6] = {nullptr};
    int w[6] = {0, 0, 0, 0, 0, 0};
    double sigma = 0, alpha = 0, kappa = 1, pw = 1;
    char bc[3] = {'0', '0', '0'};
    std::vector<double> tab[3][6];   // kappa_H b_H c_H kappa_E b_E c_E, reference order
    std::vector<HostSource> sources;

    // ---- runtime
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double* pinned = nullptr;        // small pinned staging (probe results)
    int status = FDTD_OK;
    std::string message;
    int precision = 64;
    int kernel = 0;
    int zchunk = 0;   // planes per CTA of the fused kernels (0: automatic)
    bool ext_stream = false;   // the stream belongs to the caller (FDTD_set_stream)

    // ---- z slab of a distributed solve (FDTD_slab_*): the handle's grid is
    // the slab, planes [slab_i0, slab_i0 + Nz) of a grid of slab_Nz planes
    int slab = 0;
    int slab_i0 = 0, slab_Nz = 0, slab_lo = 0, slab_hi = 0;
    int slab_np = 0;                 // probe points of all slabs
    const void* slab_zhalo[4] = {nullptr, nullptr, nullptr, nullptr};   // FDTD_slab_set_halo_source
    long long slab_Tn = 0;
    fdtdb::SourceList<float> slab_src32;
    fdtdb::SourceList<double> slab_src64;

    // ---- padded-layout device mirrors for the per-call entry points
    DevBuf lE[3], lH[3], leps[3], lmu[3];
    DevBuf lpsi[3][2][4];
    DevBuf ltab[3][6];
    std::vector<DevBuf> lsrc;        // 6 per source
    DevBuf lt0[6], lt1[6];
    bool ltab_dirty = true;

    Resident<float> r32;
    Resident<double> r64;

    int fail(int code, const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        status = code;
        message = buf;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        return fail(FDTD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
    // Records FDTD_ERR_NODEVICE when no GPU is visible.
    int probe_device() {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
            return fail(FDTD_ERR_NODEVICE, "no CUDA device is visible");
        return FDTD_OK;
    }
    // Selects the handle's device and creates its stream on first use.
    int ready() {
        if (device < 0) {
            if (probe_device() != FDTD_OK) return status;
            cudaGetDevice(&device);
        }
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
        if (!stream && !ext_stream) {
            if ((e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamCreate");
            for (auto& v : ev)
                if ((e = cudaEventCreate(&v)) != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
            if ((e = cudaMallocHost(&pinned, 64 * sizeof(double))) != cudaSuccess)
                return cuda_fail(e, "cudaMallocHost");
        }
        return FDTD_OK;
    }
    long long ncells() const { return (long long)I * J * K; }
    long long npad() const { return (long long)(I + 2) * (J + 2) * (K + 2); }
    bool whole_grid() const {
        return i0 == 0 && j0 == 0 && k0 == 0 && I == Nz && J == Ny && K == Nx;
    }

    void compute_tables();
    long long slab_cells(int a, int side) const;
    int sync_check(const char* what) {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, what);
        return FDTD_OK;
    }
};

#define CK(expr)                                                    \
    do {                                                            \
        cudaError_t e_ = (expr);                                    \
        if (e_ != cudaSuccess) return h->cuda_fail(e_, #expr);      \
    } while (0)

// ------------------------------------------------------------ CPML tables
// One coefficient triple for ramp value f (src/fdtd.cpp:992-997).
static void cpml_coeffs(const FDTDHandle* h, double f, double* kap, double* b, double* c) {
    double sigma = h->sigma * f;
    double alpha = h->alpha * (1 - f);
    double kappa = (h->kappa - 1.0) * f + 1.0;
    double bb = exp(-h->dt * (sigma / kappa + alpha));
    *kap = kappa;
    *b = bb;
    *c = (bb == 1) ? 0.0 : (bb - 1) * sigma / (sigma * kappa + kappa * kappa * alpha);
}

// Tables of src/fdtd.cpp:950-1181 with the reference's index order
// (min slab: entry q at depth q from the interior edge; max slab at w0 + q).
// Distance offsets: x/y min H (q-0.5)/w clamped at 0, E q/w; x/y max H
// (q+0.5)/w, E q/w; z min H q/w, E (q+0.5)/w; z max H q/w, E (q-0.5)/w clamped.
void FDTDHandle::compute_tables() {
    for (int a = 0; a < 3; a++) {
        int w0 = w[2 * a], w1 = w[2 * a + 1];
        for (int q = 0; q < 6; q++) tab[a][q].assign((size_t)(w0 + w1), 0.0);
        for (int side = 0; side < 2; side++) {
            int ww = side ? w1 : w0;
            for (int q = 0; q < ww; q++) {
                double dH, dE;
                bool clampH = false, clampE = false;
                if (a != 2) {
                    dH = side ? (double)(q + 0.5) / ww : (double)(q - 0.5) / ww;
                    clampH = !side;
                    dE = (double)q / ww;
                } else {
                    dH = (double)q / ww;
                    dE = side ? (double)(q - 0.5) / ww : (double)(q + 0.5) / ww;
                    clampE = side;
                }
                double fH = pow(dH, pw), fE = pow(dE, pw);
                if (clampH && fH < 0) fH = 0;
                if (clampE && fE < 0) fE = 0;
                int at = side ? w0 + q : q;
                cpml_coeffs(this, fH, &tab[a][0][at], &tab[a][1][at], &tab[a][2][at]);
                cpml_coeffs(this, fE, &tab[a][3][at], &tab[a][4][at], &tab[a][5][at]);
            }
        }
    }
    ltab_dirty = true;
    r32.coeffs_valid = false;   // tables feed the resident state too
    r64.coeffs_valid = false;
}

// The tables are sized by the widths at their last build; widths changed
// without a rebuild would index past them, so rebuild in that case.
static void ensure_tables(FDTDHandle* h) {
    for (int a = 0; a < 3; a++)
        if ((int)h->tab[a][0].size() != h->w[2 * a] + h->w[2 * a + 1]) {
            h->compute_tables();
            return;
        }
}

long long FDTDHandle::slab_cells(int a, int side) const {
    int lo[3] = {k0, j0, i0}, n[3] = {K, J, I}, N[3] = {Nx, Ny, Nz};
    int depth;
    if (!side) {
        if (!(lo[a] < w[2 * a])) return 0;
        depth = w[2 * a] - lo[a];
    } else {
        int edge = N[a] - w[2 * a + 1];
        if (!(lo[a] + n[a] > edge)) return 0;
        depth = lo[a] + n[a] - edge;
    }
    long long cells = depth;
    for (int b = 0; b < 3; b++)
        if (b != a) cells *= n[b];
    return cells;
}

// =================================================== reference ABI, setters
extern "C" {

FDTDHandle* FDTD_new(void) {
    FDTDHandle* h = new FDTDHandle();
    h->probe_device();   // records FDTD_ERR_NODEVICE when there is no GPU
    return h;
}

void FDTD_set_wavelength(FDTDHandle* h, double wavelength) {
    h->wavelength = wavelength;
    h->R = wavelength / (2 * M_PI);
}

void FDTD_set_physical_dims(FDTDHandle* h, double X, double Y, double Z, double dx, double dy,
                            double dz) {
    h->X = X; h->Y = Y; h->Z = Z;
    h->dx = dx; h->dy = dy; h->dz = dz;
}

void FDTD_set_grid_dims(FDTDHandle* h, int Nx, int Ny, int Nz) {
    h->Nx = Nx; h->Ny = Ny; h->Nz = Nz;
}

void FDTD_set_local_grid(FDTDHandle* h, int k0, int j0, int i0, int K, int J, int I) {
    h->k0 = k0; h->j0 = j0; h->i0 = i0;
    h->K = K; h->J = J; h->I = I;
}

// As in src/fdtd.cpp:96-100 the CPML tables keep the dt of their last build.
void FDTD_set_dt(FDTDHandle* h, double dt) {
    h->dt = dt;
    h->odt = 1.0 / dt;
    h->r32.coeffs_valid = false;
    h->r64.coeffs_valid = false;
}

void FDTD_set_complex_eps(FDTDHandle* h, bool complex_eps) {
    h->lossy = complex_eps;
    h->r32.coeffs_valid = false;
    h->r64.coeffs_valid = false;
}

void FDTD_set_field_arrays(FDTDHandle* h, double* Ex, double* Ey, double* Ez, double* Hx,
                           double* Hy, double* Hz) {
    h->hE[0] = Ex; h->hE[1] = Ey; h->hE[2] = Ez;
    h->hH[0] = Hx; h->hH[1] = Hy; h->hH[2] = Hz;
}

void FDTD_set_mat_arrays(FDTDHandle* h, fdtd_complex128* ex, fdtd_complex128* ey,
                         fdtd_complex128* ez, fdtd_complex128* mx, fdtd_complex128* my,
                         fdtd_complex128* mz) {
    h->heps[0] = (c128*)ex; h->heps[1] = (c128*)ey; h->heps[2] = (c128*)ez;
    h->hmu[0] = (c128*)mx; h->hmu[1] = (c128*)my; h->hmu[2] = (c128*)mz;
    h->r32.coeffs_valid = false;
    h->r64.coeffs_valid = false;
}

void FDTD_set_bc(FDTDHandle* h, char* newbc) {
    for (int a = 0; a < 3; a++) h->bc[a] = newbc[a];
}

void FDTD_set_pml_widths(FDTDHandle* h, int xmin, int xmax, int ymin, int ymax, int zmin,
                         int zmax) {
    h->w[0] = xmin; h->w[1] = xmax; h->w[2] = ymin;
    h->w[3] = ymax; h->w[4] = zmin; h->w[5] = zmax;
}

void FDTD_set_pml_properties(FDTDHandle* h, double sigma, double alpha, double kappa,
                             double pow_) {
    h->sigma = sigma; h->alpha = alpha; h->kappa = kappa; h->pw = pow_;
    h->compute_tables();
}

// Recomputes the tables (src/fdtd.cpp:779-880).  The device CPML state of the
// per-call path is released here and re-created, zeroed, by the next per-call
// half step with the chunk's slab sizes (the reference allocates it here
// uninitialised and relies on FDTD_reset_pml).
void FDTD_build_pml(FDTDHandle* h) {
    h->compute_tables();
    if (h->device < 0) return;
    cudaSetDevice(h->device);
    for (auto& a : h->lpsi)
        for (auto& sd : a)
            for (auto& b : sd) b.release();
}

void FDTD_reset_pml(FDTDHandle* h) {
    if (h->ready() != FDTD_OK) return;
    for (int a = 0; a < 3; a++)
        for (int sd = 0; sd < 2; sd++) {
            long long n = h->slab_cells(a, sd);
            for (int q = 0; q < 4; q++)
                if (h->lpsi[a][sd][q].p && n) {
                    cudaError_t e = cudaMemsetAsync(h->lpsi[a][sd][q].p, 0, sizeof(double) * n, h->stream);
                    if (e != cudaSuccess) { h->cuda_fail(e, "FDTD_reset_pml"); return; }
                }
        }
    h->sync_check("FDTD_reset_pml");
}

void FDTD_set_t0_arrays(FDTDHandle* h, fdtd_complex128* a, fdtd_complex128* b, fdtd_complex128* c,
                        fdtd_complex128* d, fdtd_complex128* e, fdtd_complex128* f) {
    fdtd_complex128* v[6] = {a, b, c, d, e, f};
    for (int q = 0; q < 6; q++) h->ht0[q] = (c128*)v[q];
}

void FDTD_set_t1_arrays(FDTDHandle* h, fdtd_complex128* a, fdtd_complex128* b, fdtd_complex128* c,
                        fdtd_complex128* d, fdtd_complex128* e, fdtd_complex128* f) {
    fdtd_complex128* v[6] = {a, b, c, d, e, f};
    for (int q = 0; q < 6; q++) h->ht1[q] = (c128*)v[q];
}

double FDTD_calc_phase_2T(double t0, double t1, double f0, double f1) {
    return fdtdb::phase_2t(t0, t1, f0, f1);
}

double FDTD_calc_amplitude_2T(double t0, double t1, double f0, double f1, double phase) {
    return fdtdb::amplitude_2t(t0, t1, f0, f1, phase);
}

double FDTD_calc_phase_3T(double t0, double t1, double t2, double f0, double f1, double f2) {
    return fdtdb::phase_3t(t0, t1, t2, f0, f1, f2);
}

double FDTD_calc_amplitude_3T(double t0, double t1, double t2, double f0, double f1, double f2,
                              double phase) {
    return fdtdb::amplitude_3t(t0, t1, t2, f0, f1, f2, phase);
}

// src/fdtd.cpp:1586-1593
void FDTD_set_source_properties(FDTDHandle* h, double src_T, double src_min) {
    h->src_T = src_T;
    h->src_min = src_min;
    h->src_k = src_T * src_T / log((1 + src_min) / src_min);
}

double FDTD_src_func_t(FDTDHandle* h, int n, double t, double phase) {
    return fdtdb::src_value(t, phase, h->src_T, h->src_min, h->src_k);
}

void FDTD_clear_sources(FDTDHandle* h) { h->sources.clear(); }

}  // extern "C"

// ============================================== per-call padded-layout path
static int legacy_upload_source_arrays(FDTDHandle* h, std::vector<fdtdb::LegacySource>& out) {
    for (size_t s = 0; s < h->sources.size(); s++) {
        const HostSource& hs = h->sources[s];
        if (hs.i0 < 0 || hs.j0 < 0 || hs.k0 < 0 || hs.I < 0 || hs.J < 0 || hs.K < 0 ||
            hs.i0 + hs.I > h->I || hs.j0 + hs.J > h->J || hs.k0 + hs.K > h->K)
            return h->fail(FDTD_ERR_ARG, "source box %zu lies outside the local chunk", s);
    }
    size_t need = h->sources.size() * 6;
    if (h->lsrc.size() < need) h->lsrc.resize(need);
    out.clear();
    for (size_t s = 0; s < h->sources.size(); s++) {
        const HostSource& hs = h->sources[s];
        fdtdb::LegacySource ls;
        long long n = (long long)hs.I * hs.J * hs.K;
        for (int c = 0; c < 6; c++) {
            DevBuf& b = h->lsrc[6 * s + c];
            CK(b.ensure(sizeof(c128) * (n > 0 ? n : 1)));
            if (n > 0) CK(cudaMemcpyAsync(b.p, hs.comp[c], sizeof(c128) * n, cudaMemcpyDefault, h->stream));
            ls.comp[c] = dptr<c128>(b);
        }
        ls.i0 = hs.i0; ls.j0 = hs.j0; ls.k0 = hs.k0; ls.I = hs.I; ls.J = hs.J; ls.K = hs.K;
        out.push_back(ls);
    }
    return FDTD_OK;
}

static int legacy_view(FDTDHandle* h, fdtdb::LegacyView& v) {
    ensure_tables(h);
    v.Nx = h->Nx; v.Ny = h->Ny; v.Nz = h->Nz;
    v.I = h->I; v.J = h->J; v.K = h->K; v.i0 = h->i0; v.j0 = h->j0; v.k0 = h->k0;
    v.odx = h->R / h->dx; v.ody = h->R / h->dy; v.odz = h->R / h->dz;
    v.dt = h->dt; v.odt = h->odt; v.lossy = h->lossy;
    for (int a = 0; a < 3; a++) v.bc[a] = h->bc[a];
    for (int q = 0; q < 6; q++) v.w[q] = h->w[q];
    for (int a = 0; a < 3; a++)
        for (int sd = 0; sd < 2; sd++)
            for (int q = 0; q < 4; q++) {
                long long n = h->slab_cells(a, sd);
                DevBuf& b = h->lpsi[a][sd][q];
                if (n > 0 && (!b.p || b.bytes < sizeof(double) * n)) {
                    // the chunk or widths changed since the last build: start from zero
                    CK(b.ensure(sizeof(double) * n));
                    CK(cudaMemsetAsync(b.p, 0, sizeof(double) * n, h->stream));
                }
                v.psi[a][sd][q] = dptr<double>(b);
            }
    if (h->ltab_dirty) {
        for (int a = 0; a < 3; a++)
            for (int q = 0; q < 6; q++) {
                size_t n = h->tab[a][q].size();
                CK(h->ltab[a][q].ensure(sizeof(double) * (n ? n : 1)));
                if (n) CK(cudaMemcpyAsync(h->ltab[a][q].p, h->tab[a][q].data(), sizeof(double) * n,
                                          cudaMemcpyDefault, h->stream));
            }
        CK(cudaStreamSynchronize(h->stream));
        h->ltab_dirty = false;
    }
    for (int a = 0; a < 3; a++)
        for (int q = 0; q < 6; q++) v.tab[a][q] = dptr<double>(h->ltab[a][q]);
    for (int c = 0; c < 3; c++) {
        v.E[c] = dptr<double>(h->lE[c]);
        v.H[c] = dptr<double>(h->lH[c]);
        v.eps[c] = dptr<c128>(h->leps[c]);
        v.mu[c] = dptr<c128>(h->lmu[c]);
    }
    return FDTD_OK;
}

// Copies the caller's padded fields (and the material component set that the
// half step reads) to the device mirrors.
static int legacy_in(FDTDHandle* h, bool need_eps, bool need_mu) {
    long long np = h->npad(), n = h->ncells();
    for (int c = 0; c < 3; c++) {
        if (!h->hE[c] || !h->hH[c]) return h->fail(FDTD_ERR_ARG, "field arrays are not set");
        CK(h->lE[c].ensure(sizeof(double) * np));
        CK(h->lH[c].ensure(sizeof(double) * np));
        CK(cudaMemcpyAsync(h->lE[c].p, h->hE[c], sizeof(double) * np, cudaMemcpyDefault, h->stream));
        CK(cudaMemcpyAsync(h->lH[c].p, h->hH[c], sizeof(double) * np, cudaMemcpyDefault, h->stream));
        if (need_eps) {
            if (!h->heps[c]) return h->fail(FDTD_ERR_ARG, "material arrays are not set");
            CK(h->leps[c].ensure(sizeof(c128) * n));
            CK(cudaMemcpyAsync(h->leps[c].p, h->heps[c], sizeof(c128) * n, cudaMemcpyDefault, h->stream));
        }
        if (need_mu) {
            if (!h->hmu[c]) return h->fail(FDTD_ERR_ARG, "material arrays are not set");
            CK(h->lmu[c].ensure(sizeof(c128) * n));
            CK(cudaMemcpyAsync(h->lmu[c].p, h->hmu[c], sizeof(c128) * n, cudaMemcpyDefault, h->stream));
        }
    }
    return FDTD_OK;
}

static int legacy_out(FDTDHandle* h) {
    long long np = h->npad();
    for (int c = 0; c < 3; c++) {
        CK(cudaMemcpyAsync(h->hE[c], h->lE[c].p, sizeof(double) * np, cudaMemcpyDefault, h->stream));
        CK(cudaMemcpyAsync(h->hH[c], h->lH[c].p, sizeof(double) * np, cudaMemcpyDefault, h->stream));
    }
    return h->sync_check("legacy half step");
}

static int legacy_half_step(FDTDHandle* h, bool is_H, double t) {
    if (h->ready() != FDTD_OK) return h->status;
    int rc;
    if ((rc = legacy_in(h, true, true)) != FDTD_OK) return rc;
    std::vector<fdtdb::LegacySource> srcs;
    if ((rc = legacy_upload_source_arrays(h, srcs)) != FDTD_OK) return rc;
    fdtdb::LegacyView v;
    if ((rc = legacy_view(h, v)) != FDTD_OK) return rc;
    if (is_H)
        fdtdb::legacy_update_H(v, srcs.data(), (int)srcs.size(), t, h->src_T, h->src_min, h->src_k,
                               h->stream);
    else
        fdtdb::legacy_update_E(v, srcs.data(), (int)srcs.size(), t, h->src_T, h->src_min, h->src_k,
                               h->stream);
    CK(cudaGetLastError());
    return legacy_out(h);
}

// Uploads t (complex snapshot arrays) to device mirrors, returns device pointers.
static int legacy_snap_in(FDTDHandle* h, c128* const* host, DevBuf* dev, c128** out) {
    long long n = h->ncells();
    for (int c = 0; c < 6; c++) {
        if (!host[c]) return h->fail(FDTD_ERR_ARG, "t0/t1 arrays are not set");
        CK(dev[c].ensure(sizeof(c128) * n));
        CK(cudaMemcpyAsync(dev[c].p, host[c], sizeof(c128) * n, cudaMemcpyDefault, h->stream));
        out[c] = dptr<c128>(dev[c]);
    }
    return FDTD_OK;
}

static int legacy_snap_out(FDTDHandle* h, c128* const* host, DevBuf* dev) {
    long long n = h->ncells();
    for (int c = 0; c < 6; c++)
        CK(cudaMemcpyAsync(host[c], dev[c].p, sizeof(c128) * n, cudaMemcpyDefault, h->stream));
    return h->sync_check("snapshot");
}

static int legacy_capture_into(FDTDHandle* h, c128* const* host, DevBuf* dev) {
    if (h->ready() != FDTD_OK) return h->status;
    int rc;
    if ((rc = legacy_in(h, false, false)) != FDTD_OK) return rc;
    c128* d[6];
    if ((rc = legacy_snap_in(h, host, dev, d)) != FDTD_OK) return rc;
    fdtdb::LegacyView v;
    if ((rc = legacy_view(h, v)) != FDTD_OK) return rc;
    fdtdb::legacy_capture(v, d, h->stream);
    CK(cudaGetLastError());
    return legacy_snap_out(h, host, dev);
}

extern "C" {

void FDTD_update_H(FDTDHandle* h, int n, double t) { legacy_half_step(h, true, t); }

void FDTD_update_E(FDTDHandle* h, int n, double t) { legacy_half_step(h, false, t); }

void FDTD_capture_t0_fields(FDTDHandle* h) { legacy_capture_into(h, h->ht0, h->lt0); }

void FDTD_capture_t1_fields(FDTDHandle* h) { legacy_capture_into(h, h->ht1, h->lt1); }

void FDTD_calc_complex_fields_2T(FDTDHandle* h, double t0, double t1) {
    if (h->ready() != FDTD_OK) return;
    if (legacy_in(h, false, false) != FDTD_OK) return;
    c128* d0[6];
    if (legacy_snap_in(h, h->ht0, h->lt0, d0) != FDTD_OK) return;
    fdtdb::LegacyView v;
    if (legacy_view(h, v) != FDTD_OK) return;
    fdtdb::legacy_extract_2t(v, d0, t0, t1, h->stream);
    legacy_snap_out(h, h->ht0, h->lt0);
}

void FDTD_calc_complex_fields_3T(FDTDHandle* h, double t0, double t1, double t2) {
    if (h->ready() != FDTD_OK) return;
    if (legacy_in(h, false, false) != FDTD_OK) return;
    c128 *d0[6], *d1[6];
    if (legacy_snap_in(h, h->ht0, h->lt0, d0) != FDTD_OK) return;
    if (legacy_snap_in(h, h->ht1, h->lt1, d1) != FDTD_OK) return;
    fdtdb::LegacyView v;
    if (legacy_view(h, v) != FDTD_OK) return;
    const c128* c1[6];
    for (int c = 0; c < 6; c++) c1[c] = d1[c];
    fdtdb::legacy_extract_3t(v, d0, c1, t0, t1, t2, h->stream);
    legacy_snap_out(h, h->ht0, h->lt0);
}

// src/fdtd.cpp:1498-1579: with calc_phase the caller's complex currents are
// rewritten in place as (|J|, -atan2(im, re)); the arrays are retained.
void FDTD_add_source(FDTDHandle* h, fdtd_complex128* Jx, fdtd_complex128* Jy, fdtd_complex128* Jz,
                     fdtd_complex128* Mx, fdtd_complex128* My, fdtd_complex128* Mz, int i0, int j0,
                     int k0, int I, int J, int K, bool calc_phase) {
    HostSource s;
    fdtd_complex128* v[6] = {Jx, Jy, Jz, Mx, My, Mz};
    for (int c = 0; c < 6; c++) s.comp[c] = (c128*)v[c];
    s.i0 = i0; s.j0 = j0; s.k0 = k0; s.I = I; s.J = J; s.K = K;
    h->sources.push_back(s);
    long long n = (long long)I * J * K;
    if (!calc_phase || n <= 0) return;
    if (h->ready() != FDTD_OK) return;
    DevBuf tmp;
    cudaError_t e = tmp.ensure(sizeof(c128) * n);
    for (int c = 0; c < 6 && e == cudaSuccess; c++) {
        e = cudaMemcpyAsync(tmp.p, s.comp[c], sizeof(c128) * n, cudaMemcpyDefault, h->stream);
        if (e != cudaSuccess) break;
        fdtdb::launch_amp_phase(dptr<c128>(tmp), n, h->stream);
        e = cudaMemcpyAsync(s.comp[c], tmp.p, sizeof(c128) * n, cudaMemcpyDefault, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    tmp.release();
    if (e != cudaSuccess) h->cuda_fail(e, "FDTD_add_source");
}

// Ghost-exchange packing helpers (src/fdtd.cpp:1789-1929).  They only move
// values between the caller's host arrays for an MPI halo exchange (no
// arithmetic), so they stay on the host; FDTD_solve_cw needs no ghost exchange.
void FDTD_copy_to_ghost_comm(double* src, fdtd_complex128* ghost, int I, int J, int K) {
    long long sj = K + 2, si = (long long)(J + 2) * (K + 2), o = 0;
    for (int side = 0; side < 2; side++, o += (long long)I * J)
        for (int i = 0; i < I; i++)
            for (int j = 0; j < J; j++)
                ghost[o + j + (long long)i * J].real = src[(i + 1) * si + (j + 1) * sj + (side ? K : 1)];
    for (int side = 0; side < 2; side++, o += (long long)I * K)
        for (int i = 0; i < I; i++)
            for (int k = 0; k < K; k++)
                ghost[o + k + (long long)i * K].real = src[(i + 1) * si + (side ? J : 1) * sj + k + 1];
    for (int side = 0; side < 2; side++, o += (long long)J * K)
        for (int j = 0; j < J; j++)
            for (int k = 0; k < K; k++)
                ghost[o + k + (long long)j * K].real = src[(side ? I : 1) * si + (j + 1) * sj + k + 1];
}

void FDTD_copy_from_ghost_comm(double* dest, fdtd_complex128* ghost, int I, int J, int K) {
    long long sj = K + 2, si = (long long)(J + 2) * (K + 2);
    long long o = 2LL * I * J + 2LL * I * K + 2LL * J * K;
    for (int side = 0; side < 2; side++, o += (long long)I * J)
        for (int i = 0; i < I; i++)
            for (int j = 0; j < J; j++)
                dest[(i + 1) * si + (j + 1) * sj + (side ? K + 1 : 0)] = ghost[o + j + (long long)i * J].real;
    for (int side = 0; side < 2; side++, o += (long long)I * K)
        for (int i = 0; i < I; i++)
            for (int k = 0; k < K; k++)
                dest[(i + 1) * si + (side ? J + 1 : 0) * sj + k + 1] = ghost[o + k + (long long)i * K].real;
    for (int side = 0; side < 2; side++, o += (long long)J * K)
        for (int j = 0; j < J; j++)
            for (int k = 0; k < K; k++)
                dest[(side ? I + 1 : 0) * si + (j + 1) * sj + k + 1] = ghost[o + k + (long long)j * K].real;
}

// ------------------------------------------------------------ additions
void FDTD_delete(FDTDHandle* h) {
    if (!h) return;
    if (h->device >= 0) {
        cudaSetDevice(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        h->r32.release_all();
        h->r64.release_all();
        for (int c = 0; c < 3; c++) {
            h->lE[c].release(); h->lH[c].release(); h->leps[c].release(); h->lmu[c].release();
        }
        for (auto& a : h->lpsi) for (auto& s : a) for (auto& b : s) b.release();
        for (auto& a : h->ltab) for (auto& b : a) b.release();
        for (auto& b : h->lsrc) b.release();
        for (int c = 0; c < 6; c++) { h->lt0[c].release(); h->lt1[c].release(); }
        for (auto& v : h->ev) if (v) cudaEventDestroy(v);
        if (h->pinned) cudaFreeHost(h->pinned);
        if (h->stream && !h->ext_stream) cudaStreamDestroy(h->stream);
    }
    delete h;
}

int FDTD_last_error(FDTDHandle* h, char* buf, int buflen) {
    if (buf && buflen > 0) {
        std::strncpy(buf, h->message.c_str(), (size_t)buflen - 1);
        buf[buflen - 1] = 0;
    }
    return h->status;
}

int FDTD_set_device(FDTDHandle* h, int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return h->fail(FDTD_ERR_NODEVICE, "no CUDA device is visible");
    if (device < 0 || device >= n) return h->fail(FDTD_ERR_ARG, "device %d out of range [0, %d)", device, n);
    if (h->stream && device != h->device)
        return h->fail(FDTD_ERR_ARG, "FDTD_set_device must precede the first device use");
    h->device = device;
    return FDTD_OK;
}

int FDTD_set_zchunk(FDTDHandle* h, int planes) {
    if (planes < 0) return h->fail(FDTD_ERR_ARG, "planes per CTA must be >= 0");
    h->zchunk = planes;
    return FDTD_OK;
}

int FDTD_set_precision(FDTDHandle* h, int bits) {
    if (bits != 32 && bits != 64) return h->fail(FDTD_ERR_ARG, "precision must be 32 or 64");
    h->precision = bits;
    return FDTD_OK;
}

int FDTD_set_kernel(FDTDHandle* h, int which) {
    if (which != 0 && which != 1 && which != 3 && which != 5 && which != 6)
        return h->fail(FDTD_ERR_ARG,
                       "kernel must be 0 (auto), 1 (scalar), 3 (fused), 5 (vector) or 6 (vector, interior/rim split)");
    h->kernel = which;
    return FDTD_OK;
}

int FDTD_host_register(void* ptr, long long bytes) {
    if (!ptr || bytes <= 0) return FDTD_ERR_ARG;
    cudaError_t e = cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();   // leave no error behind for later calls
        return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? FDTD_ERR_NODEVICE : FDTD_ERR_CUDA;
    }
    return FDTD_OK;
}

int FDTD_host_unregister(void* ptr) {
    if (!ptr) return FDTD_ERR_ARG;
    cudaError_t e = cudaHostUnregister(ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return FDTD_ERR_CUDA;
    }
    return FDTD_OK;
}

}  // extern "C"

// ================================================== device-resident solve
namespace {

template <typename T> Resident<T>& resident(FDTDHandle* h);
template <> Resident<float>& resident<float>(FDTDHandle* h) { return h->r32; }
template <> Resident<double>& resident<double>(FDTDHandle* h) { return h->r64; }

// Allocates the resident arrays for the current grid and PML widths.
// halo = 1 (z slabs): the six field arrays get one plane below and one above
// the slab; the interior starts one plane into each array.
template <typename T>
int alloc_resident(FDTDHandle* h, Resident<T>& r, bool two_sets, int halo = 0) {
    int px = (h->Nx + 31) / 32 * 32;
    bool same = r.Nx == h->Nx && r.Ny == h->Ny && r.Nz == h->Nz && r.px == px && r.halo == halo;
    if (!same) r.release_all();
    r.Nx = h->Nx; r.Ny = h->Ny; r.Nz = h->Nz; r.px = px; r.halo = halo;
    size_t cells = (size_t)h->Nz * h->Ny * px;
    size_t fcells = (size_t)(h->Nz + 2 * halo) * h->Ny * px;
    long long slab[3] = {(long long)h->Nz * h->Ny * (h->w[0] + h->w[1]),
                         (long long)h->Nz * (h->w[2] + h->w[3]) * px,
                         (long long)(h->w[4] + h->w[5]) * h->Ny * px};
    for (int s = 0; s < (two_sets ? 2 : 1); s++) {
        for (int c = 0; c < 6; c++) CK(r.F[s][c].ensure(sizeof(T) * fcells));
        for (int a = 0; a < 3; a++)
            for (int q = 0; q < 4; q++) CK(r.psi[s][a][q].ensure(sizeof(T) * (slab[a] ? slab[a] : 1)));
    }
    for (int c = 0; c < 3; c++) CK(r.bE[c].ensure(sizeof(T) * cells));
    for (int s = 0; s < 2; s++)
        for (int c = 0; c < 6; c++) CK(r.snap[s][c].ensure(sizeof(T) * cells));
    CK(r.stepbase.ensure(sizeof(long long)));
    CK(r.flag.ensure(sizeof(int) * 4));
    CK(r.err.ensure(sizeof(int) * 4));
    return FDTD_OK;
}

// Material upload (one component at a time through one staging buffer) and
// the pitched update coefficients; detects a uniform mu per component.
template <typename T>
int prepare_materials(FDTDHandle* h, Resident<T>& r) {
    ensure_tables(h);
    long long n = (long long)h->Nx * h->Ny * h->Nz;
    size_t cells = (size_t)h->Nz * h->Ny * r.px;
    CK(r.stage.ensure(sizeof(c128) * n));
    r.lossy = h->lossy;
    for (int c = 0; c < 3; c++) {
        if (!h->heps[c] || !h->hmu[c]) return h->fail(FDTD_ERR_ARG, "material arrays are not set");
        // pitched arrays: zero the row padding once so that every element is defined
        CK(cudaMemsetAsync(r.bE[c].p, 0, sizeof(T) * cells, h->stream));
        CK(cudaMemcpyAsync(r.stage.p, h->heps[c], sizeof(c128) * n, cudaMemcpyDefault, h->stream));
        T* a_out = nullptr;
        if (h->lossy) {
            CK(r.aE[c].ensure(sizeof(T) * cells));
            CK(cudaMemsetAsync(r.aE[c].p, 0, sizeof(T) * cells, h->stream));
            a_out = dptr<T>(r.aE[c]);
        }
        fdtdb::launch_material_coeffs<T>(dptr<c128>(r.stage), nullptr, h->Nx, h->Ny, h->Nz, r.px,
                                         h->dt, h->lossy, dptr<T>(r.bE[c]), a_out, nullptr, h->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(r.stage.p, h->hmu[c], sizeof(c128) * n, cudaMemcpyDefault, h->stream));
        int one = 1;
        CK(cudaMemcpyAsync(r.flag.p, &one, sizeof(int), cudaMemcpyDefault, h->stream));
        fdtdb::launch_uniform_check(dptr<c128>(r.stage), n, dptr<int>(r.flag), h->stream);
        int uniform = 0;
        c128 first;
        CK(cudaMemcpyAsync(&uniform, r.flag.p, sizeof(int), cudaMemcpyDefault, h->stream));
        CK(cudaMemcpyAsync(&first, r.stage.p, sizeof(c128), cudaMemcpyDefault, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        r.mu_uniform[c] = uniform != 0;
        r.mu_value[c] = first.real;
        if (!r.mu_uniform[c]) {
            CK(r.bH[c].ensure(sizeof(T) * cells));
            CK(cudaMemsetAsync(r.bH[c].p, 0, sizeof(T) * cells, h->stream));
            fdtdb::launch_material_coeffs<T>(nullptr, dptr<c128>(r.stage), h->Nx, h->Ny, h->Nz, r.px,
                                             h->dt, h->lossy, nullptr, nullptr, dptr<T>(r.bH[c]),
                                             h->stream);
            CK(cudaGetLastError());
        }
    }
    // CPML tables reordered by local slab index (min slab reversed) with 1/kappa
    for (int a = 0; a < 3; a++) {
        int w0 = h->w[2 * a], w1 = h->w[2 * a + 1];
        std::vector<T> t[6];
        for (int q = 0; q < 6; q++) t[q].assign((size_t)(w0 + w1 > 0 ? w0 + w1 : 1), T(0));
        for (int l = 0; l < w0 + w1; l++) {
            int tq = l < w0 ? (w0 - 1 - l) : l;
            t[0][l] = T(1.0 / h->tab[a][0][tq]);
            t[1][l] = T(h->tab[a][1][tq]);
            t[2][l] = T(h->tab[a][2][tq]);
            t[3][l] = T(1.0 / h->tab[a][3][tq]);
            t[4][l] = T(h->tab[a][4][tq]);
            t[5][l] = T(h->tab[a][5][tq]);
        }
        for (int q = 0; q < 6; q++) {
            CK(r.tab[a][q].ensure(sizeof(T) * t[q].size()));
            CK(cudaMemcpyAsync(r.tab[a][q].p, t[q].data(), sizeof(T) * t[q].size(),
                               cudaMemcpyDefault, h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
    }
    r.coeffs_valid = true;
    return FDTD_OK;
}

// Uploads the registered sources (already amplitude/phase) and folds the
// update coefficient of each cell into (A cos phase, A sin phase).
template <typename T>
int prepare_sources(FDTDHandle* h, Resident<T>& r, fdtdb::SourceList<T>& list) {
    size_t ns = h->sources.size();
    if (ns > (size_t)fdtdb::kMaxSources)
        return h->fail(FDTD_ERR_ARG, "at most %d source boxes per solve", fdtdb::kMaxSources);
    if (r.src_ap.size() < 6 * ns) { r.src_ap.resize(6 * ns); r.src_coef.resize(6 * ns); }
    list.n = (int)ns;
    for (size_t s = 0; s < ns; s++) {
        const HostSource& hs = h->sources[s];
        if (hs.i0 < 0 || hs.j0 < 0 || hs.k0 < 0 || hs.i0 + hs.I > h->Nz || hs.j0 + hs.J > h->Ny ||
            hs.k0 + hs.K > h->Nx)
            return h->fail(FDTD_ERR_ARG, "source box %zu lies outside the grid", s);
        long long n = (long long)hs.I * hs.J * hs.K;
        fdtdb::DevSource<T>& d = list.s[s];
        d.i0 = hs.i0; d.j0 = hs.j0; d.k0 = hs.k0; d.I = hs.I; d.J = hs.J; d.K = hs.K;
        for (int c = 0; c < 6; c++) {
            d.comp[c] = nullptr;
            if (!hs.comp[c] || n <= 0) continue;
            // a component that is zero everywhere adds nothing: leave it out so
            // the half step it would drive skips the source test entirely
            bool any = false;
            for (long long q = 0; q < n && !any; q++) any = hs.comp[c][q].real != 0.0;
            if (!any) continue;
            DevBuf& ap = r.src_ap[6 * s + c];
            DevBuf& co = r.src_coef[6 * s + c];
            CK(ap.ensure(sizeof(c128) * n));
            CK(co.ensure(sizeof(T) * 2 * n));
            CK(cudaMemcpyAsync(ap.p, hs.comp[c], sizeof(c128) * n, cudaMemcpyDefault, h->stream));
            const T* coef_arr;
            double coef_s = 0;
            if (c < 3) {
                coef_arr = dptr<T>(r.bE[c]);
            } else {
                int m = c - 3;
                coef_arr = r.mu_uniform[m] ? nullptr : dptr<T>(r.bH[m]);
                coef_s = h->dt / r.mu_value[m];
            }
            fdtdb::launch_source_coeffs<T>(dptr<c128>(ap), hs.i0, hs.j0, hs.k0, hs.I, hs.J, hs.K,
                                           coef_arr, coef_s, h->Ny, r.px, dptr<T>(co), h->stream);
            CK(cudaGetLastError());
            d.comp[c] = dptr<T>(co);
        }
    }
    for (int side = 0; side < 2; side++) {
        int* b = list.box[side];
        b[0] = b[2] = b[4] = 1 << 30;
        b[1] = b[3] = b[5] = -1;
        for (size_t q = 0; q < ns; q++) {
            const fdtdb::DevSource<T>& d = list.s[q];
            if (!d.comp[3 * side] && !d.comp[3 * side + 1] && !d.comp[3 * side + 2]) continue;
            b[0] = std::min(b[0], d.i0); b[1] = std::max(b[1], d.i0 + d.I);
            b[2] = std::min(b[2], d.j0); b[3] = std::max(b[3], d.j0 + d.J);
            b[4] = std::min(b[4], d.k0); b[5] = std::max(b[5], d.k0 + d.K);
        }
    }
    return FDTD_OK;
}

template <typename T>
fdtdb::GridView<T> make_view(FDTDHandle* h, Resident<T>& r, int set = 0) {
    fdtdb::GridView<T> g;
    g.Nx = h->Nx; g.Ny = h->Ny; g.Nz = h->Nz; g.px = r.px;
    g.plane = (long long)h->Ny * r.px;
    g.odx = T(h->R / h->dx); g.ody = T(h->R / h->dy); g.odz = T(h->R / h->dz);
    for (int c = 0; c < 3; c++) {
        g.bE[c] = dptr<T>(r.bE[c]);
        g.aE[c] = h->lossy ? dptr<T>(r.aE[c]) : nullptr;
        g.bHarr[c] = r.mu_uniform[c] ? nullptr : dptr<T>(r.bH[c]);
        g.bH[c] = T(h->dt / r.mu_value[c]);
        g.bc[c] = h->bc[c];
    }
    int N[3] = {h->Nx, h->Ny, h->Nz};
    for (int a = 0; a < 3; a++) {
        fdtdb::PmlAxis<T>& P = g.pml[a];
        P.w0 = h->w[2 * a]; P.w1 = h->w[2 * a + 1]; P.wsum = P.w0 + P.w1;
        P.edge_max = N[a] - P.w1;
        P.off = 0;
        for (int q = 0; q < 4; q++) P.psi[q] = dptr<T>(r.psi[set][a][q]);
        P.kinvH = dptr<T>(r.tab[a][0]); P.bH = dptr<T>(r.tab[a][1]);
        P.cH = dptr<T>(r.tab[a][2]); P.kinvE = dptr<T>(r.tab[a][3]);
        P.bE = dptr<T>(r.tab[a][4]); P.cE = dptr<T>(r.tab[a][5]);
    }
    g.zlo = g.zhi = 0;
    for (int c = 0; c < 4; c++) g.zhalo[c] = nullptr;
    g.chk = nullptr;
#ifdef FDTD_BOUNDS_CHECK
    g.chk = dptr<int>(r.err) + 1;
#endif
    g.step_tab = dptr<double4>(r.steptab);
    return g;
}

// Probe point -> offset into the pitched E arrays.  Probe indices address the
// padded local arrays of the reference; a probe on a face ghost reads the
// periodic copy that the one-rank ghost exchange leaves there
// (emopt/fdtd.py:1733-1873), and edge/corner ghosts are always zero.
long long probe_offset(const FDTDHandle* h, int px, long long pidx) {
    if (pidx < 0) return -1;
    long long K2 = h->Nx + 2, J2 = h->Ny + 2;
    long long ip = pidx / (J2 * K2), rem = pidx % (J2 * K2);
    long long jp = rem / K2, kp = rem % K2;
    long long c[3] = {kp, jp, ip};
    long long N[3] = {h->Nx, h->Ny, h->Nz};
    int ghosts = 0;
    for (int a = 0; a < 3; a++) {
        if (c[a] == 0) { c[a] = N[a]; ghosts++; }          // min ghost <- last plane
        else if (c[a] == N[a] + 1) { c[a] = 1; ghosts++; }  // max ghost <- first plane
    }
    if (ghosts > 1 || ip < 0 || ip > h->Nz + 1) return -1;
    return ((c[2] - 1) * h->Ny + (c[1] - 1)) * (long long)px + (c[0] - 1);
}

// Named ranges on the profiler timeline (NVTX; free when no tool listens).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

// Consecutive phases: next() closes the open range and opens another; the
// last one closes on scope exit, early returns included.
struct NvtxPhases {
    bool open = false;
    void next(const char* name) {
        if (open) nvtxRangePop();
        nvtxRangePushA(name);
        open = true;
    }
    ~NvtxPhases() {
        if (open) nvtxRangePop();
    }
};

template <typename T>
int solve_impl(FDTDHandle* h, const FDTDSolveOptions* o, FDTDSolveResult* res) {
    NvtxRange call("FDTD_solve_cw");
    NvtxPhases phase;
    phase.next("set-up: materials, sources, step table");
    if (!h->whole_grid())
        return h->fail(FDTD_ERR_ARG, "FDTD_solve_cw needs the whole grid as the local chunk");
    if (h->slab) return h->fail(FDTD_ERR_ARG, "the handle is a z slab: it is stepped by FDTD_slab_*");
    if (o->Tn <= 0) return h->fail(FDTD_ERR_ARG, "Tn must be positive");
    if (h->Nx <= 0 || h->Ny <= 0 || h->Nz <= 0) return h->fail(FDTD_ERR_ARG, "empty grid");
    Resident<T>& r = resident<T>(h);
    long long launches = 0;
    bool periodic = false;
    for (int a = 0; a < 3; a++)
        if (h->bc[a] != '0' && h->bc[a] != 'E' && h->bc[a] != 'H') periodic = true;
    bool small_index = (long long)h->Nz * h->Ny * ((h->Nx + 31) / 32 * 32) < (1LL << 31) &&
                       (long long)h->Nz * h->Ny * (h->w[0] + h->w[1]) < (1LL << 31);
    // kernel ids: 0 auto, 1 scalar H/E pair, 3 fused z-marching step, 5
    // vector H/E pair, 6 vector pair split into interior and rim launches.
    // Auto takes the split pair in float32 when at least 60% of the warp
    // tasks lie in no CPML slab (the 1201 x 601 x 301 grating slab, 69%:
    // 3293 instead of 3605 us per step; the 321 x 161 x 101 MMI block, 23%:
    // 143 instead of 122), else the vector pair.
    int kid = h->kernel;
    if (kid == 0) {
        kid = 5;
        if (sizeof(T) == 4 && !periodic && small_index) {
            const fdtdb::GridView<T> gv = make_view<T>(h, r, 0);
            if (fdtdb::split_interior_fraction<T>(gv) >= 0.6) kid = 6;
        }
    }
    if (periodic || !small_index) kid = 1;
    const bool fused = kid == 3;
    const bool vec = kid == 5;
    const bool split = kid == 6;
    int rc;
    CK(cudaEventRecord(h->ev[2], h->stream));
    if ((rc = alloc_resident<T>(h, r, fused)) != FDTD_OK) return rc;
    CK(cudaMemsetAsync(r.err.p, 0, sizeof(int) * 4, h->stream));
    if (!o->materials_unchanged || !r.coeffs_valid) {
        if ((rc = prepare_materials<T>(h, r)) != FDTD_OK) return rc;
        launches += 3 + 3 + 3;   // eps coefficients, uniform checks, mu coefficients (upper bound)
    }
    fdtdb::SourceList<T> src;
    if ((rc = prepare_sources<T>(h, r, src)) != FDTD_OK) return rc;
    for (int q = 0; q < src.n; q++)
        for (int c = 0; c < 6; c++) launches += src.s[q].comp[c] ? 1 : 0;

    const long long Tn = o->Tn;
    const bool fixed = o->fixed_steps > 0;
    long long last = fixed ? o->fixed_steps - 1 : (long long)floor(o->Nmax);
    if (!fixed && o->Nmax < 0) last = -1;
    long long max_steps = (last + 1 > 0 ? last + 1 : 0) + 2 * Tn + Tn + 1;
    CK(r.steptab.ensure(sizeof(double4) * max_steps));
    fdtdb::launch_step_table(dptr<double4>(r.steptab), max_steps, h->dt, h->src_T,
                             h->src_min, h->src_k, h->stream);
    launches++;

    size_t cells = (size_t)h->Nz * h->Ny * r.px;
    for (int s = 0; s < (fused ? 2 : 1); s++) {
        for (int c = 0; c < 6; c++) CK(cudaMemsetAsync(r.F[s][c].p, 0, sizeof(T) * cells, h->stream));
        for (int a = 0; a < 3; a++)
            for (int q = 0; q < 4; q++)
                CK(cudaMemsetAsync(r.psi[s][a][q].p, 0, r.psi[s][a][q].bytes, h->stream));
    }
    // convergence probe state
    int nconv = o->nconv > 0 ? o->nconv : 0;
    int nc = nconv > 0 ? nconv : 1;
    CK(r.pwin.ensure(sizeof(double) * 9 * nc));
    CK(r.pA.ensure(sizeof(double) * 2 * nc));
    CK(r.pphi.ensure(sizeof(double) * 2 * nc));
    CK(r.ptimes.ensure(sizeof(double) * 3));
    CK(r.pout.ensure(sizeof(double) * 4));
    CK(r.pmap.ensure(sizeof(long long) * nc));
    CK(cudaMemsetAsync(r.pwin.p, 0, sizeof(double) * 9 * nc, h->stream));
    CK(cudaMemsetAsync(r.pA.p, 0, sizeof(double) * 2 * nc, h->stream));
    CK(cudaMemsetAsync(r.pphi.p, 0, sizeof(double) * 2 * nc, h->stream));
    CK(cudaMemsetAsync(r.ptimes.p, 0, sizeof(double) * 3, h->stream));
    CK(cudaMemsetAsync(r.pout.p, 0, sizeof(double) * 4, h->stream));
    std::vector<long long> map((size_t)nc, -1);
    for (int q = 0; q < nconv; q++) map[q] = probe_offset(h, r.px, o->conv_pts[q]);
    CK(cudaMemcpyAsync(r.pmap.p, map.data(), sizeof(long long) * nc, cudaMemcpyDefault, h->stream));
    CK(cudaStreamSynchronize(h->stream));   // map is a stack vector
    fdtdb::ProbeDev pd;
    pd.win = dptr<double>(r.pwin); pd.A = dptr<double>(r.pA);
    pd.phi = dptr<double>(r.pphi); pd.times = dptr<double>(r.ptimes);
    pd.out = dptr<double>(r.pout); pd.map = dptr<long long>(r.pmap);
    pd.samples = nullptr;
    pd.nconv = nconv;

    long long* sb = dptr<long long>(r.stepbase);
    fdtdb::GridView<T> g0 = make_view<T>(h, r, 0);
    fdtdb::GridView<T> g1 = fused ? make_view<T>(h, r, 1) : g0;
    T* f0[6];
    T* f1[6];
    for (int c = 0; c < 6; c++) {
        f0[c] = dptr<T>(r.F[0][c]);
        f1[c] = fused ? dptr<T>(r.F[1][c]) : f0[c];
    }
    // field set that holds the state after `steps` time steps
    auto cur_set = [&](long long steps) -> T* const* { return (fused && (steps & 1)) ? f1 : f0; };
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
    const int zc = h->zchunk > 0 ? h->zchunk : fdtdb::zmarch_chunk(h->Nx, h->Ny, h->Nz, dev_sms);
    auto run = [&](long long n_first, long long count) -> int {
        fdtdb::launch_set_ll(sb, n_first, h->stream);
        launches += 1 + count * (fused ? 1 : 2);
        for (long long q = 0; q < count; q++) {
            const bool odd = (n_first + q) & 1;
            if (fused) {
                CK(fdtdb::launch_step_zmarch<T>(odd ? g1 : g0, odd ? g0 : g1, odd ? f1 : f0,
                                                odd ? f0 : f1, src, sb, (int)q, zc, h->stream));
            } else if (vec) {
                CK(fdtdb::launch_step_vec<T>(g0, f0, src, sb, (int)q, h->stream));
            } else if (split) {
                CK(fdtdb::launch_step_split<T>(g0, f0, src, sb, (int)q, h->stream));

            } else {
                fdtdb::launch_step_unfused<T>(g0, f0, src, sb, (int)q, h->stream);
            }
        }
        CK(cudaGetLastError());
        return FDTD_OK;
    };

    CK(cudaEventRecord(h->ev[0], h->stream));
    phase.next("time loop with convergence probes");
    long long n = 0;
    double Ach = 1, Pch = 1;
    double amp_rtol = o->rtol, phi_rtol = sqrt(o->rtol);
    long long nprobes = 0;
    auto not_converged = [&]() {
        if (fixed) return true;
        return Ach > amp_rtol || Pch > phi_rtol || std::isnan(Ach) || std::isinf(Ach) ||
               std::isnan(Pch) || std::isinf(Pch);
    };
    while (not_converged()) {
        if ((double)n > (fixed ? (double)last : o->Nmax)) break;
        if (n + Tn - 1 > last) {
            if ((rc = run(n, last - n + 1)) != FDTD_OK) return rc;
            n = last + 1;
            continue;
        }
        if ((rc = run(n, Tn)) != FDTD_OK) return rc;
        T* const* cs = cur_set(n + Tn);
        fdtdb::launch_probe<T>(cs[0], cs[1], cs[2], pd, sb, (int)(Tn - 1), Tn, h->dt, h->stream);
        launches++;
        CK(cudaGetLastError());
        n += Tn;
        nprobes++;
        if (!fixed) {
            CK(cudaMemcpyAsync(h->pinned, r.pout.p, sizeof(double) * 2, cudaMemcpyDefault, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            Ach = h->pinned[0];
            Pch = h->pinned[1];
            if (o->stop_nonfinite && !(std::isfinite(Ach) && std::isfinite(Pch))) break;
        }
    }
    if (fixed) {
        CK(cudaMemcpyAsync(h->pinned, r.pout.p, sizeof(double) * 2, cudaMemcpyDefault, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        Ach = h->pinned[0];
        Pch = h->pinned[1];
    }
    phase.next("t0/t1 captures and 2 Tn steps");
    const long long n0 = n;
    for (int c = 0; c < 6; c++)
        CK(cudaMemcpyAsync(r.snap[0][c].p, cur_set(n0)[c], sizeof(T) * cells, cudaMemcpyDeviceToDevice, h->stream));
    if ((rc = run(n0, Tn)) != FDTD_OK) return rc;
    for (int c = 0; c < 6; c++)
        CK(cudaMemcpyAsync(r.snap[1][c].p, cur_set(n0 + Tn)[c], sizeof(T) * cells, cudaMemcpyDeviceToDevice, h->stream));
    if ((rc = run(n0 + Tn, Tn)) != FDTD_OK) return rc;
    CK(cudaEventRecord(h->ev[1], h->stream));
    phase.next("3-sample extraction and copy-out");

    // 3-sample extraction (src/fdtd.cpp:1346-1443) with t0 = n0 dt,
    // t1 = (n0+Tn) dt, t2 = (n0+2Tn) dt; H samples half a step earlier.
    double t0 = (double)n0 * h->dt, t1 = (double)(n0 + Tn) * h->dt, t2 = (double)(n0 + 2 * Tn) * h->dt;
    fdtdb::Fit3 fE = fdtdb::make_fit3(t0, t1, t2);
    fdtdb::Fit3 fH = fdtdb::make_fit3(t0 - 0.5 * h->dt, t1 - 0.5 * h->dt, t2 - 0.5 * h->dt);
    long long ncell = (long long)h->Nx * h->Ny * h->Nz;
    T* const* fin = cur_set(n0 + 2 * Tn);
    for (int c = 0; c < 6; c++) {
        if (!h->ht0[c]) return h->fail(FDTD_ERR_ARG, "t0 arrays are not set");
        fdtdb::launch_extract_3t<T>(dptr<T>(r.snap[0][c]), dptr<T>(r.snap[1][c]),
                                    fin[c], h->Nx, h->Ny, h->Nz, r.px, c < 3 ? fE : fH,
                                    dptr<c128>(r.stage), h->stream);
        launches++;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h->ht0[c], r.stage.p, sizeof(c128) * ncell, cudaMemcpyDefault, h->stream));
    }
    if (o->copy_t1) {
        for (int c = 0; c < 6; c++) {
            if (!h->ht1[c]) return h->fail(FDTD_ERR_ARG, "t1 arrays are not set");
            CK(cudaMemcpyAsync(r.stage.p, h->ht1[c], sizeof(c128) * ncell, cudaMemcpyDefault, h->stream));
            fdtdb::launch_snapshot_real<T>(dptr<T>(r.snap[1][c]), h->Nx, h->Ny, h->Nz, r.px,
                                           dptr<c128>(r.stage), h->stream);
            CK(cudaMemcpyAsync(h->ht1[c], r.stage.p, sizeof(c128) * ncell, cudaMemcpyDefault, h->stream));
        }
    }
    CK(cudaEventRecord(h->ev[3], h->stream));
    int kerr[2] = {0, 0};
    CK(cudaMemcpyAsync(kerr, r.err.p, sizeof(int) * 2, cudaMemcpyDefault, h->stream));
    if ((rc = h->sync_check("FDTD_solve_cw")) != FDTD_OK) return rc;
    if (kerr[0]) return h->fail(FDTD_ERR_CUDA, "a bounded wait in the step kernel gave up (code %d)", kerr[0]);
    if (kerr[1]) return h->fail(FDTD_ERR_CUDA, "bounds check: a step kernel computed an index outside its array (site %d)", kerr[1]);
    float ms_steps = 0, ms_total = 0;
    cudaEventElapsedTime(&ms_steps, h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&ms_total, h->ev[2], h->ev[3]);
    res->n_main = n0;
    res->steps = n0 + 2 * Tn;
    res->A_change = Ach;
    res->phi_change = Pch;
    res->nprobes = nprobes;
    res->device_ms = ms_steps;
    res->total_ms = ms_total;
    res->launches = launches;
    res->zchunk = fused ? zc : 0;
    res->status = FDTD_OK;
    if (!fixed && not_converged()) {
        bool bad = std::isnan(Ach) || std::isinf(Ach) || std::isnan(Pch) || std::isinf(Pch);
        res->status = bad ? FDTD_NONFINITE : FDTD_NMAX;
    }
    h->status = FDTD_OK;
    h->message.clear();
    return res->status;
}

}  // namespace

extern "C" int FDTD_solve_cw(FDTDHandle* h, const FDTDSolveOptions* o, FDTDSolveResult* res) {
    if (!o || !res) return h->fail(FDTD_ERR_ARG, "null options/result");
    if (o->nconv > 0 && !o->conv_pts) return h->fail(FDTD_ERR_ARG, "null conv_pts");
    if (h->ready() != FDTD_OK) return h->status;
    std::memset(res, 0, sizeof(*res));
    return h->precision == 32 ? solve_impl<float>(h, o, res) : solve_impl<double>(h, o, res);
}

// Continuous batching of CW solves (FDTD_serve_*), in this translation unit
// so that it shares the resident state and set-up code above.
#include "serve_engine.cuh"

// z slabs of a distributed solve (FDTD_slab_*), sharing the same set-up code.
#include "slab_engine.cuh"
