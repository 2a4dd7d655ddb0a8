// slab_engine.cuh -- FDTD_slab_*: one z slab of a CW solve split over GPUs.
//
// Included at the end of fdtd_abi.cu: a slab is an ordinary handle whose grid
// is the slab (Nx x Ny x I planes, materials, sources and t0/t1 arrays in the
// slab's own coordinates, as set_local_grid chunks are in the reference,
// emopt/fdtd.py:273-297), marked by FDTD_slab_set with its place in the global
// grid.  The time loop belongs to the caller, which exchanges one plane pair
// per half step with the neighbouring slabs (src/fdtd.cpp:180 and :508: the H
// update of the top plane reads Ex, Ey one plane above, the E update of the
// bottom plane reads Hx, Hy one plane below):
//
//     for each step n:  [E halo from the slab above]  FDTD_slab_step(n, 0)
//                       [H halo from the slab below]  FDTD_slab_step(n, 1)
//
// or, overlapping each exchange with the planes that do not need it
// (FDTD_slab_step_part: part 1 = the planes that read no halo, part 2 = the
// plane next to the halo):
//
//     step(n, 0, part 1); [wait for the E halo] step(n, 0, part 2);
//     [start the H exchange] step(n, 1, part 1); [wait for the H halo]
//     step(n, 1, part 2); [start the E exchange]
//
// The field arrays carry one halo plane below and above the slab; the
// exchange writes into them (FDTD_slab_halo gives the device addresses).
// Slabs that share a device and a stream need no exchange: each can read its
// neighbours' boundary planes in place (FDTD_slab_set_halo_source), stream
// order putting every H half step of a step before every E half step.  The
// vector kernels read a neighbour plane where the slab has a neighbour and apply
// the boundary rule of the global grid where it has none, and take the z CPML
// coefficient of the global plane, so every cell is updated exactly as in the
// single-GPU solve.  The convergence probe works on the probe values of all
// slabs: FDTD_slab_sample writes the values this slab holds (zeros
// elsewhere), the caller sums the buffers of all slabs in place, and
// FDTD_slab_probe runs the probe of FDTD_solve_cw on the sum.
//
// Everything runs on the handle's stream, which FDTD_set_stream can make the
// caller's (so that a collective library's stream order applies).

namespace {

template <typename T> fdtdb::SourceList<T>& slab_src(FDTDHandle* h);
template <> fdtdb::SourceList<float>& slab_src<float>(FDTDHandle* h) { return h->slab_src32; }
template <> fdtdb::SourceList<double>& slab_src<double>(FDTDHandle* h) { return h->slab_src64; }

template <typename T>
fdtdb::GridView<T> slab_view(FDTDHandle* h, Resident<T>& r) {
    fdtdb::GridView<T> g = make_view<T>(h, r);
    g.pml[2].off = h->slab_i0;
    g.pml[2].edge_max = h->slab_Nz - h->w[5];
    g.zlo = (char)(h->slab_lo ? 1 : 0);
    g.zhi = (char)(h->slab_hi ? 1 : 0);
    // the neighbour planes: the slab's own halo planes unless
    // FDTD_slab_set_halo_source named other ones
    const long long plane = (long long)r.Ny * r.px;
    const T* own[4] = {dptr<T>(r.F[0][0]) + (h->Nz + 1) * plane, dptr<T>(r.F[0][1]) + (h->Nz + 1) * plane,
                       dptr<T>(r.F[0][3]), dptr<T>(r.F[0][4])};
    for (int c = 0; c < 4; c++)
        g.zhalo[c] = h->slab_zhalo[c] ? static_cast<const T*>(h->slab_zhalo[c]) : own[c];
    return g;
}

// Interior pointers of the six field arrays (one halo plane into each).
template <typename T>
void slab_fields(Resident<T>& r, T** f) {
    const long long plane = (long long)r.Ny * r.px;
    for (int c = 0; c < 6; c++) f[c] = dptr<T>(r.F[0][c]) + plane;
}

template <typename T>
int slab_begin_impl(FDTDHandle* h, const FDTDSolveOptions* o, const long long* cells, int np) {
    Resident<T>& r = resident<T>(h);
    int rc;
    if ((rc = alloc_resident<T>(h, r, false, 1)) != FDTD_OK) return rc;
    CK(cudaMemsetAsync(r.err.p, 0, sizeof(int) * 4, h->stream));
    if (!o->materials_unchanged || !r.coeffs_valid)
        if ((rc = prepare_materials<T>(h, r)) != FDTD_OK) return rc;
    if ((rc = prepare_sources<T>(h, r, slab_src<T>(h))) != FDTD_OK) return rc;

    const long long Tn = o->Tn;
    const bool fixed = o->fixed_steps > 0;
    long long last = fixed ? o->fixed_steps - 1 : (long long)floor(o->Nmax);
    long long max_steps = (last + 1 > 0 ? last + 1 : 0) + 2 * Tn + Tn + 1;
    CK(r.steptab.ensure(sizeof(double4) * max_steps));
    fdtdb::launch_step_table(dptr<double4>(r.steptab), max_steps, h->dt, h->src_T, h->src_min,
                             h->src_k, h->stream);
    CK(cudaGetLastError());
    const size_t fcells = (size_t)(h->Nz + 2) * h->Ny * r.px;
    for (int c = 0; c < 6; c++) CK(cudaMemsetAsync(r.F[0][c].p, 0, sizeof(T) * fcells, h->stream));
    for (int a = 0; a < 3; a++)
        for (int q = 0; q < 4; q++) CK(cudaMemsetAsync(r.psi[0][a][q].p, 0, r.psi[0][a][q].bytes, h->stream));

    const int nc = np > 0 ? np : 1;
    CK(r.pwin.ensure(sizeof(double) * 9 * nc));
    CK(r.pA.ensure(sizeof(double) * 2 * nc));
    CK(r.pphi.ensure(sizeof(double) * 2 * nc));
    CK(r.ptimes.ensure(sizeof(double) * 3));
    CK(r.pout.ensure(sizeof(double) * 4));
    CK(r.pmap.ensure(sizeof(long long) * nc));
    CK(r.psamp.ensure(sizeof(double) * 3 * nc));
    CK(cudaMemsetAsync(r.pwin.p, 0, sizeof(double) * 9 * nc, h->stream));
    CK(cudaMemsetAsync(r.pA.p, 0, sizeof(double) * 2 * nc, h->stream));
    CK(cudaMemsetAsync(r.pphi.p, 0, sizeof(double) * 2 * nc, h->stream));
    CK(cudaMemsetAsync(r.ptimes.p, 0, sizeof(double) * 3, h->stream));
    CK(cudaMemsetAsync(r.pout.p, 0, sizeof(double) * 4, h->stream));
    CK(cudaMemsetAsync(r.psamp.p, 0, sizeof(double) * 3 * nc, h->stream));
    // global cell (i*Ny + j)*Nx + k -> offset from the interior base, if held here
    std::vector<long long> map((size_t)nc, -1);
    const long long per_plane = (long long)h->Ny * h->Nx;
    for (int q = 0; q < np; q++) {
        const long long cell = cells[q];
        if (cell < 0) continue;
        const long long iz = cell / per_plane, rem = cell % per_plane;
        if (iz < h->slab_i0 || iz >= h->slab_i0 + h->Nz) continue;
        map[q] = ((iz - h->slab_i0) * h->Ny + rem / h->Nx) * (long long)r.px + rem % h->Nx;
    }
    CK(cudaMemcpyAsync(r.pmap.p, map.data(), sizeof(long long) * nc, cudaMemcpyDefault, h->stream));
    // the half-step kernels read the step table at *stepbase + n with stepbase 0
    fdtdb::launch_set_ll(dptr<long long>(r.stepbase), 0, h->stream);
    CK(cudaGetLastError());
    h->slab_np = np;
    h->slab_Tn = Tn;
    return h->sync_check("FDTD_slab_begin");
}

// Planes of half step `half` for part 0 (all), 1 (the planes that read no
// halo plane) or 2 (the plane next to a neighbour's halo: the top plane of the
// H update reads E above, the bottom plane of the E update reads H below).
void slab_planes(const FDTDHandle* h, int half, int part, int* i0, int* ni) {
    const int I = h->Nz;
    const bool edge = half == 0 ? h->slab_hi != 0 : h->slab_lo != 0;
    const int eplane = half == 0 ? I - 1 : 0;
    if (part == 0 || (!edge && part == 1)) { *i0 = 0; *ni = I; return; }
    if (!edge) { *i0 = 0; *ni = 0; return; }                // part 2 without a neighbour
    if (part == 2) { *i0 = eplane; *ni = 1; return; }
    *i0 = half == 0 ? 0 : 1;                                // part 1 with a neighbour
    *ni = I - 1;
}

template <typename T>
int slab_step_impl(FDTDHandle* h, long long n, int half, int part) {
    Resident<T>& r = resident<T>(h);
    T* f[6];
    slab_fields<T>(r, f);
    fdtdb::GridView<T> g = slab_view<T>(h, r);
    int i0, ni;
    slab_planes(h, half, part, &i0, &ni);
    CK(fdtdb::launch_half_vec<T>(g, f, slab_src<T>(h), dptr<long long>(r.stepbase), (int)n, half,
                                 i0, ni, h->stream));
    return FDTD_OK;
}

template <typename T>
int slab_halo_impl(FDTDHandle* h, void** ptrs, long long* plane_elems) {
    Resident<T>& r = resident<T>(h);
    T* f[6];
    slab_fields<T>(r, f);
    const long long plane = (long long)h->Ny * r.px;
    ptrs[0] = f[0];                            // Ex, Ey of plane 0: to the slab below
    ptrs[1] = f[1];
    ptrs[2] = f[0] + h->Nz * plane;            // Ex, Ey halo above: from the slab above
    ptrs[3] = f[1] + h->Nz * plane;
    ptrs[4] = f[3] + (h->Nz - 1) * plane;      // Hx, Hy of the top plane: to the slab above
    ptrs[5] = f[4] + (h->Nz - 1) * plane;
    ptrs[6] = f[3] - plane;                    // Hx, Hy halo below: from the slab below
    ptrs[7] = f[4] - plane;
    *plane_elems = plane;
    return FDTD_OK;
}

template <typename T>
int slab_sample_impl(FDTDHandle* h, void** samples) {
    Resident<T>& r = resident<T>(h);
    T* f[6];
    slab_fields<T>(r, f);
    fdtdb::launch_slab_sample<T>(f[0], f[1], f[2], dptr<long long>(r.pmap), h->slab_np,
                                 dptr<double>(r.psamp), h->stream);
    CK(cudaGetLastError());
    *samples = r.psamp.p;
    return FDTD_OK;
}

template <typename T>
int slab_probe_impl(FDTDHandle* h, long long n_last, double* A, double* phi) {
    Resident<T>& r = resident<T>(h);
    fdtdb::ProbeDev pd;
    pd.win = dptr<double>(r.pwin); pd.A = dptr<double>(r.pA);
    pd.phi = dptr<double>(r.pphi); pd.times = dptr<double>(r.ptimes);
    pd.out = dptr<double>(r.pout); pd.map = dptr<long long>(r.pmap);
    pd.samples = dptr<double>(r.psamp);
    pd.nconv = h->slab_np;
    fdtdb::launch_probe<T>(nullptr, nullptr, nullptr, pd, dptr<long long>(r.stepbase), (int)n_last, 0,
                           h->dt, h->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->pinned, r.pout.p, sizeof(double) * 2, cudaMemcpyDefault, h->stream));
    int rc;
    if ((rc = h->sync_check("FDTD_slab_probe")) != FDTD_OK) return rc;
    *A = h->pinned[0];
    *phi = h->pinned[1];
    return FDTD_OK;
}

template <typename T>
int slab_capture_impl(FDTDHandle* h, int which) {
    Resident<T>& r = resident<T>(h);
    T* f[6];
    slab_fields<T>(r, f);
    const size_t cells = (size_t)h->Nz * h->Ny * r.px;
    for (int c = 0; c < 6; c++)
        CK(cudaMemcpyAsync(r.snap[which][c].p, f[c], sizeof(T) * cells, cudaMemcpyDeviceToDevice, h->stream));
    return FDTD_OK;
}

// 3-sample extraction (src/fdtd.cpp:1346-1443) into the slab's t0 arrays,
// with t0 = n0 dt, t1 = (n0 + Tn) dt, t2 = (n0 + 2 Tn) dt (H half a step earlier).
template <typename T>
int slab_finish_impl(FDTDHandle* h, long long n0, long long Tn) {
    Resident<T>& r = resident<T>(h);
    T* f[6];
    slab_fields<T>(r, f);
    const double t0 = (double)n0 * h->dt, t1 = (double)(n0 + Tn) * h->dt, t2 = (double)(n0 + 2 * Tn) * h->dt;
    fdtdb::Fit3 fE = fdtdb::make_fit3(t0, t1, t2);
    fdtdb::Fit3 fH = fdtdb::make_fit3(t0 - 0.5 * h->dt, t1 - 0.5 * h->dt, t2 - 0.5 * h->dt);
    const long long ncell = (long long)h->Nx * h->Ny * h->Nz;
    CK(r.stage.ensure(sizeof(c128) * ncell));
    for (int c = 0; c < 6; c++) {
        if (!h->ht0[c]) return h->fail(FDTD_ERR_ARG, "t0 arrays are not set");
        fdtdb::launch_extract_3t<T>(dptr<T>(r.snap[0][c]), dptr<T>(r.snap[1][c]), f[c], h->Nx, h->Ny,
                                    h->Nz, r.px, c < 3 ? fE : fH, dptr<c128>(r.stage), h->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h->ht0[c], r.stage.p, sizeof(c128) * ncell, cudaMemcpyDefault, h->stream));
    }
    int kerr[2] = {0, 0};
    CK(cudaMemcpyAsync(kerr, r.err.p, sizeof(int) * 2, cudaMemcpyDefault, h->stream));
    int rc;
    if ((rc = h->sync_check("FDTD_slab_finish")) != FDTD_OK) return rc;
    if (kerr[0]) return h->fail(FDTD_ERR_CUDA, "a bounded wait in a step kernel gave up (code %d)", kerr[0]);
    if (kerr[1]) return h->fail(FDTD_ERR_CUDA, "bounds check: a step kernel computed an index outside its array (site %d)", kerr[1]);
    return FDTD_OK;
}

// A slab was begun in the handle's current precision.
bool slab_ready(FDTDHandle* h) {
    return h && h->slab && (h->precision == 32 ? h->r32.halo : h->r64.halo) == 1;
}

}  // namespace

extern "C" int FDTD_set_stream(FDTDHandle* h, void* stream) {
    if (!h) return FDTD_ERR_ARG;
    if (h->ready() != FDTD_OK) return h->status;
    CK(cudaStreamSynchronize(h->stream));
    if (!h->ext_stream && h->stream) CK(cudaStreamDestroy(h->stream));
    h->stream = (cudaStream_t)stream;
    h->ext_stream = true;
    return FDTD_OK;
}

extern "C" int FDTD_slab_set(FDTDHandle* h, int i0, int Nz_global, int has_lo, int has_hi) {
    if (!h) return FDTD_ERR_ARG;
    if (i0 < 0 || Nz_global <= 0 || i0 + h->Nz > Nz_global || h->Nz <= 0)
        return h->fail(FDTD_ERR_ARG, "slab planes [%d, %d) do not fit a grid of %d planes", i0,
                       i0 + h->Nz, Nz_global);
    if ((has_lo != 0) != (i0 > 0) || (has_hi != 0) != (i0 + h->Nz < Nz_global))
        return h->fail(FDTD_ERR_ARG, "slab neighbours do not match its place in the grid");
    h->slab = 1;
    h->slab_i0 = i0;
    h->slab_Nz = Nz_global;
    h->slab_lo = has_lo ? 1 : 0;
    h->slab_hi = has_hi ? 1 : 0;
    for (int c = 0; c < 4; c++) h->slab_zhalo[c] = nullptr;   // the slab's own halo planes
    return FDTD_OK;
}

extern "C" int FDTD_slab_begin(FDTDHandle* h, const FDTDSolveOptions* o, const long long* cells,
                               int npoints) {
    if (!h || !o) return FDTD_ERR_ARG;
    if (!h->slab) return h->fail(FDTD_ERR_ARG, "FDTD_slab_begin: the handle is not a slab (FDTD_slab_set)");
    if (h->ready() != FDTD_OK) return h->status;
    if (!h->whole_grid()) return h->fail(FDTD_ERR_ARG, "a slab handle's local grid must be its whole grid");
    if (o->Tn <= 0 || npoints < 0 || (npoints > 0 && !cells)) return h->fail(FDTD_ERR_ARG, "bad slab options");
    for (int a = 0; a < 3; a++)
        if (h->bc[a] != '0' && h->bc[a] != 'E' && h->bc[a] != 'H')
            return h->fail(FDTD_ERR_ARG, "periodic boundaries are not supported in slabs");
    if ((long long)(h->Nz + 2) * h->Ny * ((h->Nx + 31) / 32 * 32) >= (1LL << 31) ||
        (long long)h->Nz * h->Ny * (h->w[0] + h->w[1]) >= (1LL << 31))
        return h->fail(FDTD_ERR_ARG, "slab too large for 32-bit cell offsets");
    std::memset(&h->slab_src32, 0, sizeof(h->slab_src32));
    std::memset(&h->slab_src64, 0, sizeof(h->slab_src64));
    int rc = h->precision == 32 ? slab_begin_impl<float>(h, o, cells, npoints)
                                : slab_begin_impl<double>(h, o, cells, npoints);
    if (rc == FDTD_OK) { h->status = FDTD_OK; h->message.clear(); }
    return rc;
}

extern "C" int FDTD_slab_step(FDTDHandle* h, long long n, int half) {
    return FDTD_slab_step_part(h, n, half, 0);
}

extern "C" int FDTD_slab_step_part(FDTDHandle* h, long long n, int half, int part) {
    if (!slab_ready(h) || (half != 0 && half != 1) || n < 0 || n >= (1LL << 31) || part < 0 || part > 2)
        return h ? h->fail(FDTD_ERR_ARG, "FDTD_slab_step_part: no slab begun, or bad step or part")
                 : FDTD_ERR_ARG;
    return h->precision == 32 ? slab_step_impl<float>(h, n, half, part)
                              : slab_step_impl<double>(h, n, half, part);
}

// The half steps read the step table at (device step base) + n; the base is
// 0 except while a caller replays steps captured with n = 0 .. K - 1 (a CUDA
// graph): it then sets the base to the first step of the replay.
extern "C" int FDTD_slab_set_step(FDTDHandle* h, long long base) {
    if (!slab_ready(h) || base < 0 || base >= (1LL << 31))
        return h ? h->fail(FDTD_ERR_ARG, "FDTD_slab_set_step: no slab begun, or bad step") : FDTD_ERR_ARG;
    long long* sb = h->precision == 32 ? dptr<long long>(h->r32.stepbase) : dptr<long long>(h->r64.stepbase);
    fdtdb::launch_set_ll(sb, base, h->stream);
    CK(cudaGetLastError());
    return FDTD_OK;
}

extern "C" int FDTD_slab_set_halo_source(FDTDHandle* h, void* const* ptrs) {
    if (!h || !ptrs) return h ? h->fail(FDTD_ERR_ARG, "FDTD_slab_set_halo_source: null argument") : FDTD_ERR_ARG;
    if (!h->slab) return h->fail(FDTD_ERR_ARG, "FDTD_slab_set_halo_source: not a slab (FDTD_slab_set)");
    if ((ptrs[0] || ptrs[1]) && !h->slab_hi)
        return h->fail(FDTD_ERR_ARG, "FDTD_slab_set_halo_source: no slab above to read from");
    if ((ptrs[2] || ptrs[3]) && !h->slab_lo)
        return h->fail(FDTD_ERR_ARG, "FDTD_slab_set_halo_source: no slab below to read from");
    for (int c = 0; c < 4; c++) h->slab_zhalo[c] = ptrs[c];
    return FDTD_OK;
}

extern "C" int FDTD_slab_halo(FDTDHandle* h, void** ptrs, long long* plane_elems) {
    if (!slab_ready(h) || !ptrs || !plane_elems)
        return h ? h->fail(FDTD_ERR_ARG, "FDTD_slab_halo: no slab begun") : FDTD_ERR_ARG;
    return h->precision == 32 ? slab_halo_impl<float>(h, ptrs, plane_elems)
                              : slab_halo_impl<double>(h, ptrs, plane_elems);
}

extern "C" int FDTD_slab_sample(FDTDHandle* h, void** samples) {
    if (!slab_ready(h) || !samples)
        return h ? h->fail(FDTD_ERR_ARG, "FDTD_slab_sample: no slab begun") : FDTD_ERR_ARG;
    return h->precision == 32 ? slab_sample_impl<float>(h, samples) : slab_sample_impl<double>(h, samples);
}

extern "C" int FDTD_slab_probe(FDTDHandle* h, long long n_last, double* A_change, double* phi_change) {
    if (!slab_ready(h) || !A_change || !phi_change || n_last < 0 || n_last >= (1LL << 31))
        return h ? h->fail(FDTD_ERR_ARG, "FDTD_slab_probe: no slab begun, or bad step") : FDTD_ERR_ARG;
    return h->precision == 32 ? slab_probe_impl<float>(h, n_last, A_change, phi_change)
                              : slab_probe_impl<double>(h, n_last, A_change, phi_change);
}

extern "C" int FDTD_slab_capture(FDTDHandle* h, int which) {
    if (!slab_ready(h) || (which != 0 && which != 1))
        return h ? h->fail(FDTD_ERR_ARG, "FDTD_slab_capture: no slab begun, or bad snapshot") : FDTD_ERR_ARG;
    return h->precision == 32 ? slab_capture_impl<float>(h, which) : slab_capture_impl<double>(h, which);
}

extern "C" int FDTD_slab_finish(FDTDHandle* h, long long n0, long long Tn) {
    if (!slab_ready(h) || n0 < 0 || Tn <= 0)
        return h ? h->fail(FDTD_ERR_ARG, "FDTD_slab_finish: no slab begun, or bad times") : FDTD_ERR_ARG;
    int rc = h->precision == 32 ? slab_finish_impl<float>(h, n0, Tn) : slab_finish_impl<double>(h, n0, Tn);
    if (rc == FDTD_OK) { h->status = FDTD_OK; h->message.clear(); }
    return rc;
}
