// serve_engine.cuh -- FDTD_serve_*: continuous batching of CW solves.
//
// Included at the end of fdtd_abi.cu: it reuses the handle's resident state
// (Resident<float>, prepare_materials, prepare_sources, make_view) so that an
// admitted request is set up exactly as FDTD_solve_cw would set it up, and its
// result is extracted exactly as FDTD_solve_cw extracts it.
//
// A request is a configured handle plus its solve options.  Admission checks
// the engine's device-memory budget and a free slot, allocates and prepares
// the request's resident state, enters it into the slot tables and captures
// its L time steps of launches (serve_kernels.cu) as a CUDA graph of its own;
// from the next replay on (FDTD_serve_advance) the request advances with all
// other active requests: every replay launches the active requests' graphs
// on their own streams, forked from the engine stream and joined back, so
// nothing is captured again when other requests come or go.  A request
// whose loop ended (converged, step budget or fixed length) stops stepping on
// its own; FDTD_serve_collect extracts its complex fields into the handle's t0
// arrays, fills its result and frees its memory.  Admission and collection
// happen between replays, so requests come and go while others run.

struct FDTDServe {
    int device = 0;
    cudaStream_t stream = nullptr;
    double budget = 0, used = 0;
    int cap = 0, L = 0;
    fdtdb::ServeCtl* d_ctl = nullptr;
    fdtdb::ServeCtl* h_ctl = nullptr;          // pinned mirror
    std::vector<fdtdb::ServeView<float>> views;
    std::vector<FDTDHandle*> slot_h;
    std::vector<double> slot_bytes;
    std::vector<long long> admitted_step;      // replay count at admission
    std::vector<cudaGraphExec_t> slot_exec;    // per admitted request: its L steps as one graph
    std::vector<cudaStream_t> aux;             // per slot: the stream its graph runs on
    std::vector<cudaEvent_t> join;             // per slot: end of its part of a replay
    cudaEvent_t fork = nullptr;                // start of a replay on the engine stream
    long long replays = 0;
    int status = FDTD_OK;
    std::string message;

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
        cudaGetLastError();
        return fail(FDTD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
};

namespace {

#define SCK(expr)                                                   \
    do {                                                            \
        cudaError_t e_ = (expr);                                    \
        if (e_ != cudaSuccess) return s->cuda_fail(e_, #expr);      \
    } while (0)

// Device bytes a request will hold (the arrays alloc_resident, prepare_* and
// the step table allocate for it), used before admission.
double serve_estimate(const FDTDHandle* h, long long max_steps) {
    const double px = (h->Nx + 31) / 32 * 32;
    const double cells = px * h->Ny * h->Nz, n = (double)h->Nx * h->Ny * h->Nz;
    const double slab = (double)h->Nz * h->Ny * (h->w[0] + h->w[1]) +
                        (double)h->Nz * (h->w[2] + h->w[3]) * px + (double)(h->w[4] + h->w[5]) * h->Ny * px;
    double b = 4.0 * cells * (6 + 3 + 12) + 4.0 * 4 * slab + 16.0 * n + 32.0 * max_steps;
    if (h->lossy) b += 4.0 * cells * 3;
    return b + (1 << 20);
}

template <typename T>
double resident_bytes(const Resident<T>& r) {
    double b = 0;
    for (auto& s : r.F) for (auto& x : s) b += x.bytes;
    for (int c = 0; c < 3; c++) b += r.bE[c].bytes + r.aE[c].bytes + r.bH[c].bytes;
    for (auto& s : r.psi) for (auto& a : s) for (auto& x : a) b += x.bytes;
    for (auto& s : r.snap) for (auto& x : s) b += x.bytes;
    for (auto& x : r.src_ap) b += x.bytes;
    for (auto& x : r.src_coef) b += x.bytes;
    b += r.stage.bytes + r.steptab.bytes + r.pwin.bytes + r.pA.bytes + r.pphi.bytes + r.ptimes.bytes +
         r.pout.bytes + r.pmap.bytes;
    return b;
}

// Slot q's L time steps of launches, captured once on the slot's stream.
int serve_capture_request(FDTDServe* s, int q) {
    if (!s->aux[q]) {
        SCK(cudaStreamCreateWithFlags(&s->aux[q], cudaStreamNonBlocking));
        SCK(cudaEventCreateWithFlags(&s->join[q], cudaEventDisableTiming));
    }
    SCK(cudaStreamBeginCapture(s->aux[q], cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int n = 0; n < s->L && e == cudaSuccess; n++)
        e = fdtdb::launch_serve_request_step<float>(s->views[q], s->d_ctl + q, s->aux[q]);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s->aux[q], &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return s->cuda_fail(e, "serve step capture");
    }
    if (e2 != cudaSuccess) return s->cuda_fail(e2, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&s->slot_exec[q], g, 0);
    cudaGraphDestroy(g);   // the executable graph holds what it needs
    if (e != cudaSuccess) {
        s->slot_exec[q] = nullptr;
        return s->cuda_fail(e, "cudaGraphInstantiate");
    }
    return FDTD_OK;
}

}  // namespace

extern "C" FDTDServe* FDTD_serve_new(int device, double budget_bytes, int max_requests,
                                     int steps_per_replay) {
    FDTDServe* s = new FDTDServe();
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        s->fail(FDTD_ERR_NODEVICE, "no CUDA device is visible");
        return s;
    }
    if (device < 0 || device >= ndev || max_requests <= 0 || steps_per_replay <= 0 || budget_bytes <= 0) {
        s->fail(FDTD_ERR_ARG, "bad engine parameters");
        return s;
    }
    s->device = device;
    s->budget = budget_bytes;
    s->cap = max_requests;
    s->L = steps_per_replay;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_ctl, sizeof(fdtdb::ServeCtl) * s->cap);
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_ctl, sizeof(fdtdb::ServeCtl) * s->cap);
    if (e != cudaSuccess) {
        s->cuda_fail(e, "FDTD_serve_new");
        return s;
    }
    s->views.assign(s->cap, fdtdb::ServeView<float>());
    s->slot_h.assign(s->cap, nullptr);
    s->slot_exec.assign(s->cap, nullptr);
    s->aux.assign(s->cap, nullptr);
    s->join.assign(s->cap, nullptr);
    s->slot_bytes.assign(s->cap, 0);
    s->admitted_step.assign(s->cap, 0);
    std::memset(s->h_ctl, 0, sizeof(fdtdb::ServeCtl) * s->cap);
    e = cudaMemcpyAsync(s->d_ctl, s->h_ctl, sizeof(fdtdb::ServeCtl) * s->cap, cudaMemcpyDefault, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) { s->cuda_fail(e, "FDTD_serve_new"); return s; }
    s->status = FDTD_OK;
    return s;
}

extern "C" int FDTD_serve_last_error(FDTDServe* s, char* buf, int buflen) {
    if (!s) return FDTD_ERR_ARG;
    if (buf && buflen > 0) snprintf(buf, (size_t)buflen, "%s", s->message.c_str());
    return s->status;
}

// Admit one request; returns its slot (>= 0), -1 when the budget or the slot
// table has no room for it now (retry after collecting), or -(status) on an
// error with the message in FDTD_serve_last_error.
extern "C" int FDTD_serve_admit(FDTDServe* s, FDTDHandle* h, const FDTDSolveOptions* o) {
    if (!s || !h || !o) return -FDTD_ERR_ARG;
    if (s->status != FDTD_OK && s->status != FDTD_ERR_ARG) return -s->status;
    auto bad = [&](const char* why) { s->fail(FDTD_ERR_ARG, "FDTD_serve_admit: %s", why); return -FDTD_ERR_ARG; };
    if (!h->whole_grid() || h->slab) return bad("the request's handle must hold the whole grid");
    for (int a = 0; a < 3; a++)
        if (h->bc[a] != '0' && h->bc[a] != 'E' && h->bc[a] != 'H') return bad("periodic boundaries are not served");
    if (h->precision != 32) return bad("served requests use float32 storage (FDTD_set_precision 32)");
    if (o->Tn <= 0 || (o->nconv > 0 && !o->conv_pts)) return bad("bad options");
    const bool fixed = o->fixed_steps > 0;
    const long long last = fixed ? o->fixed_steps - 1 : (long long)floor(o->Nmax);
    if (last < 0 || (!fixed && o->Nmax < 0)) return bad("the step budget is empty");
    const long long Tn = o->Tn;
    const long long max_steps = (last + 1) + 2 * Tn + Tn + 1;
    if ((long long)h->Nz * h->Ny * ((h->Nx + 31) / 32 * 32) >= (1LL << 31)) return bad("grid too large to serve");
    if (h->sources.size() > (size_t)fdtdb::kMaxSources) return bad("too many sources");
    for (int q = 0; q < s->cap; q++)
        if (s->slot_h[q] == h) return bad("handle already admitted");
    const double est = serve_estimate(h, max_steps);
    if (s->used + est > s->budget) return -1;
    int slot = -1;
    for (int q = 0; q < s->cap && slot < 0; q++)
        if (!s->slot_h[q]) slot = q;
    if (slot < 0) return -1;

    if (h->device < 0) h->device = s->device;
    if (h->device != s->device) return bad("the handle is bound to another device");
    if (h->ready() != FDTD_OK) {
        s->fail(h->status, "%s", h->message.c_str());
        return -h->status;
    }
    Resident<float>& r = h->r32;
    auto hfail = [&]() { s->fail(h->status, "%s", h->message.c_str()); r.release_all(); return -h->status; };
    if (alloc_resident<float>(h, r, false) != FDTD_OK) return hfail();
    if (prepare_materials<float>(h, r) != FDTD_OK) return hfail();
    fdtdb::SourceList<float> src;
    if (prepare_sources<float>(h, r, src) != FDTD_OK) return hfail();
    auto ck = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess) { h->cuda_fail(e, what); return false; }
        return true;
    };
    if (!ck(r.steptab.ensure(sizeof(double4) * max_steps), "steptab")) return hfail();
    fdtdb::launch_step_table(dptr<double4>(r.steptab), max_steps, h->dt, h->src_T, h->src_min,
                             h->src_k, h->stream);
    const size_t cells = (size_t)h->Nz * h->Ny * r.px;
    for (int c = 0; c < 6; c++)
        if (!ck(cudaMemsetAsync(r.F[0][c].p, 0, sizeof(float) * cells, h->stream), "zero fields")) return hfail();
    for (int a = 0; a < 3; a++)
        for (int q = 0; q < 4; q++)
            if (!ck(cudaMemsetAsync(r.psi[0][a][q].p, 0, r.psi[0][a][q].bytes, h->stream), "zero psi")) return hfail();
    const int nconv = o->nconv > 0 ? o->nconv : 0, nc = nconv > 0 ? nconv : 1;
    bool okb = ck(r.pwin.ensure(sizeof(double) * 9 * nc), "probe") && ck(r.pA.ensure(sizeof(double) * 2 * nc), "probe") &&
               ck(r.pphi.ensure(sizeof(double) * 2 * nc), "probe") && ck(r.ptimes.ensure(sizeof(double) * 3), "probe") &&
               ck(r.pout.ensure(sizeof(double) * 4), "probe") && ck(r.pmap.ensure(sizeof(long long) * nc), "probe");
    if (!okb) return hfail();
    okb = ck(cudaMemsetAsync(r.pwin.p, 0, r.pwin.bytes, h->stream), "probe") &&
          ck(cudaMemsetAsync(r.pA.p, 0, r.pA.bytes, h->stream), "probe") &&
          ck(cudaMemsetAsync(r.pphi.p, 0, r.pphi.bytes, h->stream), "probe") &&
          ck(cudaMemsetAsync(r.ptimes.p, 0, r.ptimes.bytes, h->stream), "probe") &&
          ck(cudaMemsetAsync(r.pout.p, 0, r.pout.bytes, h->stream), "probe") &&
          ck(cudaMemsetAsync(r.err.p, 0, r.err.bytes, h->stream), "status");
    if (!okb) return hfail();
    std::vector<long long> map((size_t)nc, -1);
    for (int q = 0; q < nconv; q++) map[q] = probe_offset(h, r.px, o->conv_pts[q]);
    if (!ck(cudaMemcpyAsync(r.pmap.p, map.data(), sizeof(long long) * nc, cudaMemcpyDefault, h->stream), "probe map")) return hfail();
    if (h->sync_check("FDTD_serve_admit") != FDTD_OK) return hfail();

    fdtdb::ServeView<float>& v = s->views[slot];
    std::memset(&v, 0, sizeof(v));
    v.g = make_view<float>(h, r);
    for (int c = 0; c < 6; c++) {
        v.f.c[c] = dptr<float>(r.F[0][c]);
        v.snap[0][c] = dptr<float>(r.snap[0][c]);
        v.snap[1][c] = dptr<float>(r.snap[1][c]);
    }
    v.src = src;
    v.nxb = ((h->Nx + 1) / 2 + 31) / 32;
    fdtdb::ServeCtl& c = s->h_ctl[slot];
    std::memset(&c, 0, sizeof(c));
    c.n = 0;
    c.Tn = Tn;
    c.last = last;
    c.Nmax = fixed ? (double)last : o->Nmax;
    c.amp_tol = o->rtol;
    c.phi_tol = sqrt(o->rtol);
    c.dt = h->dt;
    c.fixed = fixed ? 1 : 0;
    c.stop_nf = o->stop_nonfinite ? 1 : 0;
    c.pd.win = dptr<double>(r.pwin); c.pd.A = dptr<double>(r.pA); c.pd.phi = dptr<double>(r.pphi);
    c.pd.times = dptr<double>(r.ptimes); c.pd.out = dptr<double>(r.pout); c.pd.map = dptr<long long>(r.pmap);
    c.pd.nconv = nconv;
    c.A_change = 1;
    c.phi_change = 1;
    // first pass of the loop of emopt/fdtd.py:1016-1194 at n = 0
    c.state = (Tn - 1 > last) ? fdtdb::SERVE_TAIL : fdtdb::SERVE_RUN;
    SCK(cudaMemcpyAsync(s->d_ctl + slot, &c, sizeof(c), cudaMemcpyDefault, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    if (serve_capture_request(s, slot) != FDTD_OK) {
        r.release_all();
        return -s->status;
    }
    s->slot_h[slot] = h;
    s->slot_bytes[slot] = resident_bytes(r);
    s->used += s->slot_bytes[slot];
    s->admitted_step[slot] = s->replays;
    s->status = FDTD_OK;
    s->message.clear();
    return slot;
}

// One graph replay: every active request takes steps_per_replay time steps
// (or fewer, if its loop ends).  Returns the number of requests ready to be
// collected, or -(status) on an error.
extern "C" int FDTD_serve_advance(FDTDServe* s) {
    if (!s) return -FDTD_ERR_ARG;
    NvtxRange range("FDTD_serve_advance");
    if (!s->d_ctl) return -s->fail(FDTD_ERR_CUDA, "engine not initialised");
    SCK(cudaSetDevice(s->device));
    SCK(cudaEventRecord(s->fork, s->stream));
    for (int q = 0; q < s->cap; q++) {
        if (!s->slot_h[q] || !s->slot_exec[q]) continue;
        SCK(cudaStreamWaitEvent(s->aux[q], s->fork, 0));
        SCK(cudaGraphLaunch(s->slot_exec[q], s->aux[q]));
        SCK(cudaEventRecord(s->join[q], s->aux[q]));
        SCK(cudaStreamWaitEvent(s->stream, s->join[q], 0));
    }
    SCK(cudaMemcpyAsync(s->h_ctl, s->d_ctl, sizeof(fdtdb::ServeCtl) * s->cap, cudaMemcpyDefault, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    s->replays++;
    int done = 0;
    for (int q = 0; q < s->cap; q++)
        if (s->slot_h[q] && s->h_ctl[q].state == fdtdb::SERVE_DONE) done++;
    return done;
}

// Handles of up to `max` finished requests not yet collected; returns the count.
extern "C" int FDTD_serve_finished(FDTDServe* s, FDTDHandle** done, int max) {
    if (!s) return -FDTD_ERR_ARG;
    int k = 0;
    for (int q = 0; q < s->cap && k < max; q++)
        if (s->slot_h[q] && s->h_ctl[q].state == fdtdb::SERVE_DONE) done[k++] = s->slot_h[q];
    return k;
}

// Retire up to `max` finished requests: writes their complex fields into
// their handles' t0 arrays (3-sample extraction, as FDTD_solve_cw), fills
// res[k] and done[k], frees their device memory.  Returns the count.
extern "C" int FDTD_serve_collect(FDTDServe* s, FDTDHandle** done, FDTDSolveResult* res, int max) {
    if (!s) return -FDTD_ERR_ARG;
    SCK(cudaSetDevice(s->device));
    int k = 0;
    for (int q = 0; q < s->cap && k < max; q++) {
        FDTDHandle* h = s->slot_h[q];
        if (!h || s->h_ctl[q].state != fdtdb::SERVE_DONE) continue;
        const fdtdb::ServeCtl& c = s->h_ctl[q];
        Resident<float>& r = h->r32;
        const long long n0 = c.n0, Tn = c.Tn;
        const double t0 = (double)n0 * h->dt, t1 = (double)(n0 + Tn) * h->dt, t2 = (double)(n0 + 2 * Tn) * h->dt;
        fdtdb::Fit3 fE = fdtdb::make_fit3(t0, t1, t2);
        fdtdb::Fit3 fH = fdtdb::make_fit3(t0 - 0.5 * h->dt, t1 - 0.5 * h->dt, t2 - 0.5 * h->dt);
        const long long ncell = (long long)h->Nx * h->Ny * h->Nz;
        for (int comp = 0; comp < 6; comp++) {
            if (!h->ht0[comp]) return -s->fail(FDTD_ERR_ARG, "t0 arrays of a request are not set");
            fdtdb::launch_extract_3t<float>(dptr<float>(r.snap[0][comp]), dptr<float>(r.snap[1][comp]),
                                            dptr<float>(r.F[0][comp]), h->Nx, h->Ny, h->Nz, r.px,
                                            comp < 3 ? fE : fH, dptr<c128>(r.stage), s->stream);
            SCK(cudaGetLastError());
            SCK(cudaMemcpyAsync(h->ht0[comp], r.stage.p, sizeof(c128) * ncell, cudaMemcpyDefault, s->stream));
        }
#ifdef FDTD_BOUNDS_CHECK
        int kchk = 0;
        SCK(cudaMemcpyAsync(&kchk, dptr<int>(r.err) + 1, sizeof(int), cudaMemcpyDefault, s->stream));
#endif
        SCK(cudaStreamSynchronize(s->stream));
#ifdef FDTD_BOUNDS_CHECK
        if (kchk)
            return -s->fail(FDTD_ERR_CUDA, "bounds check: the stepping kernel computed an index outside its array (site %d)", kchk);
#endif
        FDTDSolveResult& o = res[k];
        std::memset(&o, 0, sizeof(o));
        o.n_main = n0;
        o.steps = n0 + 2 * Tn;
        o.A_change = c.A_change;
        o.phi_change = c.phi_change;
        o.nprobes = c.nprobes;
        o.launches = (s->replays - s->admitted_step[q]) * (long long)s->L * 3;
        o.status = FDTD_OK;
        if (!c.fixed) {
            const bool bad = std::isnan(c.A_change) || std::isinf(c.A_change) ||
                             std::isnan(c.phi_change) || std::isinf(c.phi_change);
            const bool conv = !bad && !(c.A_change > c.amp_tol) && !(c.phi_change > c.phi_tol);
            if (!conv) o.status = bad ? FDTD_NONFINITE : FDTD_NMAX;
        }
        done[k] = h;
        k++;
        // retire the slot
        s->h_ctl[q].state = fdtdb::SERVE_FREE;
        s->h_ctl[q].capture = 0;
        SCK(cudaMemcpyAsync(s->d_ctl + q, &s->h_ctl[q], sizeof(fdtdb::ServeCtl), cudaMemcpyDefault, s->stream));
        SCK(cudaStreamSynchronize(s->stream));
        if (s->slot_exec[q]) {
            cudaGraphExecDestroy(s->slot_exec[q]);
            s->slot_exec[q] = nullptr;
        }
        r.release_all();
        s->used -= s->slot_bytes[q];
        s->slot_bytes[q] = 0;
        s->slot_h[q] = nullptr;
    }
    return k;
}

// Device bytes in use by admitted requests and the number of admitted requests.
extern "C" int FDTD_serve_info(FDTDServe* s, double* used_bytes, int* active) {
    if (!s) return FDTD_ERR_ARG;
    int n = 0;
    for (int q = 0; q < s->cap; q++) n += s->slot_h[q] ? 1 : 0;
    if (used_bytes) *used_bytes = s->used;
    if (active) *active = n;
    return s->status;
}

extern "C" void FDTD_serve_delete(FDTDServe* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (int q = 0; q < s->cap; q++)
        if (s->slot_h[q]) s->slot_h[q]->r32.release_all();
    for (auto x : s->slot_exec) if (x) cudaGraphExecDestroy(x);
    for (auto b : s->aux) if (b) cudaStreamDestroy(b);
    for (auto ev : s->join) if (ev) cudaEventDestroy(ev);
    if (s->fork) cudaEventDestroy(s->fork);
    if (s->d_ctl) cudaFree(s->d_ctl);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

#undef SCK
