// serve_kernels.cu -- kernels that advance a batch of independent CW solves.
//
// Every active request (a whole CW solve of its own grid, wavelength and
// sources) is a chain of launches of its own: per time step its H and E half
// steps and its events kernel.  The half steps are the single-solve vector
// kernels' (vec_body.cuh, one single-warp CTA per 32-vector row segment, in
// plane order), with the request's grid view, fields and sources in the
// kernel parameters; the engine captures each admitted request's chain of L
// steps as a CUDA graph of its own and replays the active requests' graphs
// on their own streams, so the requests run side by side and each walks its
// own grid in order (the L2 reuse of the single-solve kernels).
//   k_serve_half (H, then E) -- the half step, gated by the request's loop
//       state (a finished request stores nothing until it is collected); in
//       a step that follows a capture event the H half step also writes the
//       six fields it read into the request's snapshot set;
//   k_serve_event -- one CTA: advances the request's step counter and runs its
//       part of the reference loop (emopt/fdtd.py:1016-1194) on the device: a
//       probe every Tn steps with the convergence test (probe_body.cuh), the
//       tail run up to floor(Nmax), then the t0 capture, the t1 capture Tn
//       steps later and the stop at n0 + 2 Tn.
// Requests that finished stop stepping until the host retires them and runs
// the 3-sample extraction.  The step counts and probe decisions are those of
// FDTD_solve_cw for the same request.
#include "kernels.h"
#include "probe_body.cuh"
#include "vec_body.cuh"

namespace fdtdb {

namespace {

// The single-solve kernels' register bounds (vec_kernels.cu): 64 registers in
// float32 for both half steps.
template <typename T, bool IS_E>
__global__ void __launch_bounds__(IS_E || sizeof(T) == 8 ? 32 : 256, sizeof(T) == 8 ? 18 : 0)
k_serve_half(GridView<T> g, Fields<T> f, SourceList<T> src, const __grid_constant__ ServeGate<T> sg,
             const long long* step_ctr) {
    const int i = (int)blockIdx.z, j = (int)blockIdx.y, xb = (int)blockIdx.x;
    if (sizeof(T) == 4 && vecb::plain_warp<T>(g, src, IS_E ? 0 : 3, i, j, xb)) {
        if (IS_E) vec_update_E<T, false, true>(g, f, src, step_ctr, 0, i, j, xb, threadIdx.x, &sg);
        else vec_update_H<T, false, true>(g, f, src, step_ctr, 0, i, j, xb, threadIdx.x, &sg);
    } else {
        if (IS_E) vec_update_E<T, true, true>(g, f, src, step_ctr, 0, i, j, xb, threadIdx.x, &sg);
        else vec_update_H<T, true, true>(g, f, src, step_ctr, 0, i, j, xb, threadIdx.x, &sg);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_serve_event(const T* Ex, const T* Ey, const T* Ez, ServeCtl* ctl) {
    ServeCtl& c = *ctl;
    const int state = c.state;
    if (state == SERVE_FREE || state == SERVE_DONE) return;
    const long long n = c.n + 1;   // steps taken after this one
    if (state == SERVE_RUN && n % c.Tn == 0) {
        probe_block<T>(Ex, Ey, Ez, c.pd, n - 1, c.dt);
        if (threadIdx.x == 0) {
            const double A = c.pd.out[0], P = c.pd.out[1];
            c.A_change = A;
            c.phi_change = P;
            c.nprobes += 1;
            const bool finite = !(isnan(A) || isinf(A) || isnan(P) || isinf(P));
            const bool converged = !c.fixed && finite && !(A > c.amp_tol) && !(P > c.phi_tol);
            int next = SERVE_RUN;
            if (converged || (c.stop_nf && !finite) || (double)n > (c.fixed ? (double)c.last : c.Nmax))
                next = SERVE_EXTRACT;
            else if (n + c.Tn - 1 > c.last) next = SERVE_TAIL;
            if (next == SERVE_EXTRACT) { c.n0 = n; c.capture = 1; }
            else c.capture = 0;
            c.state = next;
            c.n = n;
        }
        return;
    }
    if (threadIdx.x != 0) return;
    int capture = 0;
    if (state == SERVE_TAIL && n == c.last + 1) {
        c.state = SERVE_EXTRACT;
        c.n0 = n;
        capture = 1;
    } else if (state == SERVE_EXTRACT) {
        if (n == c.n0 + c.Tn) capture = 2;
        if (n == c.n0 + 2 * c.Tn) c.state = SERVE_DONE;
    }
    c.capture = capture;
    c.n = n;
}

}  // namespace

template <typename T>
cudaError_t launch_serve_request_step(const ServeView<T>& v, ServeCtl* ctl, cudaStream_t st) {
    ServeGate<T> sg;
    sg.state = &ctl->state;
    sg.capture = &ctl->capture;
    for (int s = 0; s < 2; s++)
        for (int c = 0; c < 6; c++) sg.snap[s][c] = v.snap[s][c];
    dim3 grid((unsigned)v.nxb, (unsigned)v.g.Ny, (unsigned)v.g.Nz);
    k_serve_half<T, false><<<grid, 32, 0, st>>>(v.g, v.f, v.src, sg, &ctl->n);
    k_serve_half<T, true><<<grid, 32, 0, st>>>(v.g, v.f, v.src, sg, &ctl->n);
    k_serve_event<T><<<1, 256, 0, st>>>(v.f.c[0], v.f.c[1], v.f.c[2], ctl);
    return cudaGetLastError();
}

template cudaError_t launch_serve_request_step<float>(const ServeView<float>&, ServeCtl*, cudaStream_t);
template cudaError_t launch_serve_request_step<double>(const ServeView<double>&, ServeCtl*, cudaStream_t);

}  // namespace fdtdb
