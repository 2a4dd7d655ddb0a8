// serve_kernels.cu -- kernels that advance a batch of independent CW solves.
//
// Every active request (a whole CW solve of its own grid, wavelength and
// sources) has a view of its resident state (ServeView: grid view, field
// pointers, sources) and a control block (ServeCtl: time step, loop state,
// probe buffers) in device tables of fixed capacity.  One time step of the
// whole batch is four launches with fixed shapes, so one CUDA graph of L steps
// serves however requests come and go (only the tables change):
//   k_serve_step (H, then E) -- persistent single-warp CTAs, one resident wave,
//       split the task list that concatenates every request's warp tasks (one
//       task = 32 vectors of one row of one plane, the unit of the vector
//       kernels, vec_body.cuh) into contiguous chunks; a CTA finds the request
//       of its first task by binary search over the prefix table and walks
//       its chunk in order (77 / 86 us for H / E on a 5.2 M-cell request, 20%
//       above the single-solve kernels, against 83 / 91 us for one CTA per
//       task);
//   k_serve_events -- one CTA per slot: advances the request's step counter
//       and runs its part of the reference loop (emopt/fdtd.py:1016-1194) on
//       the device: a probe every Tn steps with the convergence test
//       (probe_body.cuh), the tail run up to floor(Nmax), then the t0 capture,
//       the t1 capture Tn steps later and the stop at n0 + 2 Tn;
//   k_serve_capture -- copies the fields of every request that asked for a
//       capture in this step into its snapshot set (all CTAs share the copy);
//       it returns at once in the usual step with no capture (a per-step count
//       that the events kernel raises and the H kernel clears).
// Requests that finished are skipped until the host retires them and runs
// the 3-sample extraction.  The step counts and probe decisions are those of
// FDTD_solve_cw for the same request.
#include "kernels.h"
#include "probe_body.cuh"
#include "vec_body.cuh"

namespace fdtdb {

namespace {

__device__ __forceinline__ int find_slot(const long long* __restrict__ task0, int nslots, long long t) {
    int lo = 0, hi = nslots;   // largest lo with task0[lo] <= t
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (task0[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// float32 bodies are held to 24 resident CTAs per SM (80 registers instead
// of 92-96: +4-8% aggregate throughput); float64 keeps its own allocation.
template <typename T, bool IS_E>
__global__ void __launch_bounds__(32, sizeof(T) == 4 ? 24 : 0) k_serve_step(const ServeView<T>* __restrict__ views,
                                                   const ServeCtl* __restrict__ ctl,
                                                   const long long* __restrict__ task0, int nslots,
                                                   int* cap_count) {
    // the view of the request being walked, copied once per request segment:
    // its parameters are then read from shared memory inside the task loop
    // (7% more aggregate throughput on a 16-request mix than reading them
    // from the global table)
    __shared__ __align__(16) unsigned char sv_raw[sizeof(ServeView<T>)];
    static_assert(sizeof(ServeView<T>) % 8 == 0 && alignof(ServeView<T>) >= 8, "view copy by 8-byte words");
    if (!IS_E && blockIdx.x == 0 && threadIdx.x == 0) *cap_count = 0;
    // CTA b takes one contiguous chunk of the task list, so the request of a
    // task is looked up once per request segment and (plane, row, block) are
    // walked by increments.
    const long long total = task0[nslots];
    const long long chunk = (total + gridDim.x - 1) / gridDim.x;
    long long t = (long long)blockIdx.x * chunk;
    const long long tend = min(total, t + chunk);
    if (t >= tend) return;
    int r = find_slot(task0, nslots, t);
    while (t < tend && r < nslots) {
        const long long rend = min(tend, task0[r + 1]);
        const int st = ctl[r].state;
        if (rend > t && st != SERVE_FREE && st != SERVE_DONE) {
            {
                const int2* a = reinterpret_cast<const int2*>(&views[r]);
                int2* b = reinterpret_cast<int2*>(sv_raw);
                for (int q = threadIdx.x; q < (int)(sizeof(ServeView<T>) / 8); q += 32) b[q] = a[q];
                __syncwarp();
            }
            const ServeView<T>& v = *reinterpret_cast<const ServeView<T>*>(sv_raw);
            const long long nxb = v.nxb;
            const int Ny = v.g.Ny;
            const long long local = t - task0[r];
            const long long row = local / nxb;
            int xb = (int)(local - row * nxb);
            int i = (int)(row / Ny);
            int j = (int)(row - (long long)i * Ny);
            for (; t < rend; t++) {
                if (IS_E) vec_update_E<T>(v.g, v.f, v.src, &ctl[r].n, 0, i, j, xb, threadIdx.x);
                else vec_update_H<T>(v.g, v.f, v.src, &ctl[r].n, 0, i, j, xb, threadIdx.x);
                if (++xb == nxb) {
                    xb = 0;
                    if (++j == Ny) { j = 0; ++i; }
                }
            }
        }
        __syncwarp();   // every lane is done with the view before the next copy
        t = rend > t ? rend : t;
        ++r;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_serve_events(const ServeView<T>* __restrict__ views,
                                                      ServeCtl* ctl, int nslots, int* cap_count) {
    const int r = blockIdx.x;
    if (r >= nslots) return;
    ServeCtl& c = ctl[r];
    const int state = c.state;
    if (state == SERVE_FREE || state == SERVE_DONE) return;
    const long long n = c.n + 1;   // steps taken after this one
    if (state == SERVE_RUN && n % c.Tn == 0) {
        const ServeView<T>& v = views[r];
        probe_block<T>(v.f.c[0], v.f.c[1], v.f.c[2], c.pd, n - 1, c.dt);
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
            if (next == SERVE_EXTRACT) { c.n0 = n; c.capture = 1; atomicAdd(cap_count, 1); }
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
    if (capture) atomicAdd(cap_count, 1);
    c.n = n;
}

template <typename T>
__global__ void __launch_bounds__(256) k_serve_capture(const ServeView<T>* __restrict__ views,
                                                       const ServeCtl* __restrict__ ctl, int nslots,
                                                       const int* cap_count) {
    if (*cap_count == 0) return;   // nothing to capture in this step (the usual case)
    for (int r = 0; r < nslots; r++) {
        const int cap = ctl[r].capture;
        if (cap == 0 || ctl[r].state == SERVE_FREE) continue;
        const ServeView<T>& v = views[r];
        const long long cells = (long long)v.g.Nz * v.g.Ny * v.g.px;
        for (int comp = 0; comp < 6; comp++) {
            const T* src = v.f.c[comp];
            T* dst = v.snap[cap - 1][comp];
            for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < cells;
                 q += (long long)gridDim.x * blockDim.x)
                dst[q] = src[q];
        }
    }
}

}  // namespace

template <typename T>
int serve_step_ctas_per_sm() {
    int a = 0, b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_serve_step<T, false>, 32, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_serve_step<T, true>, 32, 0) != cudaSuccess) {
        cudaGetLastError();
        return 16;
    }
    const int m = a < b ? a : b;
    return m > 0 ? m : 1;
}

template <typename T>
cudaError_t launch_serve_step(const ServeView<T>* views, ServeCtl* ctl, const long long* task0,
                              int nslots, long long step_ctas, int copy_ctas, int* cap_count,
                              cudaStream_t st) {
    const unsigned g = (unsigned)(step_ctas > 0 ? step_ctas : 1);
    k_serve_step<T, false><<<g, 32, 0, st>>>(views, ctl, task0, nslots, cap_count);
    k_serve_step<T, true><<<g, 32, 0, st>>>(views, ctl, task0, nslots, cap_count);
    k_serve_events<T><<<nslots, 256, 0, st>>>(views, ctl, nslots, cap_count);
    k_serve_capture<T><<<copy_ctas, 256, 0, st>>>(views, ctl, nslots, cap_count);
    return cudaGetLastError();
}

template int serve_step_ctas_per_sm<float>();
template int serve_step_ctas_per_sm<double>();
template cudaError_t launch_serve_step<float>(const ServeView<float>*, ServeCtl*, const long long*,
                                              int, long long, int, int*, cudaStream_t);
template cudaError_t launch_serve_step<double>(const ServeView<double>*, ServeCtl*,
                                               const long long*, int, long long, int, int*,
                                               cudaStream_t);

}  // namespace fdtdb
