// probe_body.cuh -- the convergence probe of the CW loop, one CTA.
//
// Window shift and per-point refit follow emopt/fdtd.py:1072-1121: each probe
// point keeps the last three samples of Ex, Ey, Ez; the 3-sample phase and
// amplitude fits (common.cuh) are folded (negative amplitude -> +pi) and summed
// over the components.  The change norms ||A1 - A0|| / ||A0|| and
// ||phi1 - phi0|| / ||phi0|| (:1137-1138) are reduced with warp shuffles, then
// across warps in shared memory, into pd.out[0..1]; pd.out[2] counts probes.
// `nprobe` is the index of the last time step taken (its time is nprobe dt).
// With pd.samples set the new samples are read from there (the probe values
// gathered from all slabs of a distributed solve) instead of from E.
#pragma once

#include "kernels.h"

namespace fdtdb {

__device__ __forceinline__ double probe_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Called by every thread of a CTA of up to 256 threads.
template <typename T>
__device__ __forceinline__ void probe_block(const T* Ex, const T* Ey, const T* Ez, const ProbeDev& pd,
                                            long long nprobe, double dt) {
    __shared__ double red[4][8];
    __shared__ double tt[3];
    if (threadIdx.x == 0) {
        pd.times[0] = pd.times[1];
        pd.times[1] = pd.times[2];
        pd.times[2] = (double)nprobe * dt;
        tt[0] = pd.times[0]; tt[1] = pd.times[1]; tt[2] = pd.times[2];
    }
    __syncthreads();
    double sdA = 0, sA0 = 0, sdP = 0, sP0 = 0;
    const T* E[3] = {Ex, Ey, Ez};
    for (int q = threadIdx.x; q < pd.nconv; q += blockDim.x) {
        double phi0 = pd.phi[pd.nconv + q], A0 = pd.A[pd.nconv + q];
        long long off = pd.map[q];
        double phs = 0, amps = 0;
        double ph[3], am[3];
        for (int c = 0; c < 3; c++) {
            double* w = pd.win + (long long)c * 3 * pd.nconv;
            double w0 = w[pd.nconv + q], w1 = w[2 * pd.nconv + q];
            double w2 = pd.samples ? pd.samples[(long long)c * pd.nconv + q]
                                   : (off >= 0 ? (double)E[c][off] : 0.0);
            w[q] = w0; w[pd.nconv + q] = w1; w[2 * pd.nconv + q] = w2;
            double f = phase_3t(tt[0], tt[1], tt[2], w0, w1, w2);
            double a = amplitude_3t(tt[0], tt[1], tt[2], w0, w1, w2, f);
            if (a < 0) { a *= -1; f += M_PI; }
            ph[c] = f; am[c] = a;
        }
        phs = ph[0] + ph[1] + ph[2];
        amps = am[0] + am[1] + am[2];
        pd.phi[q] = phi0; pd.A[q] = A0;
        pd.phi[pd.nconv + q] = phs; pd.A[pd.nconv + q] = amps;
        double dA = amps - A0, dP = phs - phi0;
        sdA += dA * dA; sA0 += A0 * A0; sdP += dP * dP; sP0 += phi0 * phi0;
    }
    sdA = probe_warp_sum(sdA); sA0 = probe_warp_sum(sA0);
    sdP = probe_warp_sum(sdP); sP0 = probe_warp_sum(sP0);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { red[0][wid] = sdA; red[1][wid] = sA0; red[2][wid] = sdP; red[3][wid] = sP0; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s[4] = {0, 0, 0, 0};
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            for (int r = 0; r < 4; r++) s[r] += red[r][w];
        pd.out[0] = sqrt(s[0]) / sqrt(s[1]);
        pd.out[1] = sqrt(s[2]) / sqrt(s[3]);
        pd.out[2] = pd.out[2] + 1.0;
    }
    __syncthreads();
}

}  // namespace fdtdb
