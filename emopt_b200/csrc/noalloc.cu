// noalloc.cu -- FDTD_amp_phase_noalloc: the amplitude/phase rewrite of
// FDTD_add_source(..., calc_phase = true) without any device allocation.
//
// FDTD_add_source stages each source component through a temporary device
// buffer (cudaMalloc, then cudaFree).  Some callers cannot allocate there:
//   * a process whose device memory is already committed -- a framework pool
//     such as torch's caching allocator holding the free memory, or other
//     solves' resident fields filling HBM -- where cudaMalloc fails;
//   * a host thread preparing the sources of the next solve while solves run
//     on other streams of the same device: cudaFree waits for all work on the
//     device, so it would stall those solves until they finish.
// This entry point stages through one fixed array in device global memory
// instead, reserved when the library's device code is loaded on a device and
// held by every GPU that loads the library until the process exits.
//
// Set-up: every call looks up the array's device address on its device
// (cudaGetSymbolAddress, with that device current).  The first lookup on a
// device also loads the library's device code there if nothing else has, so
// make the first call before any stream capture.  Looking it up each time
// (cheap once the code is loaded) keeps the address right after a
// cudaDeviceReset, which reloads the code at another address.
//
// Sharing: every call on a device uses the same array, and it keeps the last
// call's contents.  The conversion reads only the n values that the call
// itself copied in, so nothing needs clearing between calls.  Calls that
// overlap in time on the same device (two host threads) race on the array and
// corrupt each other's results; serialise them.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>

#include "../../include/emopt_fdtd.h"
#include "kernels.h"

constexpr long long kScratchBytes = 8ll << 20;  // 8 MiB = FDTD_NOALLOC_MAX_VALUES complex128
static_assert(kScratchBytes == FDTD_NOALLOC_MAX_VALUES * 16ll, "scratch size and header disagree");

// The staging array.  Host code never uses its name as a device address: it
// asks the runtime for the array's address on the current device.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

namespace {

int fail(char* msg, int msglen, int status, const char* fmt, ...) __attribute__((format(printf, 4, 5)));
int fail(char* msg, int msglen, int status, const char* fmt, ...) {
    if (msg && msglen > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(msg, (size_t)msglen, fmt, ap);
        va_end(ap);
    }
    return status;
}

}  // namespace

extern "C" int FDTD_amp_phase_noalloc(int device, void* stream, fdtd_complex128* a, long long n,
                                      char* msg, int msglen) {
    if (msg && msglen > 0) msg[0] = '\0';
    if (n < 0 || (n > 0 && a == nullptr))
        return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_amp_phase_noalloc: invalid array (n=%lld)", n);
    if (n > FDTD_NOALLOC_MAX_VALUES)
        return fail(msg, msglen, FDTD_ERR_ARG,
                    "FDTD_amp_phase_noalloc: n=%lld values exceed the fixed scratch of %lld "
                    "complex128 values (%lld bytes); convert in pieces of at most that size",
                    n, (long long)FDTD_NOALLOC_MAX_VALUES, kScratchBytes);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(msg, msglen, FDTD_ERR_NODEVICE, "FDTD_amp_phase_noalloc: no CUDA device");
    }
    if (device < 0 || device >= ndev)
        return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_amp_phase_noalloc: device %d not in [0, %d)",
                    device, ndev);
    if (n == 0) return FDTD_OK;

    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != device) e = cudaSetDevice(device);
    void* p = nullptr;
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_scratch);
    cudaStream_t st = stream ? (cudaStream_t)stream : cudaStreamPerThread;
    const size_t bytes = sizeof(fdtd_complex128) * (size_t)n;
    const char* where = "set-up";
    if (e == cudaSuccess) {
        where = "copy to device";
        e = cudaMemcpyAsync(p, a, bytes, cudaMemcpyDefault, st);
    }
    if (e == cudaSuccess) {
        where = "kernel";
        cudaGetLastError();   // an error left by an earlier call is not this launch's
        fdtdb::launch_amp_phase(reinterpret_cast<fdtdb::c128*>(p), n, st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        where = "copy to host";
        e = cudaMemcpyAsync(a, p, bytes, cudaMemcpyDefault, st);
    }
    if (e == cudaSuccess) {
        where = "synchronize";
        e = cudaStreamSynchronize(st);
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess)
        return fail(msg, msglen, FDTD_ERR_CUDA, "FDTD_amp_phase_noalloc: %s: %s", where,
                    cudaGetErrorString(e));
    return FDTD_OK;
}
