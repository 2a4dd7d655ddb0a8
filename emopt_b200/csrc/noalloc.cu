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
// Set-up: the first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current), which also loads the
// library's device code on that device if nothing else has.  Make that first
// call before any stream capture.
//
// Sharing: every call on a device uses the same array, and it keeps the last
// call's contents.  The conversion reads only the n values that the call
// itself copied in, so nothing needs clearing between calls.  Calls that
// overlap in time on the same device (two host threads) race on the array and
// corrupt each other's results; serialise them.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/emopt_fdtd.h"
#include "kernels.h"

constexpr long long kScratchBytes = 8ll << 20;  // 8 MiB = FDTD_NOALLOC_MAX_VALUES complex128
static_assert(kScratchBytes == FDTD_NOALLOC_MAX_VALUES * 16ll, "scratch size and header disagree");

// The staging array.  Host code never uses its name as a device address: it
// asks the runtime for the address on each device (scratch_address below).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_lock;
void* g_addr[kMaxDevices] = {};

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

// Device address of g_scratch on the current device `dev`, looked up once.
cudaError_t scratch_address(int dev, void** out) {
    std::lock_guard<std::mutex> g(g_lock);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return cudaSuccess;
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
    if (device < 0 || device >= ndev || device >= kMaxDevices)
        return fail(msg, msglen, FDTD_ERR_ARG, "FDTD_amp_phase_noalloc: device %d not in [0, %d)",
                    device, ndev < kMaxDevices ? ndev : kMaxDevices);
    if (n == 0) return FDTD_OK;

    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != device) e = cudaSetDevice(device);
    void* p = nullptr;
    if (e == cudaSuccess) e = scratch_address(device, &p);
    cudaStream_t st = stream ? (cudaStream_t)stream : cudaStreamPerThread;
    const size_t bytes = sizeof(fdtd_complex128) * (size_t)n;
    const char* where = "set-up";
    if (e == cudaSuccess) {
        where = "copy to device";
        e = cudaMemcpyAsync(p, a, bytes, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) {
        where = "kernel";
        fdtdb::launch_amp_phase(reinterpret_cast<fdtdb::c128*>(p), n, st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        where = "copy to host";
        e = cudaMemcpyAsync(a, p, bytes, cudaMemcpyDeviceToHost, st);
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
