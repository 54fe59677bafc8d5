// Fixed device scratch for the allocation-free IDEL2LN entry point
// (mlegs_idel2ln_static in ctx.cu).
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// solve, e.g. a host code whose own pool allocator has already reserved the
// device memory it is allowed to use, or a time loop that cannot afford
// cudaMalloc's implicit device-wide synchronisation.  The banded solve keeps
// its U rows in global scratch (NRCHOPDIM * 4 * NTCHOPDIM * NXCHOPDIM
// doubles); here that scratch is a file-scope __device__ array, so the entry
// point allocates nothing.  The array costs kStaticSolveBytes on a device
// from the first call there (CUDA's lazy module loading, the default, loads
// this file's module at the symbol lookup; with eager loading it is held from
// library load) until the process exits.
//
// Set-up: the first call on a device, with that device current, asks the
// runtime for the array's device address (cudaGetSymbolAddress) and caches it
// per device; that first call should therefore come before any stream
// capture.  The cache assumes the device's primary context lives until the
// process exits: after a cudaDeviceReset the module reloads elsewhere and the
// cached address would be stale, so hosts that reset a device must not call
// the entry point again.  `g_static_solve_scr` below is a host-side stand-in
// for the symbol; only the cached address is ever handed to a kernel.
//
// Sharing: every call on a device uses the same array, which keeps the last
// call's contents.  No entry has to start at zero: each (m, k) system writes
// every scratch entry it later reads within the same launch.  Calls whose
// kernels overlap on the GPU (two streams, or two contexts on one device)
// race on the array and must be ordered by the caller.
#include <cstdio>
#include <mutex>

#include "mlegs_internal.h"

namespace mlegs {

namespace {
constexpr size_t kStaticSolveDoubles = (size_t)8 << 20;  // 8,388,608 doubles
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_static_solve_scr[kStaticSolveDoubles];

std::mutex g_static_mu;
double* g_static_ptr[kMaxDevices] = {};
}  // namespace

const size_t kStaticSolveBytes = kStaticSolveDoubles * sizeof(double);

int static_solve_scratch(int device, size_t need_doubles, double** out, char* msg, size_t msg_len) {
    *out = nullptr;
    if (need_doubles > kStaticSolveDoubles) {
        snprintf(msg, msg_len,
                 "IDEL2LN (static scratch): the grid needs %zu bytes of solve scratch, above the fixed %zu bytes",
                 need_doubles * sizeof(double), kStaticSolveBytes);
        return 1;
    }
    if (device < 0 || device >= kMaxDevices) {
        snprintf(msg, msg_len, "IDEL2LN (static scratch): device %d outside 0..%d", device, kMaxDevices - 1);
        return 1;
    }
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[device]) {
        int cur = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e == cudaSuccess && cur != device) e = cudaErrorInvalidDevice;
        void* p = nullptr;
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_static_solve_scr);
        if (e != cudaSuccess) {
            snprintf(msg, msg_len, "IDEL2LN (static scratch): cudaGetSymbolAddress on device %d: %s", device,
                     cudaGetErrorString(e));
            return 2;
        }
        g_static_ptr[device] = (double*)p;
    }
    *out = g_static_ptr[device];
    return 0;
}

}  // namespace mlegs
