// Allocation-free entry point for the projected eigenproblem.
//
// Some callers cannot call cudaMalloc at the point where they need this
// solve: code running while a CUDA stream is being captured into a graph
// (allocation is not a capturable operation), real-time loops that must not
// touch the allocator, or hosts whose device memory is owned by another
// allocator.  For them the Jacobi eigensolver's workspace lives in a
// file-scope device array instead of memory allocated per call.  The caller
// passes the input and output buffers; nothing here allocates.
#include "krylov.cuh"
#include "../counters.h"
#include "../../../include/speigs_b200.h"

#include <cstdio>
#include <mutex>

namespace spx {
const char *set_last_error_text(const char *msg);
}

namespace {

// Largest projected matrix this entry point accepts.
constexpr int kNoAllocMaxM = 256;
constexpr size_t kNoAllocWorkDoubles = 2ull * kNoAllocMaxM * kNoAllocMaxM;

// Workspace of the Jacobi sweeps (two m x m matrices) plus a status word.
// Every GPU that loads the library holds these 1 MiB until the process exits;
// all calls share them.
static __device__ __align__(256) double g_syev_work[kNoAllocWorkDoubles + 32];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_work_addr[kMaxDevices] = {nullptr};

// Device address of the workspace on the current device.  The host-side name
// g_syev_work is only a stand-in for the device symbol, so the address is
// looked up with cudaGetSymbolAddress once per device, with that device
// current.
int work_address(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        spx::set_last_error_text("no current CUDA device");
        return SPEIGS_ERR_INTERNAL;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        spx::set_last_error_text("device ordinal beyond the no-allocation table");
        return SPEIGS_ERR_INTERNAL;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_work_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_syev_work);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            spx::set_last_error_text("cudaGetSymbolAddress of the eigensolver workspace failed");
            return SPEIGS_ERR_INTERNAL;
        }
        g_work_addr[dev] = (double *)p;
    }
    *out = g_work_addr[dev];
    return SPEIGS_OK;
}

}  // namespace

extern "C" int speigs_b200_syev_small_noalloc(int m, const double *H, double *theta, double *S,
                                              int *ord, int *status, void *stream) {
    if (m < 1 || m > kNoAllocMaxM) {
        char msg[128];
        snprintf(msg, sizeof msg, "m = %d is outside 1..%d, the range of the no-allocation "
                 "eigensolver", m, kNoAllocMaxM);
        spx::set_last_error_text(msg);
        return SPEIGS_ERR_ARG;
    }
    if (!H || !theta || !S || !ord) {
        spx::set_last_error_text("null buffer passed to the no-allocation eigensolver");
        return SPEIGS_ERR_ARG;
    }
    double *work = nullptr;
    int rc = work_address(&work);
    if (rc) return rc;
    // the status word sits after the two matrices unless the caller wants it
    int *st = status ? status : (int *)(work + kNoAllocWorkDoubles);
    cudaStream_t cs = (cudaStream_t)stream;
    // An error left pending by earlier, unrelated CUDA work on this thread
    // would be read back below as this launch's failure; report it as what
    // it is, leave it pending for its owner, and launch nothing.
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        char msg[192];
        snprintf(msg, sizeof msg, "a CUDA error from earlier work is pending (%s); nothing was "
                 "launched", cudaGetErrorString(e));
        spx::set_last_error_text(msg);
        return SPEIGS_ERR_INTERNAL;
    }
    // the workspace is fully rewritten from H by the kernel: no clearing needed
    spx::launch_syev_small_workspace(m, H, m, theta, S, ord, work, st, cs);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        spx::set_last_error_text(cudaGetErrorString(e));
        return SPEIGS_ERR_INTERNAL;
    }
    return SPEIGS_OK;
}
