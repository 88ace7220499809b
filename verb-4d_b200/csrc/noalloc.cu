// Convection_2D on one slice in caller-owned device memory, allocating nothing.
//
// Some callers cannot allocate device memory at all: code that runs inside a
// host application which owns every device allocation (a memory pool or arena
// it manages), a plugin loaded by such an application, or code on a path where
// allocating would synchronise the device or is forbidden by policy.  They
// already hold their input and output arrays on the device.  For them this
// entry point runs the same convection kernel as verb_convection_2d, with the
// kernel's scratch (the slice's face Courant tables and its G, exp(Loss*dt)
// and Sources*dt planes, the work ticket, the sub-step count and the status
// word) placed in a fixed array of device memory that belongs to the
// library's device code.  CUDA loads that code on a device lazily (the default
// since CUDA 12.2): the first call on a device loads it, which is when the
// array and the kernel take their device memory and the device may
// synchronise.  A caller that must not allocate makes one warm-up call on each
// device before it enters the region where allocation is not allowed.
//
// Limits and sharing:
//  * P_size * R_size must not exceed VERB_NOALLOC_MAX_POINTS (8192 points,
//    5 doubles each: 320 KiB of scratch); larger slices are rejected with
//    VERB_ERR_SIZE, and so are lines longer than the kernel's 512 points.
//  * Every GPU that loads the library holds the array until the process exits.
//  * All calls share the one array and it keeps the last call's contents; the
//    entry point clears the ticket and status words on each call.  Calls whose
//    executions overlap on the GPU (different streams, or different host
//    threads) race on the array and must be serialised by the caller.
//  * The first call on a device looks up the array's device address (once per
//    device, with that device current).  Make that first call before any
//    stream capture begins.
//  * Errors: the call reports the device-side status of its slice
//    (VERB_ERR_CFL, ...) and an error of its own launch.  An error that the
//    caller's earlier CUDA work left pending in the runtime is neither
//    reported nor cleared here.
#include <cuda_runtime.h>

#include <mutex>

#include "verb_internal.cuh"

namespace {

constexpr int kMaxPoints = VERB_NOALLOC_MAX_POINTS;
constexpr int kPlaneDoubles = 5 * kMaxPoints;  // >= conv_scratch_doubles(P, R) for P*R <= kMaxPoints
constexpr int kWords = 8;  // ticket, sub-step count, status (+ padding)

// The scratch: kPlaneDoubles doubles for one CTA, then kWords ints.
static __device__ __align__(256) double g_noalloc_scratch[kPlaneDoubles + kWords];

constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of g_noalloc_scratch for the current device (host code must
// not pass the symbol itself to a kernel: in host code it is a host-side
// stand-in, not a device address).
int scratch_for_current_device(double** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return VERB_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return VERB_ERR_CUDA;
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return VERB_OK;
}

}  // namespace

extern "C" int verb_convection_2d_noalloc(double* psd, const double* P, const double* R, int nP,
                                          int nR, const double* pl, const double* pu,
                                          const double* rl, const double* ru, int pl_t, int pu_t,
                                          int rl_t, int ru_t, const double* VP, const double* VR,
                                          const double* S, const double* loss, const double* G,
                                          double dt, void* stream)
{
    if (!psd || !P || !R || !pl || !pu || !rl || !ru || !VP || !VR || !S || !loss || !G ||
        nP < 1 || nR < 1 || !(dt > 0))
        return VERB_ERR_ARG;
    if ((long)nP * nR > kMaxPoints) return VERB_ERR_SIZE;
    if ((nP >= 3 && nP < 11) || (nR >= 3 && nR < 11)) return VERB_ERR_GRID;
    if (verb::conv_scratch_doubles(nP, nR) > (size_t)kPlaneDoubles) return VERB_ERR_SIZE;
    if (int s = verb::conv_check(nP, nR)) return s;
    if ((pl_t == VERB_BC_PERIODIC) != (pu_t == VERB_BC_PERIODIC)) return VERB_ERR_BC;
    if ((rl_t == VERB_BC_PERIODIC) != (ru_t == VERB_BC_PERIODIC)) return VERB_ERR_BC;
    double* scratch = nullptr;
    int s = scratch_for_current_device(&scratch);
    if (s) return s;
    int* words = reinterpret_cast<int*>(scratch + kPlaneDoubles);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // ticket, sub-step count and status start at zero on every call
    if (cudaMemsetAsync(words, 0, kWords * sizeof(double), st) != cudaSuccess) return VERB_ERR_CUDA;
    verb::ConvArgs a{};
    a.d = verb::Dims{nP, nR, 1, 1};
    a.psd = psd;
    a.Pg = P;
    a.Rg = R;
    a.VP = VP;
    a.VR = VR;
    a.S = S;
    a.loss = loss;
    a.G = G;
    a.Pl = pl;
    a.Pu = pu;
    a.Rl = rl;
    a.Ru = ru;
    a.Pl_t = pl_t;
    a.Pu_t = pu_t;
    a.Rl_t = rl_t;
    a.Ru_t = ru_t;
    a.dt = dt;
    a.scratch = scratch;      // one CTA: conv_scratch_doubles(P, R) <= kPlaneDoubles
    a.ticket = words;
    a.substeps = words + 1;
    a.status = words + 2;
    // an error the caller's earlier work left pending stays pending: only a
    // change of the runtime's last error after the launch is this call's own
    const cudaError_t before = cudaPeekAtLastError();
    verb::launch_convection(a, 1, st);
    const cudaError_t after = cudaPeekAtLastError();
    if (after != cudaSuccess && after != before) {
        cudaGetLastError();
        return VERB_ERR_CUDA;
    }
    int dev_status = 0;
    if (cudaMemcpyAsync(&dev_status, words + 2, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return VERB_ERR_CUDA;
    return dev_status;
}
