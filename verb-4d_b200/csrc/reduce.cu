// Step reductions and elementwise passes over whole 4-D fields.
//  * negative-point count  (src/VERB4D_Solver.cpp:1226-1240), exact integer,
//    and a NaN check of the PSD in the same pass
//  * max |field| of the per-step log (src/VERB4D_Solver.cpp:636-675)
//  * min(DVV*DKK - DVK*DVK) (src/VERB4D_Solver.cpp:747-753), exact min
//  * max(PSD, 1e-21)        (src/VERB4D_Solver.cpp:621, 980, 1072, 1219)
//  * field = base * scale   (UpdatableMatrix scale queue, src/UpdatableMatrix.cpp:698-708)
// Grid-stride loops sized to a multiple of the SM count; one atomic per block.
#include <mutex>
#include <set>
#include <utility>

#include "verb_internal.cuh"

namespace verb {

void allow_max_dynamic_smem(const void* func)
{
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (done.count({func, dev})) return;
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, func) != cudaSuccess) return;
    // the limit counts dynamic shared memory on top of the kernel's static part
    const int dyn = maxsm - (int)fa.sharedSizeBytes;
    if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) == cudaSuccess)
        done.insert({func, dev});
}

namespace {

constexpr int RT = 256;

int grid_for(size_t n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t want = (n + RT - 1) / RT;
    size_t cap = (size_t)sms * 8;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

// The same pass records a NaN anywhere in the PSD as VERB_ERR_NAN in the
// status word (the reference has no such check: a NaN coefficient would
// silently spread through the field; a NaN is not < 0, so the count is the
// reference's either way).
__global__ void negative_count_kernel(const double* __restrict__ psd, size_t n,
                                      unsigned long long* out, int* status)
{
    unsigned long long c = 0;
    bool nan = false;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double v = psd[i];
        c += v < 0 ? 1ull : 0ull;
        nan = nan || v != v;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    nan = __any_sync(0xffffffffu, nan);
    __shared__ unsigned long long red[RT / 32];
    __shared__ int s_nan;
    if (threadIdx.x == 0) s_nan = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = c;
        if (nan) s_nan = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < RT / 32; i++) t += red[i];
        atomicAdd(out, t);
        if (s_nan) set_error(status, VERB_ERR_NAN);
    }
}

// max |x| of up to MAXABS_FIELDS fields in one pass (Matrix4D::maxabs,
// src/Matrix.cpp:5908-5915: start at -inf, std::max(m, |x|), so NaN values
// are skipped); out[f] holds dkey(max) of field f
__global__ void maxabs_kernel(MaxabsArgs a, size_t n)
{
    double m[MAXABS_FIELDS];
#pragma unroll
    for (int f = 0; f < MAXABS_FIELDS; f++) m[f] = -INFINITY;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < MAXABS_FIELDS; f++)
            if (f < a.nf) {
                const double v = fabs(a.x[f][i]);
                m[f] = (m[f] < v) ? v : m[f];
            }
    }
    __shared__ double red[MAXABS_FIELDS][RT / 32];
#pragma unroll
    for (int f = 0; f < MAXABS_FIELDS; f++) {
        double v = m[f];
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_xor_sync(0xffffffffu, v, o);
            v = (v < t) ? t : v;
        }
        if ((threadIdx.x & 31) == 0) red[f][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < a.nf) {
        const int f = threadIdx.x;
        double v = red[f][0];
        for (int i = 1; i < RT / 32; i++) v = (v < red[f][i]) ? red[f][i] : v;
        atomicMax(a.out + f, dkey(v));
    }
}

__global__ void tensor_min_kernel(const double* __restrict__ dvv, const double* __restrict__ dkk,
                                  const double* __restrict__ dvk, size_t n,
                                  unsigned long long* out)
{
    double m = INFINITY;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double v = dvv[i] * dkk[i] - dvk[i] * dvk[i];
        m = (v < m) ? v : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, m, o);
        m = (t < m) ? t : m;
    }
    __shared__ double red[RT / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = red[0];
        for (int i = 1; i < RT / 32; i++) t = (red[i] < t) ? red[i] : t;
        atomicMin(out, dkey(t));
    }
}

__global__ void clamp_kernel(double* psd, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double v = psd[i];
        psd[i] = (v < 1e-21) ? 1e-21 : v;  // std::max(v, 1e-21)
    }
}

__global__ void scale_copy_kernel(double* dst, const double* __restrict__ src, double scale,
                                  size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i] * scale;
}

}  // namespace

void launch_negative_count(const double* psd, size_t n, unsigned long long* out, int* status,
                           cudaStream_t s)
{
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    negative_count_kernel<<<grid_for(n), RT, 0, s>>>(psd, n, out, status);
}

void launch_maxabs(const MaxabsArgs& a, size_t n, cudaStream_t s)
{
    cudaMemsetAsync(a.out, 0, MAXABS_FIELDS * sizeof(unsigned long long), s);
    maxabs_kernel<<<grid_for(n), RT, 0, s>>>(a, n);
}

void launch_tensor_min(const double* dvv, const double* dkk, const double* dvk, size_t n,
                       unsigned long long* out, cudaStream_t s)
{
    cudaMemsetAsync(out, 0xff, sizeof(unsigned long long), s);
    tensor_min_kernel<<<grid_for(n), RT, 0, s>>>(dvv, dkk, dvk, n, out);
}

void launch_clamp_positive(double* psd, size_t n, cudaStream_t s)
{
    clamp_kernel<<<grid_for(n), RT, 0, s>>>(psd, n);
}

void launch_scale_copy(double* dst, const double* src, double scale, size_t n, cudaStream_t s)
{
    scale_copy_kernel<<<grid_for(n), RT, 0, s>>>(dst, src, scale, n);
}

}  // namespace verb
