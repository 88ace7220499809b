// Updatable input fields on the device: the reference's UpdatableMatrix /
// UpdatableListMatrix time-update system (src/UpdatableMatrix.cpp:602-846,
// 913-961).  A field is a list of components; each component has a base
// array, a queue of replacement arrays (the .lst data files), a scale queue
// and from/to limit queues per grid axis.  The host side (ctx.cu) pops the
// queues at each update time; this kernel rebuilds the field from the
// components in the reference's operation order:
//   component value = base * scale (when scale != 1, :698-708), then 0 where
//   any grid coordinate lies outside its [from, to] range (MatrixLimit,
//   :269-300); field = 0 + c0 + c1 + ... (SUM, :932-939) or that sum divided
//   by the number of finite component values at the point (MEAN, :941-952).
#include <math.h>

#include "verb_internal.cuh"

namespace verb {

namespace {

__global__ void merge_components_kernel(double* __restrict__ out, MergeArgs m, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double q[4] = {m.axis[0][i], m.axis[1][i], m.axis[2][i], m.axis[3][i]};
        double acc = 0.0, cnt = 0.0;
        for (int c = 0; c < m.ncomp; c++) {
            const MergeComp& k = m.comp[c];
            double v = k.base[i];
            if (k.scale != 1.0) v *= k.scale;
            bool out_of_range = false;
#pragma unroll
            for (int a = 0; a < 4; a++) out_of_range |= q[a] < k.from[a] || q[a] > k.to[a];
            if (out_of_range) v = 0;
            acc += v;
            cnt += isfinite(v) ? 1.0 : 0.0;
        }
        out[i] = m.mean ? acc / cnt : acc;
    }
}

}  // namespace

void launch_merge_components(double* out, const MergeArgs& m, size_t n, cudaStream_t s)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t want = (n + 255) / 256, cap = (size_t)sms * 8;
    merge_components_kernel<<<(int)(want < cap ? (want ? want : 1) : cap), 256, 0, s>>>(out, m, n);
}

}  // namespace verb

// ---------------------------------------------------------------------------
// L* remapping (src/VERB4D_Solver.cpp:557-619): when L* changes, every
// (P,V,K) line of the PSD is interpolated from the old L* grid to the new one
// by Opm::MonotCubicInterpolator (src/MonotCubicInterpolator.cpp: derivatives
// :613-650, monotone test :379-470, adjustment :653-700, Hermite evaluation
// :160-225 with the basis of MonotCubicInterpolator.hpp:522-537, constant
// extrapolation).  One thread per line; consecutive threads take consecutive
// (V,K), so every access to the [P][R][V][K] arrays is coalesced.  The
// derivatives and the interpolated line go to scratch arrays of the field's
// shape (the old values are read while the new ones are formed).
namespace verb {

namespace {

__device__ __forceinline__ double h00(double t) { return 2 * t * t * t - 3 * t * t + 1; }
__device__ __forceinline__ double h10(double t) { return t * t * t - 2 * t * t + t; }
__device__ __forceinline__ double h01(double t) { return -2 * t * t * t + 3 * t * t; }
__device__ __forceinline__ double h11(double t) { return t * t * t - t * t; }

__global__ void remap_kernel(double* psd, const double* oldL, const double* newL, double* D,
                             double* O, Dims d, int* status)
{
    const size_t VK = (size_t)d.V * d.K;
    const size_t lines = (size_t)d.P * VK;
    const int n = d.R;
    for (size_t line = (size_t)blockIdx.x * blockDim.x + threadIdx.x; line < lines;
         line += (size_t)gridDim.x * blockDim.x) {
        const size_t iP = line / VK, vk = line - iP * VK;
        const size_t b = iP * (size_t)n * VK + vk;  // element i at b + i*VK
        auto X = [&](int i) { return oldL[b + (size_t)i * VK]; };
        auto F = [&](int i) { return psd[b + (size_t)i * VK]; };
        double* Dl = D + b;
        double* Ol = O + b;
        bool ok = n >= 2;
        for (int i = 0; ok && i + 1 < n; i++) ok = X(i) < X(i + 1);
        if (!ok) {  // the interpolator needs a strictly increasing L* line
            set_error(status, VERB_ERR_ARG);
            for (int i = 0; i < n; i++) Ol[(size_t)i * VK] = F(i);
            continue;
        }
        Dl[0] = (F(1) - F(0)) / (X(1) - X(0));
        Dl[(size_t)(n - 1) * VK] = (F(n - 1) - F(n - 2)) / (X(n - 1) - X(n - 2));
        for (int i = 1; i + 1 < n; i++)
            Dl[(size_t)i * VK] = (F(i + 1) - F(i)) / (2 * (X(i + 1) - X(i))) +
                                 (F(i) - F(i - 1)) / (2 * (X(i) - X(i - 1)));
        bool monotone = true;
        int i = 0;
        while (i + 1 < n && F(i) == F(i + 1)) i++;
        if (i + 1 < n) {
            const bool dec = F(i) > F(i + 1);
            for (i = i + 1; i + 1 < n; i++)
                if (dec ? (F(i) < F(i + 1)) : (F(i) > F(i + 1))) {
                    monotone = false;
                    break;
                }
        }
        if (monotone) {
            for (int j = 0; j + 1 < n; j++) {
                const double delta = (F(j + 1) - F(j)) / (X(j + 1) - X(j));
                double* dj = Dl + (size_t)j * VK;
                double* dn = Dl + (size_t)(j + 1) * VK;
                if (fabs(delta) < 1e-14) {
                    *dj = 0.0;
                    *dn = 0.0;
                } else {
                    const double alpha = *dj / delta, beta = *dn / delta;
                    if (!((alpha * alpha + beta * beta) <= 9)) {
                        const double tau = 3 / sqrt(alpha * alpha + beta * beta);
                        *dj = tau * alpha * delta;
                        *dn = tau * beta * delta;
                    }
                }
            }
        }
        int k = 0;  // lower_bound cursor, restarted when the new grid goes back
        double prev = -INFINITY;
        for (int q = 0; q < n; q++) {
            const double v = newL[b + (size_t)q * VK];
            if (!(v >= prev)) k = 0;
            prev = v;
            while (k < n && X(k) < v) k++;
            double r;
            if (k == 0) r = F(0);
            else if (k == n) r = F(n - 1);
            else {
                const double t = (v - X(k - 1)) / (X(k) - X(k - 1));
                const double h = X(k) - X(k - 1);
                r = F(k - 1) * h00(t) + Dl[(size_t)(k - 1) * VK] * h10(t) * h + F(k) * h01(t) +
                    Dl[(size_t)k * VK] * h11(t) * h;
            }
            Ol[(size_t)q * VK] = r;
        }
    }
}

}  // namespace

void launch_remap(double* psd, const double* oldL, const double* newL, double* D, double* O,
                  const Dims& d, int* status, cudaStream_t s)
{
    const size_t lines = (size_t)d.P * d.V * d.K;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t want = (lines + 127) / 128, cap = (size_t)sms * 16;
    remap_kernel<<<(int)(want < cap ? (want ? want : 1) : cap), 128, 0, s>>>(psd, oldL, newL, D, O, d,
                                                                           status);
    cudaMemcpyAsync(psd, O, d.npts() * sizeof(double), cudaMemcpyDeviceToDevice, s);
}

}  // namespace verb
