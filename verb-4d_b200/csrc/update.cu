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
