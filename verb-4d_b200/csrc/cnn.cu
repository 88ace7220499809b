// A small CNN (3x3 convolutions, zero padding, ReLU between layers) with
// FP16 weights and FP32 accumulation: forward, backward and Adam kernels.
// It maps the per-system coefficient fields and right-hand side of the local
// (V,K) systems to a warm start for their Krylov solve (no counterpart in the
// reference).
//
// Tensors are NCHW FP32 ([batch][channel][H][W], W fastest).  A layer's
// weights are [Cout][Cin][3][3] (FP32 master copy, FP16 copy used by the
// forward and backward passes) plus an FP32 bias [Cout].  The convolutions
// run on the tensor cores as implicit GEMMs (TF32 operands, FP32
// accumulation; conv3x3_mma_kernel).
#include <cuda_fp16.h>

#include <algorithm>
#include <new>
#include <vector>

#include "verb_internal.cuh"

namespace verb {

namespace {

// The three convolution passes as implicit GEMMs on the tensor cores
// (mma.sync m16n8k8, TF32 operands, FP32 accumulation).  With k = (ci, tap),
// tap = 3 (dy+1) + (dx+1), and n = (b, y, x) a pixel of the batch:
//   forward        out[co][n]  = bias[co] + sum_k w[co][k] in[ci][n + tap]
//                  (M = Cout, K = 9 Cin, N = B H W; ReLU in the epilogue)
//   input grad     gin[ci][n]  = sum_(co,tap) w[co][ci][tap] gout[co][n - tap]
//                  (M = Cin, K = 9 Cout; masked where the input's ReLU was 0)
//   weight grad    gw[co][k]   = sum_n gout[co][n] in[ci][n + tap]
//                  (M = Cout, N = 9 Cin, K = B H W split across CTAs,
//                  partial sums added atomically)
// where an index outside the image reads zero (zero padding).  The FP16
// weights are exact in TF32; activations and gradients are rounded to TF32
// (cvt.rna) as they enter the MMA.  A warp computes a 16 x 32 tile (four
// m16n8 accumulators) and fetches its fragments straight from global memory
// (L1/L2 resident at these sizes).
struct ConvGeom {
    int B, Cin, Cout, H, W;
};

__device__ __forceinline__ uint32_t to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

enum { CONV_FWD = 0, CONV_BWD_IN = 1, CONV_BWD_W = 2 };

// element (m, k) of the A operand and (k, n) of the B operand of each pass
template <int MODE>
__device__ __forceinline__ float conv_a(const ConvGeom& g, const __half* w, const float* gout, int m,
                                        int k, int M, int K)
{
    if (m >= M || k >= K) return 0.f;
    if (MODE == CONV_FWD) return __half2float(w[(size_t)m * K + k]);  // w[co][ci*9+tap]
    if (MODE == CONV_BWD_IN) {
        const int co = k / 9, tap = k - co * 9;
        return __half2float(w[((size_t)co * g.Cin + m) * 9 + tap]);
    }
    const size_t HW = (size_t)g.H * g.W;  // CONV_BWD_W: gout[b][co][p], k = (b, p)
    const int b = (int)(k / HW);
    return gout[((size_t)b * g.Cout + m) * HW + (k - b * HW)];
}

template <int MODE>
__device__ __forceinline__ float conv_b(const ConvGeom& g, const float* src, int k, int n, int K, int N)
{
    if (k >= K || n >= N) return 0.f;
    const int HW = g.H * g.W;
    int b, p, c, tap;
    if (MODE == CONV_BWD_W) {  // k = (b, p), n = (ci, tap): in[b][ci][p + tap]
        b = k / HW;
        p = k - b * HW;
        c = n / 9;
        tap = n - c * 9;
    } else {                   // k = (c, tap), n = (b, p)
        c = k / 9;
        tap = k - c * 9;
        b = n / HW;
        p = n - b * HW;
    }
    const int y = p / g.W, x = p - (p / g.W) * g.W;
    int dy = tap / 3 - 1, dx = tap - (tap / 3) * 3 - 1;
    if (MODE == CONV_BWD_IN) {  // gout[b][co][p - tap]
        dy = -dy;
        dx = -dx;
    }
    const int yy = y + dy, xx = x + dx;
    if (yy < 0 || yy >= g.H || xx < 0 || xx >= g.W) return 0.f;
    const int C = MODE == CONV_BWD_IN ? g.Cout : g.Cin;
    return src[(((size_t)b * C + c) * g.H + yy) * g.W + xx];
}

// One warp: rows m0 .. m0+15, columns n0 .. n0+31, k over [k_begin, k_end).
// grid: x = column tiles of 128 (4 warps), y = row tiles of 16, z = K chunks
// (weight gradient only).
template <int MODE>
__global__ void __launch_bounds__(128) conv3x3_mma_kernel(ConvGeom g, const float* __restrict__ src,
                                                          const __half* __restrict__ w,
                                                          const float* __restrict__ gout,
                                                          const float* __restrict__ bias,
                                                          const float* __restrict__ act,
                                                          float* __restrict__ dst, int relu,
                                                          int kchunk)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gi = lane >> 2, ti = lane & 3;
    const int HWi = g.H * g.W;
    const int M = MODE == CONV_BWD_IN ? g.Cin : g.Cout;
    const int K = MODE == CONV_FWD ? 9 * g.Cin : (MODE == CONV_BWD_IN ? 9 * g.Cout : g.B * HWi);
    const int N = MODE == CONV_BWD_W ? 9 * g.Cin : g.B * HWi;
    const int m0 = blockIdx.y * 16;
    const int n0 = (blockIdx.x * 4 + warp) * 32;
    if (n0 >= N) return;
    const int kb = MODE == CONV_BWD_W ? blockIdx.z * kchunk : 0;
    const int ke = MODE == CONV_BWD_W ? min(K, kb + kchunk) : K;
    const float* bsrc = MODE == CONV_BWD_IN ? gout : src;
    float acc[4][4] = {};
    for (int k0 = kb; k0 < ke; k0 += 8) {
        uint32_t a[4];
        a[0] = to_tf32(conv_a<MODE>(g, w, gout, m0 + gi, k0 + ti, M, ke));
        a[1] = to_tf32(conv_a<MODE>(g, w, gout, m0 + gi + 8, k0 + ti, M, ke));
        a[2] = to_tf32(conv_a<MODE>(g, w, gout, m0 + gi, k0 + ti + 4, M, ke));
        a[3] = to_tf32(conv_a<MODE>(g, w, gout, m0 + gi + 8, k0 + ti + 4, M, ke));
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int n = n0 + 8 * t + gi;
            uint32_t b[2];
            b[0] = to_tf32(conv_b<MODE>(g, bsrc, k0 + ti, n, ke, N));
            b[1] = to_tf32(conv_b<MODE>(g, bsrc, k0 + ti + 4, n, ke, N));
            mma_tf32(acc[t], a, b);
        }
    }
    // accumulator element e of tile t: row m0 + gi + 8 (e >> 1), column n0 + 8t + 2 ti + (e & 1)
#pragma unroll
    for (int t = 0; t < 4; t++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int m = m0 + gi + 8 * (e >> 1);
            const int n = n0 + 8 * t + 2 * ti + (e & 1);
            if (m >= M || n >= N) continue;
            float v = acc[t][e];
            if (MODE == CONV_BWD_W) {
                atomicAdd(&dst[(size_t)m * N + n], v);
                continue;
            }
            const int b = n / HWi, p = n - b * HWi;
            const size_t o = ((size_t)b * M + m) * HWi + p;
            if (MODE == CONV_FWD) {
                v += bias[m];
                if (relu && v < 0.f) v = 0.f;
            } else if (act && act[o] <= 0.f) {
                v = 0.f;
            }
            dst[o] = v;
        }
}

// bias gradient: one block per output channel, gb[co] = sum over the batch
__global__ void conv_bias_grad_kernel(const float* __restrict__ gout, float* __restrict__ gb, int B,
                                      int Cout, int HW)
{
    __shared__ float red[256];
    const int co = blockIdx.x;
    float acc = 0.f;
    for (size_t j = threadIdx.x; j < (size_t)B * HW; j += blockDim.x) {
        const int b = (int)(j / HW);
        acc += gout[((size_t)b * Cout + co) * HW + (j - (size_t)b * HW)];
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) gb[co] = red[0];
}

template <int MODE>
void launch_conv_mma(const ConvGeom& g, const float* src, const __half* w, const float* gout,
                     const float* bias, const float* act, float* dst, int relu, cudaStream_t s)
{
    const int HW = g.H * g.W;
    const int M = MODE == CONV_BWD_IN ? g.Cin : g.Cout;
    const int N = MODE == CONV_BWD_W ? 9 * g.Cin : g.B * HW;
    dim3 grid((N + 127) / 128, (M + 15) / 16, 1);
    int kchunk = 0;
    if (MODE == CONV_BWD_W) {
        // split the pixel reduction so that about 4 CTAs per SM run
        const long long K = (long long)g.B * HW;
        const long long want = 148 * 4 / ((long long)grid.x * grid.y) + 1;
        kchunk = (int)((K + want - 1) / want);
        kchunk = (kchunk + 7) / 8 * 8;
        grid.z = (unsigned)((K + kchunk - 1) / kchunk);
        cudaMemsetAsync(dst, 0, (size_t)M * N * sizeof(float), s);
    }
    conv3x3_mma_kernel<MODE><<<grid, 128, 0, s>>>(g, src, w, gout, bias, act, dst, relu, kchunk);
}

// mean squared error over the batch (sum / count) and its gradient
__global__ void mse_kernel(const float* __restrict__ pred, const float* __restrict__ target,
                           float* __restrict__ grad, size_t n, float* loss)
{
    __shared__ float red[256];
    float acc = 0.f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float d = pred[i] - target[i];
        grad[i] = 2.f * d / (float)n;
        acc = fmaf(d, d, acc);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)n);
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; refreshes the FP16 copy
__global__ void adam_kernel(float* __restrict__ p, __half* __restrict__ ph, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, size_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float upd = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] -= upd;
        if (ph) ph[i] = __float2half_rn(p[i]);
    }
}

__global__ void to_half_kernel(const float* __restrict__ p, __half* __restrict__ ph, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        ph[i] = __float2half_rn(p[i]);
}

int blocks_for(size_t n)
{
    size_t b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

}  // namespace

}  // namespace verb

// ---------------------------------------------------------------------------
// C ABI: a CNN object with L layers of 3x3 convolutions.

struct verb_cnn {
    int L = 0, H = 0, W = 0, maxb = 0;
    std::vector<int> cin, cout;
    // parameters: per layer [w (Cout*Cin*9) | b (Cout)] in one FP32 block
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    __half* ph = nullptr;  // FP16 weights (bias entries unused)
    std::vector<size_t> woff, boff;
    size_t np = 0;
    float* act = nullptr;   // activations of every layer output for the batch
    float* grad = nullptr;  // two gradient buffers
    float* loss = nullptr;
    std::vector<size_t> aoff;
    size_t amax = 0;
    long long t = 0;        // Adam step
    cudaStream_t s = nullptr;
};

namespace {

int ck(cudaError_t e) { return e == cudaSuccess ? VERB_OK : (e == cudaErrorMemoryAllocation ? VERB_ERR_NOMEM : VERB_ERR_CUDA); }

}  // namespace

extern "C" int verb_cnn_create(verb_cnn** out, int layers, const int* channels, int H, int W,
                               int max_batch, void* stream)
{
    if (!out || layers < 1 || !channels || H < 1 || W < 1 || max_batch < 1) return VERB_ERR_ARG;
    verb_cnn* n = new (std::nothrow) verb_cnn();
    if (!n) return VERB_ERR_NOMEM;
    n->L = layers;
    n->H = H;
    n->W = W;
    n->maxb = max_batch;
    n->s = (cudaStream_t)stream;
    size_t off = 0, aoff = 0;
    const size_t HW = (size_t)H * W;
    for (int l = 0; l < layers; l++) {
        n->cin.push_back(channels[l]);
        n->cout.push_back(channels[l + 1]);
        n->woff.push_back(off);
        off += (size_t)channels[l + 1] * channels[l] * 9;
        n->boff.push_back(off);
        off += channels[l + 1];
        n->aoff.push_back(aoff);
        aoff += (size_t)max_batch * channels[l + 1] * HW;
        n->amax = std::max(n->amax, (size_t)max_batch * std::max(channels[l], channels[l + 1]) * HW);
    }
    n->np = off;
    int s = ck(cudaMalloc(&n->p, off * sizeof(float)));
    if (!s) s = ck(cudaMalloc(&n->g, off * sizeof(float)));
    if (!s) s = ck(cudaMalloc(&n->m, off * sizeof(float)));
    if (!s) s = ck(cudaMalloc(&n->v, off * sizeof(float)));
    if (!s) s = ck(cudaMalloc(&n->ph, off * sizeof(__half)));
    if (!s) s = ck(cudaMalloc(&n->act, aoff * sizeof(float)));
    if (!s) s = ck(cudaMalloc(&n->grad, 2 * n->amax * sizeof(float)));
    if (!s) s = ck(cudaMalloc(&n->loss, sizeof(float)));
    if (!s) s = ck(cudaMemsetAsync(n->m, 0, off * sizeof(float), n->s));
    if (!s) s = ck(cudaMemsetAsync(n->v, 0, off * sizeof(float), n->s));
    if (s) {
        verb_cnn_destroy(n);
        return s;
    }
    *out = n;
    return VERB_OK;
}

extern "C" int verb_cnn_destroy(verb_cnn* n)
{
    if (!n) return VERB_OK;
    for (void* q : {(void*)n->p, (void*)n->g, (void*)n->m, (void*)n->v, (void*)n->ph, (void*)n->act,
                    (void*)n->grad, (void*)n->loss})
        cudaFree(q);
    delete n;
    return VERB_OK;
}

extern "C" int verb_cnn_param_count(const verb_cnn* n, long long* count)
{
    if (!n || !count) return VERB_ERR_ARG;
    *count = (long long)n->np;
    return VERB_OK;
}

// parameters in the order layer 0 weights [Cout][Cin][3][3], layer 0 bias, layer 1 ...
extern "C" int verb_cnn_set_params(verb_cnn* n, const float* host)
{
    if (!n || !host) return VERB_ERR_ARG;
    int s = ck(cudaMemcpyAsync(n->p, host, n->np * sizeof(float), cudaMemcpyHostToDevice, n->s));
    if (s) return s;
    verb::to_half_kernel<<<verb::blocks_for(n->np), 256, 0, n->s>>>(n->p, n->ph, n->np);
    n->t = 0;
    s = ck(cudaMemsetAsync(n->m, 0, n->np * sizeof(float), n->s));
    if (!s) s = ck(cudaMemsetAsync(n->v, 0, n->np * sizeof(float), n->s));
    if (!s) s = ck(cudaStreamSynchronize(n->s));
    return s;
}

extern "C" int verb_cnn_get_params(verb_cnn* n, float* host, float* grad_host)
{
    if (!n || !host) return VERB_ERR_ARG;
    int s = ck(cudaMemcpyAsync(host, n->p, n->np * sizeof(float), cudaMemcpyDeviceToHost, n->s));
    if (!s && grad_host)
        s = ck(cudaMemcpyAsync(grad_host, n->g, n->np * sizeof(float), cudaMemcpyDeviceToHost, n->s));
    if (!s) s = ck(cudaStreamSynchronize(n->s));
    return s;
}

namespace {

void forward(verb_cnn* n, const float* in, int B)
{
    const float* x = in;
    for (int l = 0; l < n->L; l++) {
        float* y = n->act + n->aoff[l];
        const size_t tot = (size_t)B * n->cout[l] * n->H * n->W;
        (void)tot;
        const verb::ConvGeom g{B, n->cin[l], n->cout[l], n->H, n->W};
        verb::launch_conv_mma<verb::CONV_FWD>(g, x, n->ph + n->woff[l], nullptr,
                                              n->p + n->boff[l], nullptr, y,
                                              l < n->L - 1 ? 1 : 0, n->s);
        x = y;
    }
}

}  // namespace

// out (device, B x Cout_last x H x W) = network(in (device, B x Cin x H x W))
extern "C" int verb_cnn_forward(verb_cnn* n, const float* in_dev, float* out_dev, int B)
{
    if (!n || !in_dev || !out_dev || B < 1 || B > n->maxb) return VERB_ERR_ARG;
    forward(n, in_dev, B);
    const size_t tot = (size_t)B * n->cout[n->L - 1] * n->H * n->W;
    int s = ck(cudaMemcpyAsync(out_dev, n->act + n->aoff[n->L - 1], tot * sizeof(float),
                               cudaMemcpyDeviceToDevice, n->s));
    if (!s) s = ck(cudaGetLastError());
    return s;
}

namespace {

// Backward pass from the output gradient in n->grad (first buffer) through
// the activations of the last forward pass on in_dev, then an Adam step
// (lr <= 0: gradients only).
int backward_adam(verb_cnn* n, const float* in_dev, int B, float lr)
{
    const size_t HW = (size_t)n->H * n->W;
    const int Lt = n->L - 1;
    float* g0 = n->grad;
    float* g1 = n->grad + n->amax;
    int s = VERB_OK;
    for (int l = Lt; l >= 0; l--) {
        const float* xin = l > 0 ? n->act + n->aoff[l - 1] : in_dev;
        const verb::ConvGeom g{B, n->cin[l], n->cout[l], n->H, n->W};
        verb::launch_conv_mma<verb::CONV_BWD_W>(g, xin, nullptr, g0, nullptr, nullptr,
                                                n->g + n->woff[l], 0, n->s);
        verb::conv_bias_grad_kernel<<<n->cout[l], 256, 0, n->s>>>(g0, n->g + n->boff[l], B,
                                                                  n->cout[l], (int)HW);
        if (l > 0) {
            verb::launch_conv_mma<verb::CONV_BWD_IN>(g, nullptr, n->ph + n->woff[l], g0, nullptr,
                                                     n->act + n->aoff[l - 1], g1, 0, n->s);
            std::swap(g0, g1);
        }
    }
    if (lr > 0) {
        n->t++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)n->t), c2 = 1.f - powf(b2, (float)n->t);
        verb::adam_kernel<<<verb::blocks_for(n->np), 256, 0, n->s>>>(n->p, n->ph, n->g, n->m, n->v,
                                                                     n->np, lr, b1, b2, 1e-8f, c1, c2);
    }
    return s;
}

}  // namespace

// One training step on a batch: MSE loss against target (device), backward
// pass, Adam update with learning rate lr (lr <= 0: gradients only, no
// update).  loss_host receives the batch loss.
extern "C" int verb_cnn_train_step(verb_cnn* n, const float* in_dev, const float* target_dev, int B,
                                   float lr, float* loss_host)
{
    if (!n || !in_dev || !target_dev || B < 1 || B > n->maxb) return VERB_ERR_ARG;
    forward(n, in_dev, B);
    const size_t HW = (size_t)n->H * n->W;
    const int Lt = n->L - 1;
    const size_t nout = (size_t)B * n->cout[Lt] * HW;
    int s = ck(cudaMemsetAsync(n->loss, 0, sizeof(float), n->s));
    if (s) return s;
    verb::mse_kernel<<<verb::blocks_for(nout), 256, 0, n->s>>>(n->act + n->aoff[Lt], target_dev,
                                                               n->grad, nout, n->loss);
    s = backward_adam(n, in_dev, B, lr);
    if (!s && loss_host)
        s = ck(cudaMemcpyAsync(loss_host, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->s));
    if (!s) s = ck(cudaStreamSynchronize(n->s));
    if (!s) s = ck(cudaGetLastError());
    return s;
}

// The backward pass and Adam step for an output gradient computed by the
// caller (grad_out_dev, the shape of the network's output): the activations
// are those of the last verb_cnn_forward, which must have run on in_dev.
extern "C" int verb_cnn_backward_step(verb_cnn* n, const float* in_dev, const float* grad_out_dev,
                                      int B, float lr)
{
    if (!n || !in_dev || !grad_out_dev || B < 1 || B > n->maxb) return VERB_ERR_ARG;
    const size_t nout = (size_t)B * n->cout[n->L - 1] * n->H * n->W;
    int s = ck(cudaMemcpyAsync(n->grad, grad_out_dev, nout * sizeof(float), cudaMemcpyDeviceToDevice,
                               n->s));
    if (!s) s = backward_adam(n, in_dev, B, lr);
    if (!s) s = ck(cudaGetLastError());
    return s;
}

namespace verb {

int cnn_forward_on(verb_cnn* n, const float* in, float* out, int B, cudaStream_t s)
{
    if (!n) return VERB_ERR_ARG;
    cudaStream_t keep = n->s;
    n->s = s;
    const int st = verb_cnn_forward(n, in, out, B);
    n->s = keep;
    return st;
}

int cnn_shape(const verb_cnn* n, int* cin, int* cout, int* H, int* W, int* maxb)
{
    if (!n) return VERB_ERR_ARG;
    *cin = n->cin[0];
    *cout = n->cout[n->L - 1];
    *H = n->H;
    *W = n->W;
    *maxb = n->maxb;
    return VERB_OK;
}

}  // namespace verb
