// A small CNN (3x3 convolutions, zero padding, ReLU between layers) with
// FP16 weights and FP32 accumulation: forward, backward and Adam kernels.
// It maps the per-system coefficient fields and right-hand side of the local
// (V,K) systems to a warm start for their Krylov solve (no counterpart in the
// reference).
//
// Tensors are NCHW FP32 ([batch][channel][H][W], W fastest).  A layer's
// weights are [Cout][Cin][3][3] (FP32 master copy, FP16 copy used by the
// forward and backward passes) plus an FP32 bias [Cout].  One thread computes
// one output value (forward, input gradient) or one weight gradient; the
// batch sizes here (hundreds of 31x31 or 101x91 images, 32 channels) keep
// every SM busy with plain FP32 FMA work, which is far from the tensor-core
// regime (the whole network is ~2e8 multiply-adds per batch).
#include <cuda_fp16.h>

#include <algorithm>
#include <new>
#include <vector>

#include "verb_internal.cuh"

namespace verb {

namespace {

__global__ void conv3x3_fwd_kernel(const float* __restrict__ in, const __half* __restrict__ w,
                                   const float* __restrict__ bias, float* __restrict__ out, int B,
                                   int Cin, int Cout, int H, int W, int relu)
{
    const size_t total = (size_t)B * Cout * H * W;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % W);
        const int y = (int)((i / W) % H);
        const int co = (int)((i / ((size_t)W * H)) % Cout);
        const int b = (int)(i / ((size_t)W * H * Cout));
        float acc = bias[co];
        const float* ib = in + (size_t)b * Cin * H * W;
        const __half* wc = w + (size_t)co * Cin * 9;
        for (int ci = 0; ci < Cin; ci++) {
            const float* ic = ib + (size_t)ci * H * W;
            const __half* wk = wc + ci * 9;
#pragma unroll
            for (int dy = -1; dy <= 1; dy++) {
                const int yy = y + dy;
                if (yy < 0 || yy >= H) continue;
#pragma unroll
                for (int dx = -1; dx <= 1; dx++) {
                    const int xx = x + dx;
                    if (xx < 0 || xx >= W) continue;
                    acc = fmaf(__half2float(wk[(dy + 1) * 3 + (dx + 1)]), ic[yy * W + xx], acc);
                }
            }
        }
        out[i] = (relu && acc < 0.f) ? 0.f : acc;
    }
}

// gradient wrt the layer input: full correlation with the flipped kernel;
// `act` is the input activation when the input went through a ReLU (its
// gradient is masked where the activation is 0), nullptr for the first layer
__global__ void conv3x3_bwd_input_kernel(const float* __restrict__ gout, const __half* __restrict__ w,
                                         const float* __restrict__ act, float* __restrict__ gin,
                                         int B, int Cin, int Cout, int H, int W)
{
    const size_t total = (size_t)B * Cin * H * W;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % W);
        const int y = (int)((i / W) % H);
        const int ci = (int)((i / ((size_t)W * H)) % Cin);
        const int b = (int)(i / ((size_t)W * H * Cin));
        if (act && act[i] <= 0.f) {
            gin[i] = 0.f;
            continue;
        }
        float acc = 0.f;
        const float* gb = gout + (size_t)b * Cout * H * W;
        for (int co = 0; co < Cout; co++) {
            const float* gc = gb + (size_t)co * H * W;
            const __half* wk = w + ((size_t)co * Cin + ci) * 9;
#pragma unroll
            for (int dy = -1; dy <= 1; dy++) {
                const int yy = y - dy;  // out(yy) used in(y) through tap dy
                if (yy < 0 || yy >= H) continue;
#pragma unroll
                for (int dx = -1; dx <= 1; dx++) {
                    const int xx = x - dx;
                    if (xx < 0 || xx >= W) continue;
                    acc = fmaf(__half2float(wk[(dy + 1) * 3 + (dx + 1)]), gc[yy * W + xx], acc);
                }
            }
        }
        gin[i] = acc;
    }
}

// weight and bias gradients: one block per (co, ci, tap) or per co for the bias
__global__ void conv3x3_bwd_weight_kernel(const float* __restrict__ in, const float* __restrict__ gout,
                                          float* __restrict__ gw, float* __restrict__ gb, int B,
                                          int Cin, int Cout, int H, int W)
{
    __shared__ float red[256];
    const int nw = Cout * Cin * 9;
    for (int item = blockIdx.x; item < nw + Cout; item += gridDim.x) {
        float acc = 0.f;
        const size_t HW = (size_t)H * W;
        if (item < nw) {
            const int tap = item % 9, ci = (item / 9) % Cin, co = item / (9 * Cin);
            const int dy = tap / 3 - 1, dx = tap % 3 - 1;
            for (size_t j = threadIdx.x; j < (size_t)B * HW; j += blockDim.x) {
                const int b = (int)(j / HW);
                const int p = (int)(j - (size_t)b * HW);
                const int y = p / W, x = p - (p / W) * W;
                const int yy = y + dy, xx = x + dx;
                if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
                acc = fmaf(gout[((size_t)b * Cout + co) * HW + p], in[((size_t)b * Cin + ci) * HW + yy * W + xx],
                           acc);
            }
        } else {
            const int co = item - nw;
            for (size_t j = threadIdx.x; j < (size_t)B * HW; j += blockDim.x) {
                const int b = (int)(j / HW);
                const int p = (int)(j - (size_t)b * HW);
                acc += gout[((size_t)b * Cout + co) * HW + p];
            }
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            if (item < nw) gw[item] = red[0];
            else gb[item - nw] = red[0];
        }
        __syncthreads();
    }
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
        verb::conv3x3_fwd_kernel<<<verb::blocks_for(tot), 256, 0, n->s>>>(
            x, n->ph + n->woff[l], n->p + n->boff[l], y, B, n->cin[l], n->cout[l], n->H, n->W,
            l < n->L - 1 ? 1 : 0);
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
    float* g0 = n->grad;
    float* g1 = n->grad + n->amax;
    int s = ck(cudaMemsetAsync(n->loss, 0, sizeof(float), n->s));
    if (s) return s;
    verb::mse_kernel<<<verb::blocks_for(nout), 256, 0, n->s>>>(n->act + n->aoff[Lt], target_dev, g0,
                                                               nout, n->loss);
    for (int l = Lt; l >= 0; l--) {
        const float* xin = l > 0 ? n->act + n->aoff[l - 1] : in_dev;
        verb::conv3x3_bwd_weight_kernel<<<148 * 8, 256, 0, n->s>>>(
            xin, g0, n->g + n->woff[l], n->g + n->boff[l], B, n->cin[l], n->cout[l], n->H, n->W);
        if (l > 0) {
            const size_t tin = (size_t)B * n->cin[l] * HW;
            verb::conv3x3_bwd_input_kernel<<<verb::blocks_for(tin), 256, 0, n->s>>>(
                g0, n->ph + n->woff[l], n->act + n->aoff[l - 1], g1, B, n->cin[l], n->cout[l], n->H,
                n->W);
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
    if (loss_host)
        s = ck(cudaMemcpyAsync(loss_host, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->s));
    if (!s) s = ck(cudaStreamSynchronize(n->s));
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
