// Convection data assimilation: a Kalman filter per (V,K) slice, batched over
// slices.
//
// Reference: runKalmanFilterConvection2D (src/DataAssimilationConvection.cpp:
// 124-253) with getModelMatrixConvection2D and its one-step matrix
// (src/DataAssimilationHelper.cpp:25-171), operator^ (src/MatrixOperations.cpp:
// 466-620), convertToObservationSpace (src/DataAssimilationHelper.cpp:230-269)
// and runKalmanFilter (src/DataAssimilation.cpp:18-77).  A slice of nP x nR
// points is a state of N = nP*nR values (index iR + iP*nR):
//   M    = M1^nt, M1 the first-order upwind transport matrix of the split step
//          dt/nt (Courant number <= 1), cached until the velocities change
//   M1d  = M^ceil(3/24/dt);  Q = M1d diag(t) M1d^T + diag(D)/10 (t = D but
//          (1-cf^2) D on the inner/outer L rows, which Q also keeps unless
//          growing_Q_at_boundary)
//   Pf   = M Pa M^T + Q,  K = Pf H^T (H Pf H^T + R)^-1,  x += K (y - H x),
//          Pa = Pf - K H Pf
// H selects the finite observations of the slice, so H Pf H^T, Pf H^T and
// H Pf are gathers, not products.  Dense N x N products run as one batched
// FP64 GEMM launch over the slices of a chunk (64 x 64 output tiles, 4 x 4
// outputs per thread); matrix powers use binary exponentiation with
// per-slice exponents (slices whose bit is clear sit out the product); the
// gain solves run one CTA per slice (LU with partial pivoting of the m x m
// innovation covariance, the rows of Pf H^T as right-hand sides).
#include "verb_internal.cuh"

namespace verb {

namespace {

constexpr int BT = 64;   // output tile
constexpr int BK = 16;   // k step
constexpr int GT = 256;  // threads

// C = Cin + sgn * (A diag(dk) op(B)), or A diag(dk) op(B) when Cin is null.
// A: M x K (lda), B: K x N (ldb) or, with TB, N x K; batch b -> slice
// idx[b] (idx null: b) with per-slice strides.
template <bool TB>
__global__ void __launch_bounds__(GT) bgemm_kernel(BGemm g)
{
    __shared__ double As[BK][BT + 1];
    __shared__ double Bs[BK][BT + 1];
    const int s = g.idx ? g.idx[blockIdx.z] : blockIdx.z;
    const double* A = g.A + (size_t)s * g.sA;
    const double* B = g.B + (size_t)s * g.sB;
    const double* dk = g.dk ? g.dk + (size_t)s * g.sdk : nullptr;
    double* C = g.C + (size_t)s * g.sC;
    const double* Cin = g.Cin ? g.Cin + (size_t)s * g.sCin : nullptr;
    const int i0 = blockIdx.y * BT, j0 = blockIdx.x * BT;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = 0.0;
    for (int k0 = 0; k0 < g.K; k0 += BK) {
        // A tile: 64 rows x 16 k, stored k-major
        for (int e = threadIdx.x; e < BT * BK; e += GT) {
            const int r = e / BK, k = e % BK;
            const int gi = i0 + r, gk = k0 + k;
            double v = 0.0;
            if (gi < g.M && gk < g.K) {
                v = A[(size_t)gi * g.lda + gk];
                if (dk) v = v * dk[gk];
            }
            As[k][r] = v;
        }
        // B tile: 16 k x 64 columns
        for (int e = threadIdx.x; e < BT * BK; e += GT) {
            int k, c;
            if (TB) {
                c = e / BK;
                k = e % BK;
            } else {
                k = e / BT;
                c = e % BT;
            }
            const int gk = k0 + k, gj = j0 + c;
            double v = 0.0;
            if (gk < g.K && gj < g.N) v = TB ? B[(size_t)gj * g.ldb + gk] : B[(size_t)gk * g.ldb + gj];
            Bs[k][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; k++) {
            double a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = As[k][ty + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; c++) b[c] = Bs[k][tx + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int gi = i0 + ty + 16 * r, gj = j0 + tx + 16 * c;
            if (gi < g.M && gj < g.N) {
                double v = acc[r][c];
                if (Cin) v = Cin[(size_t)gi * g.ldcin + gj] + g.sgn * v;
                C[(size_t)gi * g.ldc + gj] = v;
            }
        }
}

// Courant split per slice (splitTimeStepCourantCondition, maximum Courant
// number 1): nt[s] and the split step.
__global__ void kc_split_kernel(KCArgs a, int* nt)
{
    __shared__ double red[32];
    const int sl = a.s0 + blockIdx.x;
    const Dims d = a.d;
    const size_t VK = (size_t)d.V * d.K;
    const int N = d.P * d.R;
    const double dP = a.Pg[(size_t)d.R * VK + sl] - a.Pg[sl];  // P[1][0] - P[0][0]
    const double dR = a.Rg[VK + sl] - a.Rg[sl];                // R[0][1] - R[0][0]
    double m = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const size_t g = (size_t)i * VK + sl;
        const double c = fabs(a.VP[g] * a.dt / dP) + fabs(a.VR[g] * a.dt / dR);
        m = fmax(m, fabs(c));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
        m = fmax(m, red[0]);
        nt[blockIdx.x] = m <= 1.0 ? 1 : (int)ceil(m / 1.0);
    }
}

// One-step model matrix of slice blockIdx.y (dense N x N, zeros included)
__global__ void kc_model_kernel(KCArgs a, const int* nt, double* M1, size_t sM)
{
    const int b = blockIdx.y, sl = a.s0 + b;
    const Dims d = a.d;
    const size_t VK = (size_t)d.V * d.K;
    const int nP = d.P, nR = d.R, N = nP * nR;
    double* M = M1 + (size_t)b * sM;
    const double dts = a.dt / (double)nt[b];
    const double corr = exp(-dts / a.corr_time);
    const double dP = a.Pg[(size_t)nR * VK + sl] - a.Pg[sl];
    const double dR = a.Rg[VK + sl] - a.Rg[sl];
    // one CTA per slice (gridDim.x == 1): zero fill, then the rows
    for (size_t e = threadIdx.x; e < (size_t)N * N; e += blockDim.x) M[e] = 0.0;
    __syncthreads();
    for (int row = threadIdx.x; row < N; row += blockDim.x) {
        const int iP = row / nR, iR = row % nR;
        double* Mr = M + (size_t)row * N;
        if (iR == 0 || iR == nR - 1) {
            Mr[row] = corr;
            continue;
        }
        const int iPl = (iP == 0 || iP == nP - 1) ? nP - 2 : iP - 1;
        const int iPr = (iP == 0 || iP == nP - 1) ? 1 : iP + 1;
        const size_t g = (size_t)row * VK + sl;
        const double vp = a.VP[g], vr = a.VR[g];
        const double psd = a.psd[g];
        double lc = a.S ? a.S[g] / psd : 0.0;  // Loss = Sources / PSD (the driver's argument)
        double mcc;
        if (a.use_log)
            mcc = 1. - fabs(vp) * dts / dP - fabs(vr) * dts / dR;
        else
            mcc = 1. - fabs(vp) * dts / dP - fabs(vr) * dts / dR + dts * lc;
        if (mcc < 0) set_error(a.status, VERB_ERR_CFL);
        const double mlc = vp > 0. ? vp * dts / dP : 0.;
        const double mrc = vp > 0. ? 0. : -vp * dts / dP;
        const double mcl = vr > 0. ? vr * dts / dR : 0.;
        const double mcr = vr > 0. ? 0. : -vr * dts / dR;
        Mr[row] = mcc;
        Mr[iR + iPl * nR] = mlc;
        Mr[iR + iPr * nR] = mrc;
        Mr[iR - 1 + iP * nR] = mcl;
        Mr[iR + 1 + iP * nR] = mcr;
    }
}

// Q diagonal terms: Q += diag(D)/10, then the inner/outer L rows as the
// reference sets them; t[s][k] = the diagonal of tmp (for the GEMM scale)
__global__ void kc_tdiag_kernel(KCArgs a, double* t, size_t st)
{
    const int b = blockIdx.y;
    const int nR = a.d.R, N = a.d.P * nR;
    const double cf = exp(-a.dt / a.corr_time);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int iR = i % nR;
        t[(size_t)b * st + i] = (iR == 0 || iR == nR - 1) ? (1. - (cf * cf)) * a.model_error
                                                           : a.model_error;
    }
}

__global__ void kc_qdiag_kernel(KCArgs a, double* Q, size_t sQ)
{
    const int b = blockIdx.y;
    const int nR = a.d.R, N = a.d.P * nR;
    const double cf = exp(-a.dt / a.corr_time);
    double* q = Q + (size_t)b * sQ;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int iR = i % nR;
        double v = q[(size_t)i * N + i] + a.model_error / 10;
        if (!a.growing_q && (iR == 0 || iR == nR - 1)) v = (1. - (cf * cf)) * a.model_error;
        q[(size_t)i * N + i] = v;
    }
}

// Pa = 5 model_error I where it is all zero (first use)
__global__ void kc_pa_init_kernel(KCArgs a, double* Pa, size_t sPa)
{
    __shared__ int any;
    const int b = blockIdx.x;
    const int N = a.d.P * a.d.R;
    double* p = Pa + (size_t)(a.s0 + b) * sPa;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    int loc = 0;
    for (size_t e = threadIdx.x; e < (size_t)N * N; e += blockDim.x)
        if (p[e] != 0.0) loc = 1;
    if (loc) any = 1;
    __syncthreads();
    if (!any)
        for (int i = threadIdx.x; i < N; i += blockDim.x) p[(size_t)i * N + i] = 5 * a.model_error;
}

// Observation space of each slice: m[b] finite observations in state order,
// their indices, values and the forecast (logs in the log form).
__global__ void kc_obs_kernel(KCArgs a, int* m, int* oidx, double* y, double* x, int ldo)
{
    const int b = blockIdx.x, sl = a.s0 + b;
    const Dims d = a.d;
    const size_t VK = (size_t)d.V * d.K;
    const int N = d.P * d.R;
    double* xb = x + (size_t)b * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double v = a.psd[(size_t)i * VK + sl];
        xb[i] = a.use_log ? log(v) : v;
    }
    if (threadIdx.x == 0) {
        int c = 0;
        for (int i = 0; i < N; i++) {
            const double o = a.obs[(size_t)i * VK + sl];
            if (isfinite(o)) {
                oidx[(size_t)b * ldo + c] = i;
                y[(size_t)b * ldo + c] = a.use_log ? log(o) : o;
                c++;
            }
        }
        m[b] = c;
    }
}

// G = Pf H^T (N x mm, zero columns beyond m) and S^T (mm x mm, identity
// beyond m), S = H Pf H^T + R;  innovations y - H x (zero beyond m)
__global__ void kc_gain_setup_kernel(KCArgs a, const double* Pf, size_t sPf, double* G, double* St,
                                     size_t sW, const int* m, const int* oidx, double* y,
                                     const double* x, int ldo, int mm)
{
    const int b = blockIdx.y;
    const int N = a.d.P * a.d.R, mb = m[b];
    const double* pf = Pf + (size_t)b * sPf;
    double* g = G + (size_t)b * sW;
    double* st = St + (size_t)b * sW;
    const int* oi = oidx + (size_t)b * ldo;
    const double* yb = y + (size_t)b * ldo;
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x, nth = (size_t)gridDim.x * blockDim.x;
    for (size_t e = tid; e < (size_t)N * mm; e += nth) {
        const int i = (int)(e / mm), c = (int)(e % mm);
        g[e] = c < mb ? pf[(size_t)i * N + oi[c]] : 0.0;
    }
    for (size_t e = tid; e < (size_t)mm * mm; e += nth) {
        const int r = (int)(e / mm), c = (int)(e % mm);
        double v;
        if (r < mb && c < mb) {
            const double rv = a.use_log ? a.obs_error : (r == c ? yb[r] * a.obs_error : 0.0);
            v = pf[(size_t)oi[c] * N + oi[r]] + (r == c ? rv : 0.0);
        } else {
            v = r == c ? 1.0 : 0.0;
        }
        st[e] = v;
    }
}

// K S = G for every row of G, one CTA per slice: LU with partial pivoting of
// S^T (held in St) applied to the rows of G as right-hand sides; K
// overwrites G.
__global__ void kc_solve_kernel(KCArgs a, double* G, double* St, size_t sW, int mm)
{
    __shared__ int s_piv;
    const int b = blockIdx.x;
    const int N = a.d.P * a.d.R;
    double* Kg = G + (size_t)b * sW;
    double* Sm = St + (size_t)b * sW;
    for (int k = 0; k < mm; k++) {
        if (threadIdx.x == 0) {
            int pr = k;
            double best = fabs(Sm[(size_t)k * mm + k]);
            for (int r = k + 1; r < mm; r++) {
                const double v = fabs(Sm[(size_t)r * mm + k]);
                if (v > best) {
                    best = v;
                    pr = r;
                }
            }
            s_piv = pr;
        }
        __syncthreads();
        const int pr = s_piv;
        if (pr != k) {
            for (int c = threadIdx.x; c < mm; c += blockDim.x) {
                const double t = Sm[(size_t)k * mm + c];
                Sm[(size_t)k * mm + c] = Sm[(size_t)pr * mm + c];
                Sm[(size_t)pr * mm + c] = t;
            }
            for (int i = threadIdx.x; i < N; i += blockDim.x) {
                const double t = Kg[(size_t)i * mm + k];
                Kg[(size_t)i * mm + k] = Kg[(size_t)i * mm + pr];
                Kg[(size_t)i * mm + pr] = t;
            }
        }
        __syncthreads();
        const double piv = Sm[(size_t)k * mm + k];
        const int w = mm - k - 1;
        for (int e = threadIdx.x; e < w * (mm - k); e += blockDim.x) {
            const int r = k + 1 + e / (mm - k), c = k + e % (mm - k);
            if (c == k) continue;
            Sm[(size_t)r * mm + c] -= Sm[(size_t)r * mm + k] / piv * Sm[(size_t)k * mm + c];
        }
        for (int e = threadIdx.x; e < w * N; e += blockDim.x) {
            const int r = k + 1 + e / N, i = e % N;
            Kg[(size_t)i * mm + r] -= Sm[(size_t)r * mm + k] / piv * Kg[(size_t)i * mm + k];
        }
        __syncthreads();
        for (int r = k + 1 + threadIdx.x; r < mm; r += blockDim.x)
            Sm[(size_t)r * mm + k] = Sm[(size_t)r * mm + k] / piv;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double* kr = Kg + (size_t)i * mm;
        for (int r = mm - 1; r >= 0; r--) {
            double s = kr[r];
            for (int c = r + 1; c < mm; c++) s -= Sm[(size_t)r * mm + c] * kr[c];
            kr[r] = s / Sm[(size_t)r * mm + r];
        }
    }
}

// x += K (y - H x), NaN check, back into the PSD (exp in the log form);
// Hf = H Pf (mm x N, zero rows beyond m) for the covariance update
__global__ void kc_update_kernel(KCArgs a, const double* Kg, size_t sW, const int* m,
                                 const int* oidx, const double* y, const double* x, int ldo, int mm,
                                 const double* Pf, size_t sPf, double* Hf)
{
    const int b = blockIdx.y, sl = a.s0 + b;
    const Dims d = a.d;
    const size_t VK = (size_t)d.V * d.K;
    const int N = d.P * d.R, mb = m[b];
    const double* kb = Kg + (size_t)b * sW;
    const int* oi = oidx + (size_t)b * ldo;
    const double* yb = y + (size_t)b * ldo;
    const double* xb = x + (size_t)b * N;
    const double* pf = Pf + (size_t)b * sPf;
    double* hf = Hf + (size_t)b * sW;
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x, nth = (size_t)gridDim.x * blockDim.x;
    for (size_t i = tid; i < (size_t)N; i += nth) {
        double s = 0.0;
        for (int c = 0; c < mb; c++) s += kb[i * mm + c] * (yb[c] - xb[oi[c]]);
        double v = xb[i] + s;
        if (isnan(v)) set_error(a.status, VERB_ERR_NAN);
        if (a.use_log) v = pow(2.718281828459045, v);
        a.psd[i * VK + sl] = v;
    }
    for (size_t e = tid; e < (size_t)mm * N; e += nth) {
        const int c = (int)(e / N), j = (int)(e % N);
        hf[e] = c < mb ? pf[(size_t)oi[c] * N + j] : 0.0;
    }
}

__global__ void kc_copy_kernel(const double* src, size_t ss, double* dst, size_t sd, size_t n,
                               const int* idx)
{
    const int b = idx ? idx[blockIdx.y] : blockIdx.y;
    const double* s = src + (size_t)b * ss;
    double* t = dst + (size_t)b * sd;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        t[e] = s[e];
}

inline unsigned gridx(size_t n, int per = 256, unsigned cap = 64) {
    size_t b = (n + per - 1) / per;
    return (unsigned)(b < cap ? (b ? b : 1) : cap);
}

}  // namespace

void launch_bgemm(const BGemm& g, bool tb, int batch, cudaStream_t s)
{
    dim3 grid((g.N + BT - 1) / BT, (g.M + BT - 1) / BT, batch);
    if (tb)
        bgemm_kernel<true><<<grid, GT, 0, s>>>(g);
    else
        bgemm_kernel<false><<<grid, GT, 0, s>>>(g);
}

void launch_kc_split(const KCArgs& a, int nb, int* nt, cudaStream_t s)
{
    kc_split_kernel<<<nb, 256, 0, s>>>(a, nt);
}

void launch_kc_model(const KCArgs& a, int nb, const int* nt, double* M1, size_t sM, cudaStream_t s)
{
    kc_model_kernel<<<dim3(1, nb), 256, 0, s>>>(a, nt, M1, sM);
}

void launch_kc_tdiag(const KCArgs& a, int nb, double* t, size_t st, cudaStream_t s)
{
    kc_tdiag_kernel<<<dim3(gridx((size_t)a.d.P * a.d.R), nb), 256, 0, s>>>(a, t, st);
}

void launch_kc_qdiag(const KCArgs& a, int nb, double* Q, size_t sQ, cudaStream_t s)
{
    kc_qdiag_kernel<<<dim3(gridx((size_t)a.d.P * a.d.R), nb), 256, 0, s>>>(a, Q, sQ);
}

void launch_kc_pa_init(const KCArgs& a, int nb, double* Pa, size_t sPa, cudaStream_t s)
{
    kc_pa_init_kernel<<<nb, 256, 0, s>>>(a, Pa, sPa);
}

void launch_kc_obs(const KCArgs& a, int nb, int* m, int* oidx, double* y, double* x, int ldo,
                   cudaStream_t s)
{
    kc_obs_kernel<<<nb, 256, 0, s>>>(a, m, oidx, y, x, ldo);
}

void launch_kc_gain(const KCArgs& a, int nb, const double* Pf, size_t sPf, double* G, double* St,
                    size_t sW, const int* m, const int* oidx, double* y, const double* x, int ldo,
                    int mm, cudaStream_t s)
{
    const size_t N = (size_t)a.d.P * a.d.R;
    kc_gain_setup_kernel<<<dim3(gridx(N * mm), nb), 256, 0, s>>>(a, Pf, sPf, G, St, sW, m, oidx, y,
                                                                 x, ldo, mm);
    kc_solve_kernel<<<nb, 256, 0, s>>>(a, G, St, sW, mm);
}

void launch_kc_update(const KCArgs& a, int nb, const double* Kg, size_t sW, const int* m,
                      const int* oidx, const double* y, const double* x, int ldo, int mm,
                      const double* Pf, size_t sPf, double* Hf, cudaStream_t s)
{
    const size_t N = (size_t)a.d.P * a.d.R;
    kc_update_kernel<<<dim3(gridx(N * mm), nb), 256, 0, s>>>(a, Kg, sW, m, oidx, y, x, ldo, mm, Pf,
                                                            sPf, Hf);
}

void launch_kc_copy(const double* src, size_t ss, double* dst, size_t sd, size_t n, int nb,
                    const int* idx, cudaStream_t s)
{
    kc_copy_kernel<<<dim3(gridx(n), nb), 256, 0, s>>>(src, ss, dst, sd, n, idx);
}

}  // namespace verb
