// Radial Kalman-filter assimilation, batched over (P,V,K) columns.
//
// Reference: runKalmanFilterDiffusion1D (src/DataAssimilationDiffusion.cpp:151-253),
// getModelMatrixDiffusion1D (src/DataAssimilationHelper.cpp:174-198),
// convertToObservationSpace (:271-305) and runKalmanFilter
// (src/DataAssimilation.cpp:18-77).  Per column, with n = R:
//   A, B  = the radial operator with zero sources/losses (A's last-row
//           sub-diagonal is dropped by CalculationMatrix::toMatrix2D,
//           src/Matrix.cpp:6495-6575, and that is kept here)
//   F     = B A^-1          (trans_solve: X A = B)
//   Pf    = F Pa F^T + Q,   Q = model_error I,  Pa0 = 5 model_error I
//   K     = Pf H^T (H Pf H^T + R)^-1,  R = obs_error I
//   x    += K (y - H x);    Pa = Pf - K H Pf
// H selects the finite observations; with none, K = 0 (the reference's dummy
// one-row H of zeros), so x is unchanged and Pa = Pf.
//
// One persistent CTA processes one column at a time.  Dense n x n operands
// live in a per-CTA global workspace (L2-resident); products use 32x32
// shared-memory tiles.  F comes from n tridiagonal solves with A^T (O(n^2)),
// and the gain from an LU with partial pivoting of the m x m innovation
// covariance.  FP64 throughout; compiled with -fmad=false except for the
// explicit fma() in the products.
#include "verb_internal.cuh"

namespace verb {

namespace {

constexpr int KF_THREADS = 256;
constexpr int TILE = 32;

// C[i][j] = sum_k A[i][k] * B[k][j]   (B transposed when tb: B[j][k])
// then C = (sub ? Cin - C : C).  Row-major with leading dimensions.
__device__ void gemm(double* C, int ldc, const double* A, int lda, const double* B, int ldb,
                     int M, int N, int Kd, bool tb, const double* Cin, int ldcin, double* sm)
{
    double* As = sm;                  // [TILE][TILE+1]
    double* Bs = sm + TILE * (TILE + 1);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads, 2x2 outputs each
    for (int i0 = 0; i0 < M; i0 += TILE)
        for (int j0 = 0; j0 < N; j0 += TILE) {
            double acc[2][2] = {{0, 0}, {0, 0}};
            for (int k0 = 0; k0 < Kd; k0 += TILE) {
                for (int e = threadIdx.x; e < TILE * TILE; e += blockDim.x) {
                    const int r = e / TILE, c = e % TILE;
                    const int ai = i0 + r, ak = k0 + c;
                    As[r * (TILE + 1) + c] = (ai < M && ak < Kd) ? A[(size_t)ai * lda + ak] : 0.0;
                    const int bk = k0 + r, bj = j0 + c;
                    double bv = 0.0;
                    if (bk < Kd && bj < N) bv = tb ? B[(size_t)bj * ldb + bk] : B[(size_t)bk * ldb + bj];
                    Bs[r * (TILE + 1) + c] = bv;
                }
                __syncthreads();
#pragma unroll 8
                for (int k = 0; k < TILE; k++) {
                    const double a0 = As[(2 * ty) * (TILE + 1) + k], a1 = As[(2 * ty + 1) * (TILE + 1) + k];
                    const double b0 = Bs[k * (TILE + 1) + 2 * tx], b1 = Bs[k * (TILE + 1) + 2 * tx + 1];
                    acc[0][0] = fma(a0, b0, acc[0][0]);
                    acc[0][1] = fma(a0, b1, acc[0][1]);
                    acc[1][0] = fma(a1, b0, acc[1][0]);
                    acc[1][1] = fma(a1, b1, acc[1][1]);
                }
                __syncthreads();
            }
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    const int i = i0 + 2 * ty + a, j = j0 + 2 * tx + b;
                    if (i < M && j < N)
                        C[(size_t)i * ldc + j] = Cin ? Cin[(size_t)i * ldcin + j] - acc[a][b] : acc[a][b];
                }
        }
    __syncthreads();
}

__global__ void __launch_bounds__(KF_THREADS) kf_kernel(KFArgs a)
{
    extern __shared__ double sm[];
    const Dims d = a.d;
    const int n = d.R;
    const size_t RR = (size_t)n * n;
    double* gsm = sm;                                 // gemm tiles: 2*TILE*(TILE+1)
    double* x = gsm + 2 * TILE * (TILE + 1);          // [n] forecast
    double* lo = x + n;                               // A^T Thomas: sub, diag, sup
    double* dg = lo + n;
    double* up = dg + n;
    double* bd = up + n;                              // diag of B
    double* gam = bd + n;                             // Thomas factors of A^T
    double* bet = gam + n;
    double* y = bet + n;                              // innovations [n]
    int* oidx = (int*)(y + n);                        // observed indices [n]
    __shared__ int s_col, s_m, s_any, s_nan;
    double* W = a.work + (size_t)blockIdx.x * 5 * RR;
    double* F = W;
    double* T = W + RR;
    double* Pf = W + 2 * RR;
    double* Sm = W + 3 * RR;   // m x m innovation covariance, LU in place
    double* Kg = W + 4 * RR;   // n x m: Pf H^T, then K
    const size_t VK = (size_t)d.V * d.K;
    const int ncols = a.p_index >= 0 ? (int)VK : (int)(d.P * VK);

    for (;;) {
        if (threadIdx.x == 0) s_col = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int col = s_col;
        __syncthreads();
        if (col >= ncols) break;
        const size_t p = a.p_index >= 0 ? (size_t)a.p_index : (size_t)col / VK;
        const size_t vk = a.p_index >= 0 ? (size_t)col : (size_t)col % VK;
        const size_t cid = a.p_index >= 0 ? vk : p * VK + vk;  // Pa holds the columns in use
        double* Pa = a.Pa + cid * RR;
        auto gi = [&](int r) { return (p * d.R + r) * VK + vk; };

        // forecast, observations and the radial operator (zero sources/losses)
        if (threadIdx.x == 0) {
            int m = 0;
            for (int r = 0; r < n; r++) {
                x[r] = a.psd[gi(r)];
                const double o = a.obs[gi(r)];
                if (isfinite(o)) {
                    oidx[m] = r;
                    y[m] = o;
                    m++;
                }
            }
            s_m = m;
            // rows of A (getCalculationMatrix1DDiffusion with S = Loss = 0)
            const double sc = a.dll_scale;
            for (int r = 0; r < n; r++) {
                double al = 0, ad = 0, au = 0, b = 0;
                if (r == 0) {
                    const double dh = a.Rg[gi(1)] - a.Rg[gi(0)];
                    if (a.Ll_t == VERB_BC_CONSTANT_VALUE) { ad = 1; au = 0; }
                    else { ad = 1 / dh; au = -1 / dh; }
                } else if (r == n - 1) {
                    const double dh = a.Rg[gi(r)] - a.Rg[gi(r - 1)];
                    if (a.Lu_t == VERB_BC_CONSTANT_VALUE) { ad = 1; al = 0; }
                    else { ad = 1 / dh; al = -1 / dh; }
                } else {
                    const double xm = a.Rg[gi(r - 1)], x0 = a.Rg[gi(r)], xp = a.Rg[gi(r + 1)];
                    double Dm = a.DLL[gi(r - 1)], D0 = a.DLL[gi(r)], Dp = a.DLL[gi(r + 1)];
                    if (sc != 1.0) { Dm *= sc; D0 *= sc; Dp *= sc; }
                    const double Gm = a.G[gi(r - 1)], G0 = a.G[gi(r)], Gp = a.G[gi(r + 1)];
                    ad += 1.0 / a.dt;
                    b += 1.0 / a.dt;
                    ad -= 0.0;
                    {
                        double dh1 = x0 - xm, dh21 = x0 - xp, dh22 = xm - x0;
                        double cp = -0.5 / G0 / dh1;
                        ad += +cp / dh21 * D0 * G0;
                        au += -cp / dh21 * D0 * G0;
                        al += -cp / dh22 * Dm * Gm;
                        ad += +cp / dh22 * Dm * Gm;
                    }
                    {
                        double dh1 = x0 - xp, dh21 = x0 - xm, dh22 = xp - x0;
                        double cp = -0.5 / G0 / dh1;
                        ad += +cp / dh21 * D0 * G0;
                        al += -cp / dh21 * D0 * G0;
                        au += -cp / dh22 * Dp * Gp;
                        ad += +cp / dh22 * Dp * Gp;
                    }
                }
                if (r == n - 1) al = 0.0;  // toMatrix2D drops the last row's sub-diagonal
                // A^T: sub-diagonal of A^T row r is A[r-1][r] = up[r-1]; super is A[r+1][r]
                dg[r] = ad;
                bd[r] = b;
                up[r] = au;   // temporarily A's super-diagonal
                lo[r] = al;   // A's sub-diagonal
            }
            // Thomas factors of A^T: sub'[r] = up[r-1], sup'[r] = lo[r+1]
            double bt = dg[0];
            bet[0] = bt;
            gam[0] = 0;
            for (int r = 1; r < n; r++) {
                const double g = lo[r] / bt;  // sup'[r-1] = lo[r]
                bt = dg[r] - up[r - 1] * g;
                gam[r] = g;
                bet[r] = bt;
            }
        }
        __syncthreads();
        const int m = s_m;

        // F = B A^-1: row i solves A^T f = b_i e_i
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double* f = F + (size_t)i * n;
            double u = 0.0;
            for (int r = 0; r < n; r++) {
                const double rhs = (r == i) ? bd[i] : 0.0;
                u = (rhs - (r ? up[r - 1] * u : 0.0)) / bet[r];
                f[r] = u;
            }
            for (int r = n - 1; r >= 1; r--) {
                u = f[r - 1] - gam[r] * u;
                f[r - 1] = u;
            }
        }
        // Pa initialisation on first use (src/DataAssimilationDiffusion.cpp:213-218)
        if (threadIdx.x == 0) s_any = 0;
        __syncthreads();
        for (size_t e = threadIdx.x; e < RR; e += blockDim.x)
            if (Pa[e] != 0.0) s_any = 1;
        __syncthreads();
        if (!s_any)
            for (int i = threadIdx.x; i < n; i += blockDim.x) Pa[(size_t)i * n + i] = 5 * a.model_error;
        __syncthreads();
        // Pf = F Pa F^T + Q
        gemm(T, n, F, n, Pa, n, n, n, n, false, nullptr, 0, gsm);
        gemm(Pf, n, T, n, F, n, n, n, n, true, nullptr, 0, gsm);
        for (int i = threadIdx.x; i < n; i += blockDim.x) Pf[(size_t)i * n + i] += a.model_error;
        __syncthreads();
        if (m == 0) {
            // no observation: x += 0 (the reference's dummy row), and the
            // NaN check still applies (src/DataAssimilation.cpp:62-67)
            bool bad = false;
            for (int i = threadIdx.x; i < n; i += blockDim.x) bad = bad || isnan(x[i]);
            if (__syncthreads_or(bad) && threadIdx.x == 0) set_error(a.status, VERB_ERR_NAN);
            for (size_t e = threadIdx.x; e < RR; e += blockDim.x) Pa[e] = Pf[e];
            __syncthreads();
            continue;
        }
        // PfHt (n x m) and S = H Pf H^T + R (m x m)
        for (int e = threadIdx.x; e < n * m; e += blockDim.x) {
            const int i = e / m, c = e % m;
            Kg[(size_t)i * m + c] = Pf[(size_t)i * n + oidx[c]];
        }
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            const int r = e / m, c = e % m;
            // S^T, since K S = PfHt is solved as S^T K^T = PfHt^T
            Sm[(size_t)r * m + c] = Pf[(size_t)oidx[c] * n + oidx[r]] + (r == c ? a.obs_error : 0.0);
        }
        for (int c = threadIdx.x; c < m; c += blockDim.x) y[c] = y[c] - x[oidx[c]];
        __syncthreads();
        // K S = PfHt  <=>  S^T K^T = PfHt^T: LU of S^T (held in Sm) with partial
        // pivoting; each row of Kg is one right-hand side.
        for (int k = 0; k < m; k++) {
            if (threadIdx.x == 0) {
                int pr = k;
                double best = fabs(Sm[(size_t)k * m + k]);
                for (int r = k + 1; r < m; r++) {
                    const double v = fabs(Sm[(size_t)r * m + k]);
                    if (v > best) { best = v; pr = r; }
                }
                s_col = pr;
            }
            __syncthreads();
            const int pr = s_col;
            if (pr != k) {
                for (int c = threadIdx.x; c < m; c += blockDim.x) {
                    const double t = Sm[(size_t)k * m + c];
                    Sm[(size_t)k * m + c] = Sm[(size_t)pr * m + c];
                    Sm[(size_t)pr * m + c] = t;
                }
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    const double t = Kg[(size_t)i * m + k];
                    Kg[(size_t)i * m + k] = Kg[(size_t)i * m + pr];
                    Kg[(size_t)i * m + pr] = t;
                }
            }
            __syncthreads();
            const double piv = Sm[(size_t)k * m + k];
            for (int e = threadIdx.x; e < (m - k - 1) * (m - k); e += blockDim.x) {
                const int r = k + 1 + e / (m - k), c = k + e % (m - k);
                if (c == k) continue;
                const double l = Sm[(size_t)r * m + k] / piv;
                Sm[(size_t)r * m + c] -= l * Sm[(size_t)k * m + c];
            }
            for (int e = threadIdx.x; e < (m - k - 1) * n; e += blockDim.x) {
                const int r = k + 1 + e / n, i = e % n;
                const double l = Sm[(size_t)r * m + k] / piv;
                Kg[(size_t)i * m + r] -= l * Kg[(size_t)i * m + k];
            }
            __syncthreads();
            for (int r = k + 1 + threadIdx.x; r < m; r += blockDim.x)
                Sm[(size_t)r * m + k] = Sm[(size_t)r * m + k] / piv;
            __syncthreads();
        }
        // back substitution per row of Kg (each row i is one right-hand side)
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double* kr = Kg + (size_t)i * m;
            for (int r = m - 1; r >= 0; r--) {
                double s = kr[r];
                for (int c = r + 1; c < m; c++) s -= Sm[(size_t)r * m + c] * kr[c];
                kr[r] = s / Sm[(size_t)r * m + r];
            }
        }
        __syncthreads();
        // x += K (y - H x); NaN check (src/DataAssimilation.cpp:53-67)
        if (threadIdx.x == 0) s_nan = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double s = 0.0;
            for (int c = 0; c < m; c++) s += Kg[(size_t)i * m + c] * y[c];
            const double v = x[i] + s;
            if (isnan(v)) s_nan = 1;
            a.psd[gi(i)] = v;
        }
        // T = H Pf (m x n): rows of Pf at the observed indices
        for (int e = threadIdx.x; e < m * n; e += blockDim.x) {
            const int c = e / n, j = e % n;
            T[(size_t)c * n + j] = Pf[(size_t)oidx[c] * n + j];
        }
        __syncthreads();
        if (s_nan) set_error(a.status, VERB_ERR_NAN);
        // Pa = Pf - K (H Pf)
        gemm(Pa, n, Kg, m, T, n, n, n, m, false, Pf, n, gsm);
    }
}

}  // namespace

int kf_ctas(const Dims& d, int p_index)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t cols = p_index >= 0 ? (size_t)d.V * d.K : (size_t)d.P * d.V * d.K;
    size_t nctas = (size_t)sms * 2;
    return (int)(nctas < cols ? nctas : cols);
}

void launch_kf(const KFArgs& a, int nctas, cudaStream_t s)
{
    const int n = a.d.R;
    cudaMemsetAsync(a.ticket, 0, sizeof(int), s);
    const size_t smem = (2 * TILE * (TILE + 1) + 8 * (size_t)n) * sizeof(double) + n * sizeof(int);
    kf_kernel<<<nctas, KF_THREADS, smem, s>>>(a);
}

}  // namespace verb
