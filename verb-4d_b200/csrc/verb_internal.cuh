// Internal declarations shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "verb4d_b200.h"

namespace verb {

// Raise a kernel's dynamic shared-memory limit to the device maximum, once per
// (kernel, device).  The attribute belongs to the function, not to a launch,
// so setting it per launch to that launch's size would race when contexts of
// different sizes are driven from different host threads (ensembles).
void allow_max_dynamic_smem(const void* func);

struct Dims {
    int P, R, V, K;
    __host__ __device__ size_t npts() const { return (size_t)P * R * V * K; }
    __host__ __device__ size_t at(int p, int r, int v, int k) const
    {
        return (((size_t)p * R + r) * V + v) * K + k;
    }
};

// Device-side status word: the first non-zero code wins.
__device__ __forceinline__ void set_error(int* status, int code)
{
    if (status) atomicCAS(status, 0, code);
}

// --- radial ------------------------------------------------------------------
struct RadialArgs {
    Dims d;
    double* psd;
    const double *L, *DLL, *G, *S, *loss;
    double dll_scale;
    const double *Ll, *Lu;
    int Ll_t, Lu_t;
    double dt;
    int radial_sources;
    double *fa, *fbet, *fgam;  // cached Thomas factors [R][P*V*K]
    int* status;
};
void launch_radial_factor(const RadialArgs& a, cudaStream_t s);
void launch_radial_solve(const RadialArgs& a, cudaStream_t s);
void launch_tridag(const double* a, const double* b, const double* c, const double* r, double* u,
                  long n, cudaStream_t s);

// --- convection data assimilation (kfconv.cu) ---------------------------------
// batched row-major FP64 GEMM: C[s] = Cin[s] + sgn * A[s] diag(dk[s]) op(B[s])
// (Cin null: no addend; dk null: no scale); batch b works on slice idx[b]
struct BGemm {
    const double* A; size_t sA; int lda;
    const double* B; size_t sB; int ldb;
    double* C; size_t sC; int ldc;
    const double* Cin; size_t sCin; int ldcin;
    double sgn;
    const double* dk; size_t sdk;
    int M, N, K;
    const int* idx;
};
void launch_bgemm(const BGemm& g, bool tb, int batch, cudaStream_t s);
struct KCArgs {
    Dims d;
    int s0;  // first (V,K) slice of the chunk (slice = v*K + k)
    double dt, model_error, obs_error, corr_time;
    int use_log, growing_q;
    const double *Pg, *Rg, *VP, *VR, *S;
    double* psd;
    const double* obs;
    int* status;
};
void launch_kc_split(const KCArgs& a, int nb, int* nt, cudaStream_t s);
void launch_kc_model(const KCArgs& a, int nb, const int* nt, double* M1, size_t sM, cudaStream_t s);
void launch_kc_tdiag(const KCArgs& a, int nb, double* t, size_t st, cudaStream_t s);
void launch_kc_qdiag(const KCArgs& a, int nb, double* Q, size_t sQ, cudaStream_t s);
void launch_kc_pa_init(const KCArgs& a, int nb, double* Pa, size_t sPa, cudaStream_t s);
void launch_kc_obs(const KCArgs& a, int nb, int* m, int* oidx, double* y, double* x, int ldo,
                   cudaStream_t s);
void launch_kc_gain(const KCArgs& a, int nb, const double* Pf, size_t sPf, double* G, double* St,
                    size_t sW, const int* m, const int* oidx, double* y, const double* x, int ldo,
                    int mm, cudaStream_t s);
void launch_kc_update(const KCArgs& a, int nb, const double* Kg, size_t sW, const int* m,
                      const int* oidx, const double* y, const double* x, int ldo, int mm,
                      const double* Pf, size_t sPf, double* Hf, cudaStream_t s);
void launch_kc_copy(const double* src, size_t ss, double* dst, size_t sd, size_t n, int nb,
                    const int* idx, cudaStream_t s);

// --- convection ----------------------------------------------------------------
struct ConvArgs {
    Dims d;
    double* psd;
    const double *Pg, *Rg, *VP, *VR, *S, *loss, *G;
    const double *Pl, *Pu, *Rl, *Ru;
    int Pl_t, Pu_t, Rl_t, Ru_t;
    double dt;
    double* scratch;     // per-CTA conv_scratch_doubles(P, R): Courant tables and planes
    int* substeps;       // [V][K] out
    int* ticket;         // work counter (zeroed before launch)
    int* status;
};
int conv_ctas(int P, int R);
int conv_check(int P, int R);  // VERB_ERR_SIZE for slices the kernel cannot hold
size_t conv_smem_bytes(int P, int R);
size_t conv_scratch_doubles(int P, int R);
void launch_convection(const ConvArgs& a, int nctas, cudaStream_t s);
// the same kernel compiled with multiply-add contraction (convection.cu)
int conv_ctas_fma(int P, int R);
int conv_check_fma(int P, int R);
size_t conv_smem_bytes_fma(int P, int R);
void launch_convection_fma(const ConvArgs& a, int nctas, cudaStream_t s);
// one thread per line, streaming register windows (convection_stream.cu)
int conv_stream_check(int P, int R);  // VERB_ERR_SIZE: the shape needs convection.cu
size_t conv_stream_scratch_doubles(int P, int R);
int conv_stream_ctas(int P, int R);
int conv_stream_ctas_max(int P, int R);
void launch_convection_stream(const ConvArgs& a, int nctas, cudaStream_t s);
void launch_convection_line(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                            int ubc_t, const double* ux, double dt, int* status, cudaStream_t s);

// --- local ---------------------------------------------------------------------
struct LocalArgs {
    Dims d;
    double* psd;
    const double *Vg, *Kg, *DVV, *DKK, *DVK, *DKV, *G, *S, *loss;  // DKV: the Dyx term
    const double *Vl, *Vu, *Kl, *Ku;
    int Vl_t, Vu_t, Kl_t, Ku_t;
    double dt;          // sub-step dt (dt / num_substeps)
    int local_sources;
    int include_boundary;
    int kl, kv, klp, kvp;  // band sizes and padded column strides
    double* Lf;         // [sys][n][klp]   L multipliers of column j
    double* Uf;         // [sys][n][kvp]   U column j, rows j-kv..j (index kv = diagonal)
    // FP32 copies of the factors (mixed-precision form; the same layout with
    // the strides klp32, kvp32), used instead of Lf/Uf when factors32 is set
    int factors32, klp32, kvp32;
    float* Lf32;
    float* Uf32;
    // ragged (trimmed) systems: system s keeps pitch-angle indices k0[s]..K-1
    // (unknowns V*(K-k0[s]) from offset uoff[s]); the new lower K edge is a
    // ConstantValue 0 boundary.  nullptr: every system is the full V*K grid.
    const int* k0;
    const long long* uoff;
    // local solve shape (local_solve_variant_shape), chosen by the autotuner
    int solve_variant;
    // optional per-system selection: only systems with (sel[sys] & sel_mask)
    // != 0 are processed
    const unsigned char* sel;
    unsigned char sel_mask;
    int32_t* ipiv;      // [sys][n]        0-based pivot rows
    double* work;       // [sys][n]        rhs / solution in unknown order (iK*V + iV)
    unsigned long long* negatives;  // optional: count of PSD < 0 written by the store kernel
    int* status;
};
size_t local_factor_smem(int V);
// returns the number of kernels launched
int launch_local_factor(const LocalArgs& a, cudaStream_t s);
void launch_local_rhs(const LocalArgs& a, bool from_work, cudaStream_t s);
void launch_local_solve(const LocalArgs& a, cudaStream_t s);
int local_solve_variants();
void local_solve_variant_shape(int v, int* warps, int* fwd, int* bwd, int* rw = nullptr);
void launch_local_store(const LocalArgs& a, cudaStream_t s);
// r = b - A x for every system (A assembled on the fly in the reference's order)
void launch_local_residual(const LocalArgs& a, const double* b, const double* x, double* r,
                           cudaStream_t s);
// x += d; red[0] = max |d|, red[1] = max |x| (dkey-ordered, atomicMax)
void launch_local_update(const LocalArgs& a, double* x, const double* d, unsigned long long* red,
                         cudaStream_t s);
// ---- Krylov form of the local solve (learned warm start) -------------------
// FP32 copy of every system's 9 diagonals, [sys][9][n] (slot (dy+1)*3+(dx+1))
void launch_local_assemble32(const LocalArgs& a, float* A9, cudaStream_t s);
// batched right-Jacobi-preconditioned BiCGSTAB in FP32: A d = r for every
// selected system, d from 0; iters[sys] += iterations, ok[sys] = converged
// (ok may be nullptr);
// scratch: 6 vectors of n floats per system
// Cp: the learned preconditioner's coefficients [sys][25][n] (nullptr: Jacobi)
void launch_bicgstab(const LocalArgs& a, const float* A9, const float* Cp, const double* r, double* d,
                     float* scratch, int maxit, float tol, int* iters, unsigned char* ok,
                     cudaStream_t s);
// features of the learned preconditioner, [sys][9][K'][V] (log10 |diag| dt and
// the off-diagonal entries over the diagonal)
void launch_precond_features(const LocalArgs& a, const float* A9, float* feat, cudaStream_t s);
// its training gradient for nprobe probes per system (systems of nx * ny
// unknowns, contiguous): gC [sys][25][n], loss += |A M z - z|^2 / count
int launch_precond_grad(const float* A9, const float* C, const float* Z, float* gC, float* loss,
                        int nsys, int nx, int ny, int nprobe, cudaStream_t s);
// the PSD of every system in the unknown order
void launch_gather_state(const LocalArgs& a, double* x, cudaStream_t s);
// features of the state f (unknown order) for the warm-start CNN:
// feat [sys][4][K][V] = (log10 D_VV - m)/2, (log10 D_KK - m)/2,
// D_VK/sqrt(D_VV D_KK), f/max|f|; scale[sys] = max|f| (1 where f = 0)
void launch_local_features(const LocalArgs& a, const double* f, float* feat, double* scale,
                           cudaStream_t s);
// warm start x = f + out * scale (out == nullptr: x = f)  /  target = (x - f) / scale
void launch_warm_start(const LocalArgs& a, const double* b, const float* out, const double* scale,
                       double* x, cudaStream_t s);
void launch_local_targets(const LocalArgs& a, const double* b, const double* x, const double* scale,
                          float* target, cudaStream_t s);
// per system: rel = max|b - A x| / max|b| (FP64).  pend[sys] = 0 when
// rel <= tol, 2 (give up: LU) when a previous rel is recorded and
// rel > stall * prev, else 1; cnt[0] / cnt[1] count the 1s / 2s; prev[sys]
// becomes rel; maxkey holds the largest rel (as a dkey)
void launch_residual_check(const LocalArgs& a, const double* b, const double* x, double tol,
                           double stall, double* prev, unsigned char* pend, unsigned int* cnt,
                           unsigned long long* maxkey, cudaStream_t s);
// forward pass of a warm-start network on stream s (cnn.cu)
int cnn_forward_on(verb_cnn* n, const float* in, float* out, int B, cudaStream_t s);
int cnn_shape(const verb_cnn* n, int* cin, int* cout, int* H, int* W, int* maxb);
// weighted Jacobi sweep x += omega * r / diag (diag from the FP32 diagonals)
void launch_jacobi_update(const LocalArgs& a, const float* A9, const double* r, double* x,
                          double omega, cudaStream_t s);
// x[sys] <- y[sys] for systems with sel[sys] != 0
void launch_masked_copy(const LocalArgs& a, double* x, const double* y, cudaStream_t s);
// unknowns of all systems (V*K*P*R, or the sum over trimmed systems)

// --- reductions / elementwise ---------------------------------------------------
void launch_negative_count(const double* psd, size_t n, unsigned long long* out, int* status,
                           cudaStream_t s);
constexpr int MAXABS_FIELDS = 8;
struct MaxabsArgs {
    const double* x[MAXABS_FIELDS];
    int nf;
    unsigned long long* out;  // [MAXABS_FIELDS] dkey of max |x| per field
};
void launch_maxabs(const MaxabsArgs& a, size_t n, cudaStream_t s);
void launch_tensor_min(const double* dvv, const double* dkk, const double* dvk, size_t n,
                       unsigned long long* out_ordered, cudaStream_t s);
void launch_clamp_positive(double* psd, size_t n, cudaStream_t s);
void launch_scale_copy(double* dst, const double* src, double scale, size_t n, cudaStream_t s);

// --- updatable fields ------------------------------------------------------------------
constexpr int MAX_COMPONENTS = 8;
struct MergeComp {
    const double* base;
    double scale;
    double from[4], to[4];  // limits per grid axis (P, R or L, V, K)
};
struct MergeArgs {
    MergeComp comp[MAX_COMPONENTS];
    int ncomp;
    int mean;                // 0: sum, 1: mean over finite component values
    const double* axis[4];   // grid coordinates of every point
};
void launch_merge_components(double* out, const MergeArgs& m, size_t n, cudaStream_t s);
// PSD lines interpolated from the old L* grid to the new one (scratch D, O: one
// field each); the result is copied into psd
void launch_remap(double* psd, const double* oldL, const double* newL, double* D, double* O,
                  const Dims& d, int* status, cudaStream_t s);

// Monotone mapping of doubles to unsigned 64-bit keys (for atomicMin on doubles).
__host__ __device__ __forceinline__ unsigned long long dkey(double v)
{
    unsigned long long u;
#ifdef __CUDA_ARCH__
    u = (unsigned long long)__double_as_longlong(v);
#else
    memcpy(&u, &v, 8);
#endif
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __forceinline__ double dkey_inv(unsigned long long k)
{
    unsigned long long u = (k & 0x8000000000000000ull) ? (k & ~0x8000000000000000ull) : ~k;
    double v;
    memcpy(&v, &u, 8);
    return v;
}

// --- Kalman filter -------------------------------------------------------------------
struct KFArgs {
    Dims d;
    double* psd;
    const double *Rg, *DLL, *G, *Ll, *Lu;
    double dll_scale;
    int Ll_t, Lu_t;
    const double* obs;   // device [P][R][V][K]
    double* Pa;          // [cols][R][R]
    double* work;        // [ctas][5][R][R]
    int* ticket;
    double dt, model_error, obs_error;
    int p_index;
    int* status;
};
int kf_ctas(const Dims& d, int p_index);
void launch_kf(const KFArgs& a, int nctas, cudaStream_t s);

}  // namespace verb
