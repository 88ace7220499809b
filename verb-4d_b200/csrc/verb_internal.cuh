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
    int32_t* ipiv;      // [sys][n]        0-based pivot rows
    double* work;       // [sys][n]        rhs / solution in unknown order (iK*V + iV)
    unsigned long long* negatives;  // optional: count of PSD < 0 written by the store kernel
    int* status;
};
size_t local_factor_smem(int V);
void launch_local_factor(const LocalArgs& a, cudaStream_t s);
void launch_local_rhs(const LocalArgs& a, bool from_work, cudaStream_t s);
void launch_local_solve(const LocalArgs& a, cudaStream_t s);
void launch_local_store(const LocalArgs& a, cudaStream_t s);
// r = b - A x for every system (A assembled on the fly in the reference's order)
void launch_local_residual(const LocalArgs& a, const double* b, const double* x, double* r,
                           cudaStream_t s);
// x += d; red[0] = max |d|, red[1] = max |x| (dkey-ordered, atomicMax)
void launch_local_update(const LocalArgs& a, double* x, const double* d, unsigned long long* red,
                         cudaStream_t s);
// unknowns of all systems (V*K*P*R, or the sum over trimmed systems)

// --- reductions / elementwise ---------------------------------------------------
void launch_negative_count(const double* psd, size_t n, unsigned long long* out, cudaStream_t s);
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
