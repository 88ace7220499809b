// Local (V,K) diffusion: banded LU with partial pivoting, factors cached in HBM.
//
// Reference: Diffusion_2D (src/Diffusion_2D.cpp:19-153) assembles a
// 9-diagonal operator over the unknown index in = iK*V + iV
// (AddBoundaries_2D and SecondDerivativeApproximation_2D,
// src/MatrixSolver.cpp:118-213, 439-494) and Lapack
// (src/MatrixSolver.cpp:223-340) factors it with dgbtrf (kl = ku = V+1) and
// solves with dgbtrs once per diffusion sub-step.  With LU_CACHING the
// factors are kept per (P,R) system and only recomputed when the local
// coefficients change (src/VERB4D_Solver.cpp:1091-1096).
//
// Kernels:
//  * local_factor_kernel: one CTA per system.  Rows of A are assembled on the
//    device with the reference's operation order (bit-identical matrix) and
//    factored by the unblocked banded LU of LAPACK's xGBTF2 (partial pivoting,
//    multipliers scaled by the reciprocal pivot, rank-1 updates as fused
//    multiply-adds).
//    The active (kl+1) x (kv+1) window lives in shared memory as a circular
//    buffer over rows and columns.  Output: L multipliers (Lf, column j
//    contiguous), U columns (Uf, rows j-kv..j contiguous) and 0-based pivots.
//  * local_rows_kernel + local_factor_rw_kernel: the same factorisation with
//    the window in registers (eight warps, bands up to V = 110): the rows are
//    assembled beforehand and parked in the L columns they precede, and
//    stream into a shared-memory ring by cp.async.  local_factor_kernel is
//    kept for wider bands.
//  * local_rhs_kernel / local_store_kernel: tile transposes between the PSD
//    slab [V][K] and the unknown order, forming RHS = B o f + C.
//  * local_solve_kernel: one warp per system, the forward (L, interleaved row
//    swaps as in xGBTRS) and backward (U, column-oriented as in xTBSV)
//    substitutions.  The solution window lives in shared memory; the factor
//    columns stream through a per-warp cp.async ring so that each warp keeps
//    several columns in flight.  This kernel moves the whole factor cache
//    once per sub-step and is HBM-bound.  local_solve_rw_kernel keeps the
//    solution window in registers instead.
//
// All arithmetic follows the CPU restatement of xGBTF2/xGBTRS/xTBSV operation
// by operation without FMA contraction (the file is compiled with
// -fmad=false) except the factorisation's rank-1 update, which both compute
// as one fused multiply-add per element (fma()), so factors, pivots and
// solutions are bit-identical to it.
#include "verb_internal.cuh"

namespace verb {

namespace {

// slot of diagonal offset (dx,dy): offset = dy*nx + dx
__device__ __forceinline__ int dslot(int dx, int dy) { return (dy + 1) * 3 + (dx + 1); }

struct SysView {
    const double *x, *y, *Dxx, *Dyy, *Dxy, *Dyx, *G, *S, *loss;
    const double *xl, *xu, *yl, *yu;
    int nx, ny;      // logical grid of the system (ny = K - k0)
    int ld;          // stride of the V index in the [V][K] fields (K)
    bool trimmed;    // lower K edge is the loss-cone edge (ConstantValue 0)
};

__device__ __forceinline__ int sys_k0(const LocalArgs& a, int sys) { return a.k0 ? a.k0[sys] : 0; }

// first unknown of system sys in the work / pivot arrays
__device__ __forceinline__ size_t sys_uoff(const LocalArgs& a, int sys)
{
    return a.uoff ? (size_t)a.uoff[sys] : (size_t)sys * a.d.V * a.d.K;
}

__device__ __forceinline__ SysView sys_view(const LocalArgs& a, int sys)
{
    const int k0 = sys_k0(a, sys);
    const size_t base = (size_t)sys * a.d.V * a.d.K + k0;
    SysView v;
    v.x = a.Vg + base;
    v.y = a.Kg + base;
    v.Dxx = a.DVV + base;
    v.Dyy = a.DKK + base;
    v.Dxy = a.DVK + base;
    v.Dyx = a.DKV + base;
    v.G = a.G + base;
    v.S = a.S + base;
    v.loss = a.loss + base;
    v.xl = a.Vl + (size_t)sys * a.d.K + k0;
    v.xu = a.Vu + (size_t)sys * a.d.K + k0;
    v.yl = a.Kl + (size_t)sys * a.d.V;
    v.yu = a.Ku + (size_t)sys * a.d.V;
    v.nx = a.d.V;
    v.ny = a.d.K - k0;
    v.ld = a.d.K;
    v.trimmed = k0 > 0;
    return v;
}

// SecondDerivativeApproximation_2D (src/MatrixSolver.cpp:439-494) adding into
// the 9 diagonal values of row (ix,iy).
__device__ __forceinline__ void sda2(double* r, const SysView& v, int ix, int iy, int dx1, int dy1,
                                     int dx2, int dy2, const double* D, double mult)
{
    const int ld = v.ld;
#define P2(a, b) ((a) * ld + (b))
    const double x0 = v.x[P2(ix, iy)] + v.y[P2(ix, iy)];
    const double x1 = v.x[P2(ix + dx1, iy + dy1)] + v.y[P2(ix + dx1, iy + dy1)];
    const double x2 = v.x[P2(ix + dx2, iy + dy2)] + v.y[P2(ix + dx2, iy + dy2)];
    const double x12 = v.x[P2(ix + dx1 + dx2, iy + dy1 + dy2)] + v.y[P2(ix + dx1 + dx2, iy + dy1 + dy2)];
    const double dh1 = x0 - x1;
    const double dh21 = x0 - x2;
    const double dh22 = x1 - x12;
    const double G0 = v.G[P2(ix, iy)], G1 = v.G[P2(ix + dx1, iy + dy1)];
    const double D0 = D[P2(ix, iy)], D1 = D[P2(ix + dx1, iy + dy1)];
    const double cp = mult / G0 / dh1;
    r[dslot(0, 0)] += +cp / dh21 * D0 * G0;
    r[dslot(dx2, dy2)] += -cp / dh21 * D0 * G0;
    r[dslot(dx1, dy1)] += -cp / dh22 * D1 * G1;
    r[dslot(dx1 + dx2, dy1 + dy2)] += +cp / dh22 * D1 * G1;
#undef P2
}

// One row of matr_A (src/Diffusion_2D.cpp:68-130).  Returns 0 or VERB_ERR_BC.
__device__ int assemble_row(const SysView& v, int types[4], double dt, int in, double r[9])
{
    const int nx = v.nx, ny = v.ny, ld = v.ld;
    const int ix = in % nx, iy = in / nx;
    const int p = ix * ld + iy;
#pragma unroll
    for (int s = 0; s < 9; s++) r[s] = 0.0;
    int t = -1, s1 = 0;
    double dh = 0.0;
    if (ix == 0 && nx >= 3) {
        t = types[0];
        s1 = dslot(1, 0);
        dh = v.x[p + ld] - v.x[p];
    } else if (ix == nx - 1 && nx >= 3) {
        t = types[1];
        s1 = dslot(-1, 0);
        dh = v.x[p] - v.x[p - ld];
    } else if (iy == 0 && ny >= 3) {
        t = v.trimmed ? VERB_BC_CONSTANT_VALUE : types[2];
        s1 = dslot(0, 1);
        dh = v.y[p + 1] - v.y[p];
    } else if (iy == ny - 1 && ny >= 3) {
        t = types[3];
        s1 = dslot(0, -1);
        dh = v.y[p] - v.y[p - 1];
    }
    if (t >= 0) {
        if (t == VERB_BC_CONSTANT_VALUE) {
            r[4] = 1;
            r[s1] = 0;
        } else if (t == VERB_BC_CONSTANT_DERIVATIVE) {
            r[4] = 1 / dh;
            r[s1] = -1 / dh;
        } else {
            return VERB_ERR_BC;
        }
        return 0;
    }
    r[4] += 1.0 / dt;
    r[4] -= v.loss[p];
    if (nx >= 3) {
        sda2(r, v, ix, iy, -1, 0, 1, 0, v.Dxx, -0.5);
        sda2(r, v, ix, iy, 1, 0, -1, 0, v.Dxx, -0.5);
    }
    if (ny >= 3) {
        sda2(r, v, ix, iy, 0, -1, 0, 1, v.Dyy, -0.5);
        sda2(r, v, ix, iy, 0, 1, 0, -1, v.Dyy, -0.5);
    }
    if (nx >= 3 && ny >= 3) {
        sda2(r, v, ix, iy, 0, -1, 1, 0, v.Dxy, -0.25);  // y_left,  x_right
        sda2(r, v, ix, iy, 0, 1, -1, 0, v.Dxy, -0.25);  // y_right, x_left
        sda2(r, v, ix, iy, 0, -1, -1, 0, v.Dxy, -0.25); // y_left,  x_left
        sda2(r, v, ix, iy, 0, 1, 1, 0, v.Dxy, -0.25);   // y_right, x_right
        sda2(r, v, ix, iy, -1, 0, 0, 1, v.Dyx, -0.25);  // x_left,  y_right (d/dy Dyx d/dx)
        sda2(r, v, ix, iy, 1, 0, 0, -1, v.Dyx, -0.25);  // x_right, y_left
        sda2(r, v, ix, iy, -1, 0, 0, -1, v.Dyx, -0.25); // x_left,  y_left
        sda2(r, v, ix, iy, 1, 0, 0, 1, v.Dyx, -0.25);   // x_right, y_right
    }
    return 0;
}

__device__ __forceinline__ bool skip_system(const LocalArgs& a, int sys)
{
    if (a.sel && !(a.sel[sys] & a.sel_mask)) return true;
    if (a.k0 && a.d.K - a.k0[sys] < 3) return true;  // trimmed below a solvable grid
    if (a.include_boundary) return false;
    const int r = sys % a.d.R;
    return r == 0 || r == a.d.R - 1;
}

constexpr int FACT_THREADS = 512;
constexpr int FACT_COLS = 7;  // columns per lane in the rank-1 update: kv + 1 <= 224 (V <= 111)
// Assembled rows are staged in a ring of STAGE_ROWS rows, a whole ring at a
// time (one row per thread), when the window's next entering row reaches a
// multiple of STAGE_ROWS.  256 rows (18 KB) still fit beside the window at
// V = 111.
constexpr int STAGE_ROWS = 256;

// The factorisation always runs in FP64 (pivots and multipliers as LAPACK's);
// T is the storage type of the factors: double, or float for the
// mixed-precision form, whose solves are refined in FP64.
template <typename T>
__global__ void __launch_bounds__(FACT_THREADS) local_factor_kernel(LocalArgs a)
{
    extern __shared__ double sm[];
    const int sys = blockIdx.x;
    if (skip_system(a, sys)) return;
    const int nx = a.d.V;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const int kl = a.kl, ku = a.kl, kv = a.kv;
    const int RW = kl + 1;          // window rows
    const int CW = kv + 1;          // window columns (row pitch)
    double* W = sm;                 // [RW][CW]
    double* mult = W + (size_t)RW * CW;  // [RW]
    double* colj = mult + RW;       // [RW]
    double* stage = colj + RW;      // [STAGE_ROWS][9]
    __shared__ int s_jp;
    __shared__ double s_piv;
    const SysView v = sys_view(a, sys);
    int types[4] = {a.Vl_t, a.Vu_t, a.Kl_t, a.Ku_t};
    const bool f32 = sizeof(T) == sizeof(float);
    const int klp = f32 ? a.klp32 : a.klp, kvp = f32 ? a.kvp32 : a.kvp;
    T* Lf = (f32 ? (T*)a.Lf32 : (T*)a.Lf) + u0 * klp;
    T* Uf = (f32 ? (T*)a.Uf32 : (T*)a.Uf) + u0 * kvp;
    int32_t* ip = a.ipiv + u0;
    const int tid = threadIdx.x;

    auto stage_rows = [&](int q0) {
        for (int q = q0 + tid; q < q0 + STAGE_ROWS && q < n; q += blockDim.x) {
            double r[9];
            const int st = assemble_row(v, types, a.dt, q, r);
            if (st) set_error(a.status, st);
#pragma unroll
            for (int s = 0; s < 9; s++) stage[(q & (STAGE_ROWS - 1)) * 9 + s] = r[s];
        }
    };
    // value of original row q at window column slot cs, when the window's
    // first column is c0 (column of slot cs is c0 + ((cs - c0%CW) mod CW))
    auto row_value = [&](int q, int col) -> double {
        const int d = col - q;
        const int dy = (d < -1) ? -1 : (d > 1 ? 1 : 0);
        const int dx = d - dy * nx;
        if (dx < -1 || dx > 1 || col < 0 || col >= n) return 0.0;
        return stage[(q & (STAGE_ROWS - 1)) * 9 + dslot(dx, dy)];
    };

    for (int i = tid; i < RW * CW; i += blockDim.x) W[i] = 0.0;
    stage_rows(0);
    __syncthreads();
    // rows 0..kl into the window (columns 0..kv)
    for (int i = tid; i < RW * CW; i += blockDim.x) {
        const int q = i / CW, c = i - q * CW;
        if (q < n) W[q * CW + c] = row_value(q, c);
    }
    __syncthreads();

    int ju = 0;
    for (int j = 0; j < n; j++) {
        const int km = min(kl, n - 1 - j);
        const int rsj = j % RW, csj = j % CW;
        // [A] pivot: first index of max |column j| over rows j..j+km (idamax)
        if (tid < 32) {
            double best = -1.0;
            int bi = 0;
            for (int i = tid; i <= km; i += 32) {
                const double val = W[((j + i) % RW) * CW + csj];
                colj[i] = val;
                const double av = fabs(val);
                if (av > best) {
                    best = av;
                    bi = i;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (tid == 0) {
                // idamax: a NaN first element is the maximum (nothing compares
                // greater), elsewhere NaN never is
                if (colj[0] != colj[0]) bi = 0;
                s_jp = bi;
                s_piv = W[((j + bi) % RW) * CW + csj];
                ip[j] = j + bi;
            }
        }
        __syncthreads();
        const int jp = s_jp;
        const double piv = s_piv;
        const bool nz = piv != 0.0;
        if (nz) {
            ju = max(ju, min(j + ku + jp, n - 1));
            // [B] multipliers (from the pre-swap column) and the row swap
            const double rcp = 1.0 / piv;
            for (int i = 1 + tid; i <= km; i += blockDim.x) {
                const double val = (i == jp) ? colj[0] : colj[i];
                const double m = val * rcp;
                mult[i] = m;
                Lf[(size_t)j * klp + (i - 1)] = (T)m;
            }
            if (jp != 0) {
                const int rp = (j + jp) % RW;
                for (int c = j + tid; c <= ju; c += blockDim.x) {
                    const int cs = c % CW;
                    const double t = W[rsj * CW + cs];
                    W[rsj * CW + cs] = W[rp * CW + cs];
                    W[rp * CW + cs] = t;
                }
            }
        } else {
            set_error(a.status, VERB_ERR_PIVOT);
            for (int i = 1 + tid; i <= km; i += blockDim.x) Lf[(size_t)j * klp + (i - 1)] = (T)colj[i];
        }
        __syncthreads();
        // [C] U row j out; rank-1 update of rows j+1..j+km, columns j+1..ju
        for (int c = j + tid; c <= ju && c <= j + kv; c += blockDim.x)
            Uf[(size_t)c * kvp + (kv - (c - j))] = (T)W[rsj * CW + (c % CW)];
        if (nz && km > 0 && ju > j) {
            // warp w updates rows w+1, w+1+nw, ...; lane l columns j+1+l+32k.
            // The pivot row's values (negated, as xGER's temp) stay in
            // registers; window slots advance by wrap, not modulo.
            const int ncol = ju - j;  // <= kv <= 32 * FACT_COLS
            const int lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
            double ty[FACT_COLS];
            int csl[FACT_COLS];
            int cs = (j + 1 + lane) % CW;
#pragma unroll
            for (int k = 0; k < FACT_COLS; k++) {
                csl[k] = cs;
                ty[k] = (lane + 32 * k < ncol) ? -W[rsj * CW + cs] : 0.0;
                cs += 32;
                while (cs >= CW) cs -= CW;
            }
            int r = (j + 1 + wid) % RW;
            for (int i = 1 + wid; i <= km; i += nw) {
                const double m = mult[i];
                double* Wr = W + (size_t)r * CW;
#pragma unroll
                for (int k = 0; k < FACT_COLS; k++)
                    if (ty[k] != 0.0) {
                        double* w = Wr + csl[k];
                        *w = fma(m, ty[k], *w);  // xGER: A(i,k) + x(i)*temp, temp = -y(k), fused
                    }
                r += nw;
                while (r >= RW) r -= RW;
            }
        }
        __syncthreads();
        // [D] slide: row slot j <- original row j+kl+1, column slot j <- column j+kv+1
        const int q = j + kl + 1;
        if (q < n && (q & (STAGE_ROWS - 1)) == 0 && q >= STAGE_ROWS) {
            stage_rows(q);
            __syncthreads();
        }
        for (int cs = tid; cs < CW; cs += blockDim.x) {
            double val = 0.0;
            if (q < n) {
                const int c0 = j + 1;
                const int col = c0 + ((cs - (c0 % CW)) % CW + CW) % CW;
                val = row_value(q, col);
            }
            W[rsj * CW + cs] = val;
        }
        for (int rs = tid; rs < RW; rs += blockDim.x)
            if (rs != rsj) W[rs * CW + csj] = 0.0;
        __syncthreads();
    }
}

// The same factorisation with the (kl+1) x (kv+1) circular window held in
// registers for the whole run.  NW warps (eight in use); warp w owns row slots
// w + NW q (q < NR), lane l column slots l + 32 k (k < NC), value R[q][k].  Per column
// j there are two block barriers:
//   top   the lanes that own column slot j % CW search their own rows for the
//         first maximum of |x| (they updated those values themselves at
//         column j-1, so no barrier is needed before the search) and post the
//         column and their warp's candidate;
//   B1    every thread combines the NW candidates (idamax: first maximum,
//         NaN skipped unless it is the first entry); the multipliers go to
//         Lf; every thread forms one window slot of the row that enters at
//         the next column; the owners of row j and of the pivot row post them;
//   B2    the swap over columns j..ju in the owners' registers, U row j out,
//         the rank-1 update of every owned slot (multipliers from the posted
//         column, the pivot row from shared memory), and the slide: column
//         slot j % CW is cleared, row slot j % RW takes row j+kl+1 (formed at
//         the previous column).
// The row and column slots of the pivot step are reached through a switch on
// their index (registers cannot be indexed at run time), so only the rank-1
// update touches every slot.  Every element sees the same operations in the
// same order as in local_factor_kernel (LAPACK's xGBTF2, the rank-1 update
// fused): factors and pivots are bit-identical, and the update costs no
// shared-memory traffic.
// f(R[q]) for a run-time q < NR
template <int NR, int NC, typename F>
__device__ __forceinline__ void frw_row(double (&R)[NR][NC], int q, F&& f)
{
    switch (q) {
#define VERB_ROW(Q) \
    case Q:         \
        if constexpr (Q < NR) f(R[Q]); \
        break;
        VERB_ROW(0) VERB_ROW(1) VERB_ROW(2) VERB_ROW(3) VERB_ROW(4) VERB_ROW(5) VERB_ROW(6)
        VERB_ROW(7) VERB_ROW(8) VERB_ROW(9) VERB_ROW(10) VERB_ROW(11) VERB_ROW(12) VERB_ROW(13)
#undef VERB_ROW
        default: break;
    }
}

template <int K, int NR, int NC, typename F>
__device__ __forceinline__ void frw_col_k(double (&R)[NR][NC], F& f)
{
#pragma unroll
    for (int q = 0; q < NR; q++) f(q, R[q][K]);
}

// f(q, R[q][k]) for every q, for a run-time k < NC
template <int NR, int NC, typename F>
__device__ __forceinline__ void frw_col(double (&R)[NR][NC], int k, F&& f)
{
    switch (k) {
#define VERB_COL(K) \
    case K:         \
        if constexpr (K < NC) frw_col_k<K>(R, f); \
        break;
        VERB_COL(0) VERB_COL(1) VERB_COL(2) VERB_COL(3) VERB_COL(4) VERB_COL(5) VERB_COL(6)
#undef VERB_COL
        default: break;
    }
}

// Every row of A, assembled once before the factorisation and parked in the
// L-factor column of the same index: row q's nine diagonal values go to
// Lf[q][0..8] (as FP64, also when the factors are FP32).  local_factor_rw_kernel
// reads row q at column q-kl-1 (or for the first window) and writes L column q
// only at column q, so the parked row is always read before it is overwritten.
template <typename T>
__device__ __forceinline__ double* frw_row_slot(const LocalArgs& a, size_t u)
{
    if constexpr (sizeof(T) == sizeof(float)) return (double*)(a.Lf32 + u * a.klp32);
    else return a.Lf + u * a.klp;
}

template <typename T>
__global__ void local_rows_kernel(LocalArgs a)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const SysView v = sys_view(a, sys);
    int types[4] = {a.Vl_t, a.Vu_t, a.Kl_t, a.Ku_t};
    double r[9];
    const int st = assemble_row(v, types, a.dt, q, r);
    if (st) set_error(a.status, st);
    double* dst = frw_row_slot<T>(a, sys_uoff(a, sys) + q);
#pragma unroll
    for (int s2 = 0; s2 < 9; s2++) dst[s2] = r[s2];
}

__device__ __forceinline__ void cp_async_8(double* dst, const double* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void frw_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void frw_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <typename T, int NR, int NC, int NW>
__global__ void __launch_bounds__(NW * 32, 1) local_factor_rw_kernel(LocalArgs a)
{
    extern __shared__ double sm[];
    const int sys = blockIdx.x;
    if (skip_system(a, sys)) return;
    const int nx = a.d.V;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const int kl = a.kl, ku = a.kl, kv = a.kv;
    const int RW = kl + 1;          // window rows
    const int CW = kv + 1;          // window columns
    double* stage = sm;             // [2 STAGE_ROWS][9] ring of parked rows
    double* rowA = stage + (size_t)2 * STAGE_ROWS * 9;  // [CW] row j before the swap
    double* rowB = rowA + CW;       // [CW] the pivot row (row j after the swap)
    double* colv = rowB + CW;       // [2][RW] column j by offset, by parity of j
    double* nrow = colv + 2 * RW;   // [2][CW] the window row that enters at column j, by parity
    __shared__ double s_best[NW];
    __shared__ int s_bi[NW];
    const bool f32 = sizeof(T) == sizeof(float);
    const int klp = f32 ? a.klp32 : a.klp, kvp = f32 ? a.kvp32 : a.kvp;
    T* Lf = (f32 ? (T*)a.Lf32 : (T*)a.Lf) + u0 * klp;
    T* Uf = (f32 ? (T*)a.Uf32 : (T*)a.Uf) + u0 * kvp;
    int32_t* ip = a.ipiv + u0;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

    // rows 256 b .. 256 b + 255 (parked by local_rows_kernel) into ring half
    // b % 2, asynchronously
    const double* rows = frw_row_slot<T>(a, u0);
    const size_t rstride = f32 ? (size_t)a.klp32 / 2 : (size_t)a.klp;  // doubles
    auto fetch_block = [&](int b) {
        const int q0 = b * STAGE_ROWS;
        const int cnt = min(STAGE_ROWS, n - q0) * 9;
        for (int e = tid; e < cnt; e += blockDim.x) {
            const int q = q0 + e / 9, s2 = e - (e / 9) * 9;
            cp_async_8(stage + (size_t)(q & (2 * STAGE_ROWS - 1)) * 9 + s2, rows + q * rstride + s2);
        }
        frw_commit();
    };
    auto row_value = [&](int q, int col) -> double {
        const int d = col - q;
        const int dy = (d < -1) ? -1 : (d > 1 ? 1 : 0);
        const int dx = d - dy * nx;
        if (dx < -1 || dx > 1 || col < 0 || col >= n) return 0.0;
        return stage[(q & (2 * STAGE_ROWS - 1)) * 9 + dslot(dx, dy)];
    };

    double R[NR][NC];
    fetch_block(0);
    if (n > STAGE_ROWS) fetch_block(1);
    frw_wait_all();
    __syncthreads();
    // the row entering at column jj (row jj+kl+1) over window slots: slot cs
    // holds column jj+1+((cs-(jj+1)) mod CW); cjj = jj mod CW
    auto fill_row = [&](int jj, int cjj) {
        const int qr = jj + kl + 1;
        for (int cs = tid; cs < CW; cs += blockDim.x) {
            int c = cs - cjj - 1;
            if (c < 0) c += CW;
            nrow[(jj & 1) * CW + cs] = qr < n ? row_value(qr, jj + 1 + c) : 0.0;
        }
    };
    fill_row(0, 0);
#pragma unroll
    for (int q = 0; q < NR; q++)
#pragma unroll
        for (int k = 0; k < NC; k++) {
            const int rs = wid + NW * q, cs = lane + 32 * k;
            R[q][k] = (rs < RW && cs < CW && rs < n) ? row_value(rs, cs) : 0.0;
        }

    int ju = 0;
    int rj = 0, cj = 0;   // window slots of row j and column j (j mod RW, j mod CW)
    for (int j = 0; j < n; j++) {
        const int km = min(kl, n - 1 - j);
        const int lc = cj & 31, kc = cj >> 5;
        double* cv = colv + (j & 1) * RW;
        // [top] this warp's candidate pivot in column j
        if (lane == lc) {
            // four interleaved first-maximum chains (rows q mod 4), merged at
            // the end with the same rule: a shorter dependency chain than one
            // pass over the thread's NR rows
            double best[4] = {-1.0, -1.0, -1.0, -1.0};
            int bi[4] = {1 << 30, 1 << 30, 1 << 30, 1 << 30};
            frw_col(R, kc, [&](int q, double& val) {
                const int rs = wid + NW * q;
                int i = rs - rj;
                if (i < 0) i += RW;
                if (rs < RW && i <= km) {
                    cv[i] = val;
                    const double av = fabs(val);
                    if (av > best[q & 3] || (av == best[q & 3] && i < bi[q & 3])) {
                        best[q & 3] = av;
                        bi[q & 3] = i;
                    }
                }
            });
#pragma unroll
            for (int c = 1; c < 4; c++)
                if (best[c] > best[0] || (best[c] == best[0] && bi[c] < bi[0])) {
                    best[0] = best[c];
                    bi[0] = bi[c];
                }
            s_best[wid] = best[0];
            s_bi[wid] = bi[0];
        }
        __syncthreads();
        // [B1] the pivot, the multipliers, the rows of the swap.  The NW
        // candidates are combined by shuffles in every warp (lanes 0..NW-1
        // hold them; the other lanes of each group carry empty candidates).
        double best = lane < NW ? s_best[lane] : -1.0;
        int jp = lane < NW ? s_bi[lane] : 1 << 30;
        constexpr int GROUP = NW > 16 ? 32 : (NW > 8 ? 16 : 8);  // power of two >= NW
#pragma unroll
        for (int o = GROUP / 2; o > 0; o >>= 1) {
            const double b = __shfl_xor_sync(0xffffffffu, best, o);
            const int bi = __shfl_xor_sync(0xffffffffu, jp, o);
            if (b > best || (b == best && bi < jp)) {
                best = b;
                jp = bi;
            }
        }
        jp = __shfl_sync(0xffffffffu, jp, 0);
        // idamax: a NaN first element is the maximum (nothing compares
        // greater), elsewhere NaN never is
        const double c0 = cv[0];
        if (c0 != c0 || jp > km) jp = 0;
        const double piv = cv[jp];
        const bool nz = piv != 0.0;
        const bool swap = nz && jp != 0;
        const int rp = rj + jp < RW ? rj + jp : rj + jp - RW;
        if (tid == 0) ip[j] = j + jp;
        double rcp = 0.0;
        if (nz) {
            ju = max(ju, min(j + ku + jp, n - 1));
            rcp = 1.0 / piv;
            for (int i = 1 + tid; i <= km; i += blockDim.x) {
                const double val = (i == jp) ? c0 : cv[i];
                Lf[(size_t)j * klp + (i - 1)] = (T)(val * rcp);
            }
        } else {
            if (tid == 0) set_error(a.status, VERB_ERR_PIVOT);
            for (int i = 1 + tid; i <= km; i += blockDim.x) Lf[(size_t)j * klp + (i - 1)] = (T)cv[i];
        }
        {
            // next column's entering row; its ring block must be present
            const int qf = j + 1 + kl + 1;
            if (j + 1 < n && qf < n && (qf & (STAGE_ROWS - 1)) == 0 && qf >= STAGE_ROWS) {
                frw_wait_all();
                __syncthreads();
                if (qf + STAGE_ROWS < n) fetch_block(qf / STAGE_ROWS + 1);
            }
            if (j + 1 < n) fill_row(j + 1, cj + 1 == CW ? 0 : cj + 1);
        }
        const bool own_j = wid == rj % NW;
        const bool own_p = swap && wid == rp % NW;
        const int qj = rj / NW, qp = rp / NW;
        auto post = [&](double* dst) {
            return [&, dst](double (&row)[NC]) {
#pragma unroll
                for (int k = 0; k < NC; k++) {
                    const int cs = lane + 32 * k;
                    if (cs < CW) dst[cs] = row[k];
                }
            };
        };
        if (own_j) frw_row(R, qj, post(swap ? rowA : rowB));
        if (own_p) frw_row(R, qp, post(rowB));
        __syncthreads();
        // [B2] swap, U row j, rank-1 update, slide
        const int ncol = ju - j;   // columns j+1..ju take the update
        int cofs[NC];              // column offset c - j of each owned slot
#pragma unroll
        for (int k = 0; k < NC; k++) {
            int c = lane + 32 * k - cj;
            if (c < 0) c += CW;
            cofs[k] = c;
        }
        if (swap) {
            auto take = [&](const double* src) {
                return [&, src](double (&row)[NC]) {
#pragma unroll
                    for (int k = 0; k < NC; k++) {
                        const int cs = lane + 32 * k;
                        if (cs < CW && cofs[k] <= ncol) row[k] = src[cs];
                    }
                };
            };
            if (own_j) frw_row(R, qj, take(rowB));
            if (own_p) frw_row(R, qp, take(rowA));
        }
        for (int c = j + tid; c <= ju && c <= j + kv; c += blockDim.x) {
            const int cs = cj + (c - j) < CW ? cj + (c - j) : cj + (c - j) - CW;
            Uf[(size_t)c * kvp + (kv - (c - j))] = (T)rowB[cs];
        }
        if (nz && km > 0 && ncol > 0) {
            double ty[NC];
#pragma unroll
            for (int k = 0; k < NC; k++) {
                const int cs = lane + 32 * k;
                ty[k] = (cs < CW && cofs[k] >= 1 && cofs[k] <= ncol) ? -rowB[cs] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < NR; q++) {
                const int rs = wid + NW * q;
                int i = rs - rj;
                if (i < 0) i += RW;
                if (rs >= RW || i < 1 || i > km) continue;
                const double m = ((i == jp) ? c0 : cv[i]) * rcp;
                // xGER: A(i,k) + x(i)*temp with temp = -y(k), one fused
                // multiply-add, skipped where temp = 0 (as a select, so that
                // the lanes do not diverge)
#pragma unroll
                for (int k = 0; k < NC; k++) {
                    const double u = fma(m, ty[k], R[q][k]);
                    R[q][k] = ty[k] != 0.0 ? u : R[q][k];
                }
            }
        }
        // column slot cj now holds column j+CW, zero in every row but the new one
        if (lane == lc) frw_col(R, kc, [](int, double& val) { val = 0.0; });
        // row slot rj <- row j+kl+1 over columns j+1..j+CW (slot cs holds
        // column j+1+((cs-(j+1)) mod CW))
        if (own_j)
            frw_row(R, qj, [&](double (&row)[NC]) {
#pragma unroll
                for (int k = 0; k < NC; k++) {
                    const int cs = lane + 32 * k;
                    row[k] = cs < CW ? nrow[(j & 1) * CW + cs] : 0.0;
                }
            });
        if (++rj == RW) rj = 0;
        if (++cj == CW) cj = 0;
    }
}

// RHS = B o f + C in unknown order (src/MatrixSolver.cpp:309-320), through a
// 32x32 shared-memory tile transpose of the [V][K] slab.
__global__ void local_rhs_kernel(LocalArgs a, int from_work)
{
    __shared__ double tile[32][33];
    const int sys = blockIdx.z;
    if (skip_system(a, sys)) return;
    const int V = a.d.V, K = a.d.K;
    const int kz = sys_k0(a, sys), ny = K - kz;  // unknowns: pitch-angle indices kz..K-1
    const double* psd = a.psd + (size_t)sys * V * K;
    double* w = a.work + sys_uoff(a, sys);
    const int v0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    if (!from_work) {
        for (int r = ty; r < 32; r += 8) {
            const int iv = v0 + r, ik = k0 + tx;
            if (iv < V && ik < K) tile[r][tx] = psd[(size_t)iv * K + ik];
        }
    } else {
        for (int r = ty; r < 32; r += 8) {
            const int ik = k0 + r, iv = v0 + tx;
            if (iv < V && ik >= kz && ik < K) tile[tx][r] = w[(size_t)(ik - kz) * V + iv];
        }
    }
    __syncthreads();
    const SysView sv = sys_view(a, sys);
    const double bint = 0.0 + 1.0 / a.dt;
    const double ls = (double)a.local_sources;
    for (int r = ty; r < 32; r += 8) {
        const int ik = k0 + r, iv = v0 + tx;
        if (iv >= V || ik >= K || ik < kz) continue;
        const int ix = iv, iy = ik - kz;
        double b, c;
        if (ix == 0 && V >= 3) {
            b = 0.0;
            c = sv.xl[iy];
        } else if (ix == V - 1 && V >= 3) {
            b = 0.0;
            c = sv.xu[iy];
        } else if (iy == 0 && ny >= 3) {
            b = 0.0;
            c = sv.trimmed ? 0.0 : sv.yl[ix];
        } else if (iy == ny - 1 && ny >= 3) {
            b = 0.0;
            c = sv.yu[ix];
        } else {
            b = bint;
            c = 0.0;
            c += sv.S[(size_t)ix * K + iy] * ls;
        }
        double rhs = tile[tx][r];
        rhs *= b;
        rhs += c;
        w[(size_t)iy * V + iv] = rhs;
    }
}

__global__ void local_store_kernel(LocalArgs a)
{
    __shared__ double tile[32][33];
    const int sys = blockIdx.z;
    if (skip_system(a, sys)) return;
    const int V = a.d.V, K = a.d.K;
    const int kz = sys_k0(a, sys);
    double* psd = a.psd + (size_t)sys * V * K;
    const double* w = a.work + sys_uoff(a, sys);
    const int v0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const int ik = k0 + r, iv = v0 + tx;
        if (iv < V && ik >= kz && ik < K) tile[tx][r] = w[(size_t)(ik - kz) * V + iv];
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int iv = v0 + r, ik = k0 + tx;
        if (iv < V && ik >= kz && ik < K) psd[(size_t)iv * K + ik] = tile[r][tx];
    }
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// cnt 16-byte chunks, cnt <= 32 * MAXT, by the 32 lanes of a warp: a fixed
// number of predicated copies instead of a loop with a run-time trip count
template <int MAXT>
__device__ __forceinline__ void warp_copy16(void* dst, const void* src, int cnt, int lane)
{
#pragma unroll
    for (int t = 0; t < MAXT; t++) {
        const int c = lane + 32 * t;
        if (c < cnt) cp_async16((char*)dst + 16 * c, (const char*)src + 16 * c);
    }
}
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Solve variants: warps (systems) per CTA, L and U factor columns in flight
// per warp.  More columns in flight hide more latency per warp but take
// shared memory that would otherwise hold more resident warps; the best
// trade depends on the grid, so the autotuner picks one per context.
// The second group keeps the right-hand-side window in registers instead of
// shared memory (local_solve_rw_kernel).
// The last group caps the registers (at least minb CTAs per SM: 36 resident
// systems per SM) so that a 48 x 101 grid's 4848 systems are resident in one
// wave instead of 32 per SM and a tail of 112.
struct SolveShape {
    int warps, fwd, bwd, rw;
    int minb = 1;
};
constexpr SolveShape SOLVE_SHAPES[] = {
    {4, 4, 2, 0},  {4, 6, 3, 0},  {2, 6, 4, 0},  {2, 8, 6, 0},  {1, 8, 6, 0},  {1, 12, 8, 0},
    {1, 12, 10, 0}, {1, 16, 12, 0}, {1, 24, 16, 0},
    {4, 4, 3, 1},  {4, 6, 4, 1},  {2, 8, 6, 1},  {2, 12, 8, 1}, {1, 12, 8, 1}, {1, 16, 12, 1},
    {4, 4, 2, 1, 9}, {2, 6, 3, 1, 18}, {4, 6, 3, 1, 9}};
constexpr int N_SOLVE_SHAPES = sizeof(SOLVE_SHAPES) / sizeof(SOLVE_SHAPES[0]);
constexpr int FWD_WIN = 128;   // >= kl + 1
constexpr int BWD_WIN = 256;   // >= kv + 1

// ring of factor columns per warp, in doubles (16-byte multiples)
__host__ __device__ constexpr size_t solve_ring_doubles(int klp, int kvp, int esize, int fd, int bd)
{
    return ((size_t)(fd * klp > bd * kvp ? fd * klp : bd * kvp) * esize + 15) / 16 * 2;
}

// T: storage type of the factors.  The substitutions run in FP64 either way
// (float factors are widened as they are used).
template <typename T, int SOLVE_WARPS, int FWD_DEPTH, int BWD_DEPTH>
__global__ void __launch_bounds__(SOLVE_WARPS * 32) local_solve_kernel(LocalArgs a, int nsys)
{
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sys = blockIdx.x * SOLVE_WARPS + warp;
    if (sys >= nsys || skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const bool f32 = sizeof(T) == sizeof(float);
    const int kl = a.kl, kv = a.kv, klp = f32 ? a.klp32 : a.klp, kvp = f32 ? a.kvp32 : a.kvp;
    constexpr int VEC = 16 / sizeof(T);  // elements per 16-byte cp.async
    const size_t per_warp = BWD_WIN + solve_ring_doubles(klp, kvp, sizeof(T), FWD_DEPTH, BWD_DEPTH);
    double* win = sm + (size_t)warp * per_warp;
    T* ring = (T*)(win + BWD_WIN);
    double* w = a.work + u0;
    const T* Lf = (f32 ? (const T*)a.Lf32 : (const T*)a.Lf) + u0 * klp;
    const T* Uf = (f32 ? (const T*)a.Uf32 : (const T*)a.Uf) + u0 * kvp;
    const int32_t* ip = a.ipiv + u0;

    // ---------------- forward: L with interleaved row interchanges (xGBTRS) --------
    for (int i = lane; i < FWD_WIN && i < n; i += 32) win[i] = w[i];
    auto issue_L = [&](int col) {
        if (col < n - 1) {
            T* dst = ring + (col % FWD_DEPTH) * klp;
            const T* src = Lf + (size_t)col * klp;
            warp_copy16<FWD_WIN * 8 / 16 / 32>(dst, src, klp / VEC, lane);
        }
    };
    for (int c = 0; c < FWD_DEPTH; c++) {
        issue_L(c);
        cp_commit();
    }
    int pv_cur = (lane < n) ? ip[lane] : 0;
    int pv_next = (32 + lane < n) ? ip[32 + lane] : 0;
    __syncwarp();
    for (int j = 0; j < n - 1; j++) {
        if ((j & 31) == 0 && j > 0) {
            pv_cur = pv_next;
            const int nx = j + 32 + lane;
            pv_next = (nx < n) ? ip[nx] : 0;
        }
        cp_wait<FWD_DEPTH - 1>();
        __syncwarp();
        const int lm = min(kl, n - 1 - j);
        const int l = __shfl_sync(0xffffffffu, pv_cur, j & 31);
        const double bj_old = win[j & (FWD_WIN - 1)];
        const double bl = win[l & (FWD_WIN - 1)];
        const double bj = (l != j) ? bl : bj_old;
        const T* Lc = ring + (j % FWD_DEPTH) * klp;
        const double tmp = -bj;
        const bool upd = bj != 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int t = lane + 32 * k;
            const int i = j + 1 + t;
            if (t < lm) {
                double cur = (i == l) ? bj_old : win[i & (FWD_WIN - 1)];
                if (upd) cur = cur + (double)Lc[t] * tmp;  // xGER in xGBTRS
                win[i & (FWD_WIN - 1)] = cur;
            }
        }
        __syncwarp();
        if (lane == 0) {
            w[j] = bj;
            if (j + FWD_WIN < n) cp_async8(&win[j & (FWD_WIN - 1)], &w[j + FWD_WIN]);
        }
        issue_L(j + FWD_DEPTH);
        cp_commit();
    }
    cp_wait<0>();
    __syncwarp();
    if (lane == 0) w[n - 1] = win[(n - 1) & (FWD_WIN - 1)];
    __syncwarp();

    // ---------------- backward: U, column oriented (xTBSV 'U','N','N') ------------
    for (int i = n - 1 - lane; i >= 0 && i > n - 1 - BWD_WIN; i -= 32) win[i & (BWD_WIN - 1)] = w[i];
    auto issue_U = [&](int col) {
        if (col >= 0) {
            T* dst = ring + ((n - 1 - col) % BWD_DEPTH) * kvp;
            const T* src = Uf + (size_t)col * kvp;
            warp_copy16<BWD_WIN * 8 / 16 / 32>(dst, src, kvp / VEC, lane);
        }
    };
    for (int c = 0; c < BWD_DEPTH; c++) {
        issue_U(n - 1 - c);
        cp_commit();
    }
    __syncwarp();
    for (int j = n - 1; j >= 0; j--) {
        cp_wait<BWD_DEPTH - 1>();
        __syncwarp();
        const T* Uc = ring + ((n - 1 - j) % BWD_DEPTH) * kvp;
        double bj = win[j & (BWD_WIN - 1)];
        if (bj != 0.0) {
            bj = bj / (double)Uc[kv];
#pragma unroll
            for (int k = 0; k < 7; k++) {
                const int d = 1 + lane + 32 * k;
                const int i = j - d;
                if (d <= kv && i >= 0) {
                    double* x = &win[i & (BWD_WIN - 1)];
                    *x = *x - bj * (double)Uc[kv - d];  // xTBSV: X(I) - TEMP*A(L+I,J)
                }
            }
        }
        __syncwarp();
        if (lane == 0) {
            w[j] = bj;
            if (j - BWD_WIN >= 0) cp_async8(&win[j & (BWD_WIN - 1)], &w[j - BWD_WIN]);
        }
        issue_U(j - BWD_DEPTH);
        cp_commit();
    }
    cp_wait<0>();
}

// The same solve with the right-hand-side window in registers.  Forward
// (xGBTRS with interleaved row interchanges), at column j the window holds
// positions j .. j+32FS-1: lane i's slot m holds position
// j + ((i - j) & 31) + 32m, so the updates of column j (positions
// j+1 .. j+lm) touch every lane's slots in place, the pivot row l is read from
// lane l & 31, slot (l - j) >> 5, and only lane j & 31 shifts its slots down
// (position j leaves, position j + 32FS enters) when the column is done.
// Backward (xTBSV), at column j the window holds j .. j-32BS+1 the same way
// downwards.  The factor columns still stream through a per-warp cp.async
// ring in shared memory (read with rotated, conflict-free accesses), and the
// right-hand-side entries that enter the window are staged with them.  The
// operations and their order are those of local_solve_kernel, so the result is
// bit-identical; what changes is that the window no longer costs shared-memory
// loads and stores per column, which the old kernel's column chain waited on.
template <typename T, int SOLVE_WARPS, int FWD_DEPTH, int BWD_DEPTH, int FS, int BS, int MINB>
__global__ void __launch_bounds__(SOLVE_WARPS * 32, MINB) local_solve_rw_kernel(LocalArgs a, int nsys)
{
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sys = blockIdx.x * SOLVE_WARPS + warp;
    if (sys >= nsys || skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const bool f32 = sizeof(T) == sizeof(float);
    const int kl = a.kl, kv = a.kv, klp = f32 ? a.klp32 : a.klp, kvp = f32 ? a.kvp32 : a.kvp;
    constexpr int VEC = 16 / sizeof(T);
    constexpr int FWIN = 32 * FS, BWIN = 32 * BS;
    constexpr int STAGE = (FWD_DEPTH > BWD_DEPTH ? FWD_DEPTH : BWD_DEPTH) + 1 & ~1;
    const size_t per_warp = STAGE + solve_ring_doubles(klp, kvp, sizeof(T), FWD_DEPTH, BWD_DEPTH);
    double* stage = sm + (size_t)warp * per_warp;  // entering right-hand-side entries
    T* ring = (T*)(stage + STAGE);
    double* w = a.work + u0;
    const T* Lf = (f32 ? (const T*)a.Lf32 : (const T*)a.Lf) + u0 * klp;
    const T* Uf = (f32 ? (const T*)a.Uf32 : (const T*)a.Uf) + u0 * kvp;
    const int32_t* ip = a.ipiv + u0;

    // ---------------- forward: L with interleaved row interchanges (xGBTRS) --------
    double s[FS > BS ? FS : BS];
#pragma unroll
    for (int m = 0; m < FS; m++) {
        const int p = lane + 32 * m;
        s[m] = p < n ? w[p] : 0.0;
    }
    // column col's multipliers, and b[col + FWIN] (which enters the window
    // when column col is done)
    // (slot: col mod FWD_DEPTH, kept as a running index by the caller)
    auto issue_L = [&](int col, int slot) {
        if (col < n - 1) {
            T* dst = ring + slot * klp;
            const T* src = Lf + (size_t)col * klp;
            warp_copy16<FWD_WIN * 8 / 16 / 32>(dst, src, klp / VEC, lane);
            if (lane == 0) {
                double* st = &stage[slot];
                if (col + FWIN < n) cp_async8(st, &w[col + FWIN]);
                else *st = 0.0;
            }
        }
    };
    for (int c = 0; c < FWD_DEPTH; c++) {
        issue_L(c, c);
        cp_commit();
    }
    int fslot = 0;  // j mod FWD_DEPTH
    int pv_cur = (lane < n) ? ip[lane] : 0;
    int pv_next = (32 + lane < n) ? ip[32 + lane] : 0;
    for (int j = 0; j < n - 1; j++) {
        if ((j & 31) == 0 && j > 0) {
            pv_cur = pv_next;
            const int nx = j + 32 + lane;
            pv_next = (nx < n) ? ip[nx] : 0;
        }
        cp_wait<FWD_DEPTH - 1>();
        __syncwarp();
        const int lm = min(kl, n - 1 - j);
        const int l = __shfl_sync(0xffffffffu, pv_cur, j & 31);
        const double bj_old = __shfl_sync(0xffffffffu, s[0], j & 31);
        double bj = bj_old;
        if (l != j) {  // the same for the whole warp: an interchange
            const int sl = (l - j) >> 5;  // slot of position l in lane l & 31
            double v = s[0];
#pragma unroll
            for (int m = 1; m < FS; m++) v = (sl == m) ? s[m] : v;
            bj = __shfl_sync(0xffffffffu, v, l & 31);
            if (lane == (l & 31)) {
#pragma unroll
                for (int m = 0; m < FS; m++)
                    if (sl == m) s[m] = bj_old;
            }
        }
        if (bj != 0.0) {
            const T* Lc = ring + fslot * klp;
            const double tmp = -bj;
            const int o = (lane - j) & 31;
#pragma unroll
            for (int m = 0; m < FS; m++) {
                const int e = o + 32 * m - 1;  // position j + 1 + e; 0 <= e < lm
                if ((unsigned)e < (unsigned)lm) s[m] = s[m] + (double)Lc[e] * tmp;  // xGER in xGBTRS
            }
        }
        if (lane == (j & 31)) {
            w[j] = bj;
#pragma unroll
            for (int m = 0; m + 1 < FS; m++) s[m] = s[m + 1];
            s[FS - 1] = stage[fslot];
        }
        __syncwarp();
        issue_L(j + FWD_DEPTH, fslot);
        cp_commit();
        fslot = fslot + 1 == FWD_DEPTH ? 0 : fslot + 1;
    }
    cp_wait<0>();
    __syncwarp();
    if (lane == ((n - 1) & 31)) w[n - 1] = s[0];
    __syncwarp();

    // ---------------- backward: U, column oriented (xTBSV 'U','N','N') ------------
#pragma unroll
    for (int m = 0; m < BS; m++) {
        const int p = (n - 1) - ((n - 1 - lane) & 31) - 32 * m;
        s[m] = p >= 0 ? w[p] : 0.0;
    }
    // (slot: (n-1-col) mod BWD_DEPTH, kept as a running index by the caller)
    auto issue_U = [&](int col, int slot) {
        if (col >= 0) {
            T* dst = ring + slot * kvp;
            const T* src = Uf + (size_t)col * kvp;
            warp_copy16<BWD_WIN * 8 / 16 / 32>(dst, src, kvp / VEC, lane);
            if (lane == 0) {
                double* st = &stage[slot];
                if (col - BWIN >= 0) cp_async8(st, &w[col - BWIN]);
                else *st = 0.0;
            }
        }
    };
    for (int c = 0; c < BWD_DEPTH; c++) {
        issue_U(n - 1 - c, c);
        cp_commit();
    }
    int bslot = 0;  // (n-1-j) mod BWD_DEPTH
    for (int j = n - 1; j >= 0; j--) {
        cp_wait<BWD_DEPTH - 1>();
        __syncwarp();
        const T* Uc = ring + bslot * kvp;
        double bj = __shfl_sync(0xffffffffu, s[0], j & 31);
        if (bj != 0.0) {
            bj = bj / (double)Uc[kv];
            const int o = (j - lane) & 31;
            const unsigned dmax = (unsigned)min(kv, j);
#pragma unroll
            for (int m = 0; m < BS; m++) {
                const int d = o + 32 * m;  // position j - d; 1 <= d <= min(kv, j)
                if ((unsigned)(d - 1) < dmax)
                    s[m] = s[m] - bj * (double)Uc[kv - d];  // xTBSV: X(I) - TEMP*A(L+I,J)
            }
        }
        if (lane == (j & 31)) {
            w[j] = bj;
#pragma unroll
            for (int m = 0; m + 1 < BS; m++) s[m] = s[m + 1];
            s[BS - 1] = stage[bslot];
        }
        __syncwarp();
        issue_U(j - BWD_DEPTH, bslot);
        cp_commit();
        bslot = bslot + 1 == BWD_DEPTH ? 0 : bslot + 1;
    }
    cp_wait<0>();
}

// r = b - A x per unknown (refinement of the mixed-precision form).  A's row
// comes from assemble_row, so it is the matrix the factorisation saw; the
// 9-point product is summed in FP64.
__global__ void local_residual_kernel(LocalArgs a, const double* b, const double* x, double* r)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int nx = a.d.V;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const SysView v = sys_view(a, sys);
    int types[4] = {a.Vl_t, a.Vu_t, a.Kl_t, a.Ku_t};
    const size_t base = sys_uoff(a, sys);
    for (int in = blockIdx.x * blockDim.x + threadIdx.x; in < n; in += gridDim.x * blockDim.x) {
        double row[9];
        const int st = assemble_row(v, types, a.dt, in, row);
        if (st) set_error(a.status, st);
        double acc = b[base + in];
#pragma unroll
        for (int dy = -1; dy <= 1; dy++)
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                const double m = row[dslot(dx, dy)];
                const int col = in + dy * nx + dx;
                if (m != 0.0 && col >= 0 && col < n) acc -= m * x[base + col];
            }
        r[base + in] = acc;
    }
}

// x += d over every system (blockIdx.y); red[0] = max |d|, red[1] = max |x|
// as dkey values.
__global__ void local_update_kernel(LocalArgs a, double* x, const double* d, unsigned long long* red)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t base = sys_uoff(a, sys);
    double md = 0.0, mx = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = x[base + i] + d[base + i];
        x[base + i] = v;
        md = fmax(md, fabs(d[base + i]));
        mx = fmax(mx, fabs(v));
    }
    for (int o = 16; o > 0; o >>= 1) {
        md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&red[0], dkey(md));
        atomicMax(&red[1], dkey(mx));
    }
}

// ---------------------------------------------------------------------------
// Krylov form of the local solve (learned warm start).

__global__ void local_assemble32_kernel(LocalArgs a, float* A9)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const SysView v = sys_view(a, sys);
    int types[4] = {a.Vl_t, a.Vu_t, a.Kl_t, a.Ku_t};
    float* A = A9 + sys_uoff(a, sys) * 9;
    for (int in = blockIdx.x * blockDim.x + threadIdx.x; in < n; in += gridDim.x * blockDim.x) {
        double row[9];
        const int st = assemble_row(v, types, a.dt, in, row);
        if (st) set_error(a.status, st);
#pragma unroll
        for (int k = 0; k < 9; k++) A[(size_t)k * n + in] = (float)row[k];
    }
}

// block-wide sum of v (all threads get the result); red has 32 floats
__device__ __forceinline__ float block_sum(float v, float* red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    float t = l < nw ? red[l] : 0.f;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    return t;
}

__device__ __forceinline__ float mv_row(const float* A, const float* y, int n, int nx, int i)
{
    float acc = 0.f;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++)
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
            const int col = i + dy * nx + dx;
            const float m = A[(size_t)((dy + 1) * 3 + (dx + 1)) * n + i];
            if (m != 0.f && col >= 0 && col < n) acc = fmaf(m, y[col], acc);
        }
    return acc;
}

// ---- learned preconditioner ----------------------------------------------
// M v (i) = sum over the 5 x 5 neighbourhood o of i of
//           (delta(o = 0) + C[o](i)) v(i + o) / diag(i + o)
// on the system's (V, K') grid (no wrap-around at its edges): a sparse
// approximate inverse whose 25 coefficients per unknown a CNN predicts from
// the matrix (C = 0 is the Jacobi preconditioner).  C is [sys][25][n], slot
// o = (dy + 2) * 5 + (dx + 2).
constexpr int PC_TAPS = 25;

__device__ __forceinline__ float precond_row(const float* C, const float* w, int n, int nx, int ny,
                                             int i)
{
    const int iy = i / nx, ix = i - iy * nx;
    float acc = 0.f;
#pragma unroll
    for (int dy = -2; dy <= 2; dy++) {
        const int yy = iy + dy;
        if (yy < 0 || yy >= ny) continue;
#pragma unroll
        for (int dx = -2; dx <= 2; dx++) {
            const int xx = ix + dx;
            if (xx < 0 || xx >= nx) continue;
            const int o = (dy + 2) * 5 + (dx + 2);
            const float c = C[(size_t)o * n + i] + (o == 12 ? 1.f : 0.f);
            acc = fmaf(c, w[yy * nx + xx], acc);
        }
    }
    return acc;
}

// features of the learned preconditioner, [sys][9][K'][V]: log10(|diag| dt)
// and the eight off-diagonal entries of each row over its diagonal
__global__ void precond_features_kernel(LocalArgs a, const float* A9, float* feat)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const float* A = A9 + u0 * 9;
    float* f = feat + u0 * 9;
    const float dt = (float)a.dt;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float d = A[(size_t)4 * n + i];
        f[i] = log10f(fmaxf(fabsf(d) * dt, 1e-30f));
        int c = 1;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            if (k == 4) continue;
            f[(size_t)c * n + i] = d != 0.f ? A[(size_t)k * n + i] / d : 0.f;
            c++;
        }
    }
}

// Training signal of the learned preconditioner for nprobe probe vectors z
// per system, on the Jacobi-scaled system (unit diagonal) so that every row
// counts alike whatever its scale: with A~ = D^-1 A and M~ = M D (the
// stencil of C without the division, so A M = I exactly when A~ M~ = I),
// y = M~ z, e = A~ y - z, loss += |e|^2 / cnt and
// gC[o](i) = (2 / cnt) sum_z (A^T D^-1 e)(i) z(i + o), the gradient of the
// loss with respect to C.  One CTA per system; z, y and e live in shared
// memory (3 n floats).
__global__ void precond_grad_kernel(const float* A9, const float* C, const float* Z, float* gC,
                                    float* loss, int nx, int ny, int nprobe, float inv_cnt)
{
    extern __shared__ float psm[];
    __shared__ float red[32];
    const int sys = blockIdx.x;
    const int n = nx * ny;
    const float* A = A9 + (size_t)sys * 9 * n;
    const float* dg = A + (size_t)4 * n;
    const float* Cs = C + (size_t)sys * PC_TAPS * n;
    float* g = gC + (size_t)sys * PC_TAPS * n;
    float* z = psm;
    float* y = z + n;
    float* e = y + n;
    for (size_t i = threadIdx.x; i < (size_t)PC_TAPS * n; i += blockDim.x) g[i] = 0.f;
    float lsum = 0.f;
    for (int q = 0; q < nprobe; q++) {
        const float* zq = Z + ((size_t)sys * nprobe + q) * n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) z[i] = zq[i];
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            // y = M~ z: the stencil of delta + C on z
            const int iy = i / nx, ix = i - iy * nx;
            float acc = 0.f;
#pragma unroll
            for (int dy = -2; dy <= 2; dy++) {
                const int yy = iy + dy;
                if (yy < 0 || yy >= ny) continue;
#pragma unroll
                for (int dx = -2; dx <= 2; dx++) {
                    const int xx = ix + dx;
                    if (xx < 0 || xx >= nx) continue;
                    const int o = (dy + 2) * 5 + (dx + 2);
                    acc = fmaf(Cs[(size_t)o * n + i] + (o == 12 ? 1.f : 0.f), z[yy * nx + xx], acc);
                }
            }
            y[i] = acc;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float ei = mv_row(A, y, n, nx, i) / dg[i] - z[i];
            e[i] = ei / dg[i];  // D^-1 e, the operand of A^T below
            lsum = fmaf(ei, ei, lsum);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            // (A^T D^-1 e)(i): rows r = i - off with A[k](r) multiplying x(r + off)
            float gy = 0.f;
#pragma unroll
            for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                for (int dx = -1; dx <= 1; dx++) {
                    const int r = i - (dy * nx + dx);
                    if (r < 0 || r >= n) continue;
                    gy = fmaf(A[(size_t)((dy + 1) * 3 + (dx + 1)) * n + r], e[r], gy);
                }
            gy *= 2.f * inv_cnt;
            const int iy = i / nx, ix = i - iy * nx;
#pragma unroll
            for (int dy = -2; dy <= 2; dy++) {
                const int yy = iy + dy;
                if (yy < 0 || yy >= ny) continue;
#pragma unroll
                for (int dx = -2; dx <= 2; dx++) {
                    const int xx = ix + dx;
                    if (xx < 0 || xx >= nx) continue;
                    g[(size_t)((dy + 2) * 5 + (dx + 2)) * n + i] += gy * z[yy * nx + xx];
                }
            }
        }
        __syncthreads();
    }
    lsum = block_sum(lsum, red);
    if (threadIdx.x == 0) atomicAdd(loss, lsum * inv_cnt);
}

// One CTA per system.  Right preconditioning with M = diag(A) (Jacobi), or
// the learned sparse approximate inverse when Cp is given:
// van der Vorst's BiCGSTAB on A M^-1 u = r, d = M^-1 u accumulated directly.
__global__ void bicgstab_kernel(LocalArgs a, const float* A9, const float* Cp, const double* rr,
                                double* dd, float* scratch, int maxit, float tol, int* iters,
                                unsigned char* ok)
{
    __shared__ float red[32];
    const int sys = blockIdx.x;
    if (skip_system(a, sys)) return;
    const int nx = a.d.V;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const float* A = A9 + u0 * 9;
    const float* dg = A + (size_t)4 * n;
    float* r = scratch + u0 * 6;
    float* rh = r + n;
    float* p = rh + n;
    float* v = p + n;
    float* y = v + n;  // y, then z
    float* t = y + n;
    double* d = dd + u0;
    const double* b = rr + u0;
    const float* Cs = Cp ? Cp + u0 * PC_TAPS : nullptr;
    const int ny = n / nx;
    float bn = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float bi = (float)b[i];
        r[i] = bi;
        rh[i] = bi;
        p[i] = 0.f;
        v[i] = 0.f;
        d[i] = 0.0;
        bn = fmaf(bi, bi, bn);
    }
    bn = sqrtf(block_sum(bn, red));
    float rho = 1.f, alpha = 1.f, omega = 1.f;
    int it = 0;
    bool conv = bn == 0.f;
    while (!conv && it < maxit) {
        it++;
        float rho1 = 0.f;
        for (int i = threadIdx.x; i < n; i += blockDim.x) rho1 = fmaf(rh[i], r[i], rho1);
        rho1 = block_sum(rho1, red);
        if (rho1 == 0.f || !isfinite(rho1)) break;
        const float beta = (rho1 / rho) * (alpha / omega);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            p[i] = r[i] + beta * (p[i] - omega * v[i]);
            if (!Cs) y[i] = p[i] / dg[i];
        }
        __syncthreads();
        if (Cs) {
            // M p = (I + C) D^-1 p: the scaled vector once (t is free here)
            for (int i = threadIdx.x; i < n; i += blockDim.x) t[i] = p[i] / dg[i];
            __syncthreads();
            for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = precond_row(Cs, t, n, nx, ny, i);
            __syncthreads();
        }
        float rv = 0.f;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float vi = mv_row(A, y, n, nx, i);
            v[i] = vi;
            rv = fmaf(rh[i], vi, rv);
        }
        rv = block_sum(rv, red);
        if (rv == 0.f || !isfinite(rv)) break;
        alpha = rho1 / rv;
        float sn = 0.f;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            d[i] += (double)(alpha * y[i]);
            const float si = r[i] - alpha * v[i];
            r[i] = si;  // r now holds s
            sn = fmaf(si, si, sn);
        }
        sn = sqrtf(block_sum(sn, red));
        if (sn <= tol * bn) {
            conv = true;
            break;
        }
        if (Cs) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) t[i] = r[i] / dg[i];
            __syncthreads();  // every scaled s entry is written before M reads its neighbours
            for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = precond_row(Cs, t, n, nx, ny, i);
        } else {
            for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = r[i] / dg[i];  // z
        }
        __syncthreads();
        float ts = 0.f, tt = 0.f;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float ti = mv_row(A, y, n, nx, i);
            t[i] = ti;
            ts = fmaf(ti, r[i], ts);
            tt = fmaf(ti, ti, tt);
        }
        ts = block_sum(ts, red);
        tt = block_sum(tt, red);
        if (tt == 0.f || !isfinite(tt)) break;
        omega = ts / tt;
        float rn = 0.f;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            d[i] += (double)(omega * y[i]);
            const float ri = r[i] - omega * t[i];
            r[i] = ri;
            rn = fmaf(ri, ri, rn);
        }
        rn = sqrtf(block_sum(rn, red));
        if (rn <= tol * bn) conv = true;
        if (omega == 0.f) break;
        rho = rho1;
    }
    if (threadIdx.x == 0) {
        iters[sys] += it;
        if (ok) ok[sys] = conv ? 1 : 0;
    }
}

// the PSD of every system in the unknown order (the state the step starts from)
__global__ void gather_state_kernel(LocalArgs a, double* x)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int V = a.d.V, K = a.d.K, kz = sys_k0(a, sys), n = V * (K - kz);
    const size_t u0 = sys_uoff(a, sys);
    const double* f = a.psd + (size_t)sys * V * K + kz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int iy = i / V, iv = i - iy * V;
        x[u0 + i] = f[(size_t)iv * K + iy];
    }
}

// features [sys][4][K'][V] over the system's pitch-angle rows (K' = K - k0);
// f is the state the step starts from (unknown order)
__global__ void local_features_kernel(LocalArgs a, const double* fstate, float* feat, double* scale)
{
    __shared__ float red[32];
    const int sys = blockIdx.x;
    if (skip_system(a, sys)) return;
    const int V = a.d.V, K = a.d.K, kz = sys_k0(a, sys), ny = K - kz;
    const int n = V * ny;
    const size_t u0 = sys_uoff(a, sys);
    const double* b = fstate + u0;
    float m = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, fabsf((float)b[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = fmaxf(t, red[w]);
        red[0] = t > 0.f ? t : 1.f;
    }
    __syncthreads();
    const float sc = red[0];
    if (threadIdx.x == 0) scale[sys] = sc;
    const size_t fb = (size_t)sys * V * K;  // field slab [V][K]
    const float med = log10f(1e-5f * 86400.f);
    float* f = feat + u0 * 4;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int iy = i / V, iv = i - iy * V;
        const size_t g = fb + (size_t)iv * K + kz + iy;
        const float dvv = (float)a.DVV[g], dkk = (float)a.DKK[g], dvk = (float)a.DVK[g];
        f[i] = (log10f(dvv) - med) * 0.5f;
        f[(size_t)n + i] = (log10f(dkk) - med) * 0.5f;
        f[(size_t)2 * n + i] = dvk / sqrtf(dvv * dkk);
        f[(size_t)3 * n + i] = (float)b[i] / sc;
    }
}

__global__ void warm_start_kernel(LocalArgs a, const double* b, const float* out, const double* scale,
                                  double* x)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const double s = scale[sys];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[u0 + i] = out ? b[u0 + i] + (double)out[u0 + i] * s : b[u0 + i];
}

__global__ void local_targets_kernel(LocalArgs a, const double* b, const double* x, const double* scale,
                                     float* target)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const double s = scale[sys];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        target[u0 + i] = (float)((x[u0 + i] - b[u0 + i]) / s);
}

__global__ void residual_check_kernel(LocalArgs a, const double* b, const double* x, double tol,
                                      double stall, double* prev, unsigned char* pend,
                                      unsigned int* cnt, unsigned long long* maxkey)
{
    __shared__ double rmax[32], bmax[32];
    const int sys = blockIdx.x;
    if (skip_system(a, sys)) return;
    const int nx = a.d.V;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const SysView v = sys_view(a, sys);
    int types[4] = {a.Vl_t, a.Vu_t, a.Kl_t, a.Ku_t};
    const size_t base = sys_uoff(a, sys);
    double mr = 0.0, mb = 0.0;
    for (int in = threadIdx.x; in < n; in += blockDim.x) {
        double row[9];
        assemble_row(v, types, a.dt, in, row);
        double acc = b[base + in];
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const double m = row[dslot(dx, dy)];
                const int col = in + dy * nx + dx;
                if (m != 0.0 && col >= 0 && col < n) acc -= m * x[base + col];
            }
        mr = fmax(mr, fabs(acc));
        mb = fmax(mb, fabs(b[base + in]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
        mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    }
    if ((threadIdx.x & 31) == 0) {
        rmax[threadIdx.x >> 5] = mr;
        bmax[threadIdx.x >> 5] = mb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double R = 0, Bm = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            R = fmax(R, rmax[w]);
            Bm = fmax(Bm, bmax[w]);
        }
        const double rel = Bm > 0 ? R / Bm : R;
        const bool nan = !(rel == rel);
        unsigned char st = 0;
        if (!(rel <= tol)) {
            const double p = prev[sys];
            st = (nan || (p > 0 && rel > stall * p)) ? 2 : 1;
            atomicAdd(&cnt[st - 1], 1u);
        }
        pend[sys] = st;
        prev[sys] = nan ? 1e300 : rel;
        atomicMax(maxkey, dkey(nan ? 1e300 : rel));
    }
}

// weighted Jacobi sweep on the guess: x += omega * r / diag(A) (r = b - A x)
__global__ void jacobi_update_kernel(LocalArgs a, const float* A9, const double* r, double* x,
                                     double omega)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    const float* dg = A9 + u0 * 9 + (size_t)4 * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[u0 + i] += omega * r[u0 + i] / (double)dg[i];
}

__global__ void masked_copy_kernel(LocalArgs a, double* x, const double* y)
{
    const int sys = blockIdx.y;
    if (skip_system(a, sys)) return;  // a.sel selects the systems to copy
    const int n = a.d.V * (a.d.K - sys_k0(a, sys));
    const size_t u0 = sys_uoff(a, sys);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[u0 + i] = y[u0 + i];
}

}  // namespace

void launch_local_residual(const LocalArgs& a, const double* b, const double* x, double* r,
                           cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    dim3 grid((n + 255) / 256, a.d.P * a.d.R);
    local_residual_kernel<<<grid, 256, 0, s>>>(a, b, x, r);
}

void launch_local_update(const LocalArgs& a, double* x, const double* d, unsigned long long* red,
                         cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    dim3 grid((n + 255) / 256, a.d.P * a.d.R);
    local_update_kernel<<<grid, 256, 0, s>>>(a, x, d, red);
}

void launch_local_assemble32(const LocalArgs& a, float* A9, cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    local_assemble32_kernel<<<dim3((n + 255) / 256, a.d.P * a.d.R), 256, 0, s>>>(a, A9);
}

void launch_precond_features(const LocalArgs& a, const float* A9, float* feat, cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    precond_features_kernel<<<dim3((n + 255) / 256, a.d.P * a.d.R), 256, 0, s>>>(a, A9, feat);
}

int launch_precond_grad(const float* A9, const float* C, const float* Z, float* gC, float* loss,
                        int nsys, int nx, int ny, int nprobe, cudaStream_t s)
{
    const size_t smem = (size_t)3 * nx * ny * sizeof(float);
    allow_max_dynamic_smem((const void*)precond_grad_kernel);
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem + 32 * sizeof(float) > (size_t)maxsm) return VERB_ERR_SIZE;
    precond_grad_kernel<<<nsys, 256, smem, s>>>(A9, C, Z, gC, loss, nx, ny, nprobe,
                                                1.f / ((float)nsys * nprobe * nx * ny));
    return VERB_OK;
}

void launch_bicgstab(const LocalArgs& a, const float* A9, const float* Cp, const double* r, double* d,
                     float* scratch, int maxit, float tol, int* iters, unsigned char* ok,
                     cudaStream_t s)
{
    bicgstab_kernel<<<a.d.P * a.d.R, 256, 0, s>>>(a, A9, Cp, r, d, scratch, maxit, tol, iters, ok);
}

void launch_gather_state(const LocalArgs& a, double* x, cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    gather_state_kernel<<<dim3((n + 255) / 256, a.d.P * a.d.R), 256, 0, s>>>(a, x);
}

void launch_local_features(const LocalArgs& a, const double* f, float* feat, double* scale,
                           cudaStream_t s)
{
    local_features_kernel<<<a.d.P * a.d.R, 256, 0, s>>>(a, f, feat, scale);
}

void launch_warm_start(const LocalArgs& a, const double* b, const float* out, const double* scale,
                       double* x, cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    warm_start_kernel<<<dim3((n + 255) / 256, a.d.P * a.d.R), 256, 0, s>>>(a, b, out, scale, x);
}

void launch_local_targets(const LocalArgs& a, const double* b, const double* x, const double* scale,
                          float* target, cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    local_targets_kernel<<<dim3((n + 255) / 256, a.d.P * a.d.R), 256, 0, s>>>(a, b, x, scale, target);
}

void launch_residual_check(const LocalArgs& a, const double* b, const double* x, double tol,
                           double stall, double* prev, unsigned char* pend, unsigned int* cnt,
                           unsigned long long* maxkey, cudaStream_t s)
{
    residual_check_kernel<<<a.d.P * a.d.R, 256, 0, s>>>(a, b, x, tol, stall, prev, pend, cnt,
                                                         maxkey);
}

void launch_jacobi_update(const LocalArgs& a, const float* A9, const double* r, double* x,
                          double omega, cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    jacobi_update_kernel<<<dim3((n + 255) / 256, a.d.P * a.d.R), 256, 0, s>>>(a, A9, r, x, omega);
}

void launch_masked_copy(const LocalArgs& a, double* x, const double* y, cudaStream_t s)
{
    const int n = a.d.V * a.d.K;
    masked_copy_kernel<<<dim3((n + 255) / 256, a.d.P * a.d.R), 256, 0, s>>>(a, x, y);
}

size_t local_factor_smem(int V)
{
    const int kl = V + 1, kv = 2 * kl;
    return ((size_t)(kl + 1) * (kv + 1) + 2 * (kl + 1) + STAGE_ROWS * 9) * sizeof(double);
}

namespace {

template <typename T, int NR, int NC, int NW>
void launch_factor_rw(const LocalArgs& a, cudaStream_t s)
{
    const int kl = a.d.V + 1, kv = 2 * kl;
    dim3 g((a.d.V * a.d.K + 255) / 256, a.d.P * a.d.R);
    local_rows_kernel<T><<<g, 256, 0, s>>>(a);
    const size_t smem = ((size_t)2 * STAGE_ROWS * 9 + 4 * (kv + 1) + 2 * (kl + 1)) * sizeof(double);
    allow_max_dynamic_smem((const void*)local_factor_rw_kernel<T, NR, NC, NW>);
    local_factor_rw_kernel<T, NR, NC, NW><<<a.d.P * a.d.R, NW * 32, smem, s>>>(a);
}

// Eight warps hold the register window.  Twelve and sixteen warps (fewer
// slots and instructions per thread) were measured no faster at V = 101
// (1.20 s and 1.42 s against 1.19 s for 48 x 101 x 101 x 91): the column
// chain, not the per-thread work, sets the time.
constexpr int FRW_WARPS = 8;

// Register window shape: NC = ceil((kv+1)/32) column slots per lane and
// NR = ceil((kl+1)/8) row slots per thread, NR in {2 NC - 1, 2 NC} since
// kv + 1 = 2 (kl+1) - 1.  NC <= 7 keeps the window in 255 registers
// (V <= 110); wider bands take local_factor_kernel.
template <typename T>
bool launch_factor_rw_t(const LocalArgs& a, cudaStream_t s)
{
    const int RW = a.d.V + 2, CW = 2 * (a.d.V + 1) + 1;
    const int nc = (CW + 31) / 32, nr = (RW + FRW_WARPS - 1) / FRW_WARPS;
    if (nc > 7 || (nr != 2 * nc && nr != 2 * nc - 1)) return false;
    // a parked row needs 9 doubles of an L column; systems index grid.y of
    // the parking launch
    if (a.factors32 ? a.klp32 < 18 : a.klp < 9) return false;
    if (a.d.P * a.d.R > 65535) return false;
#define VERB_FRW(NR, NC)                                                              \
    if (nc == NC && nr == NR) {                                                       \
        launch_factor_rw<T, NR, NC, FRW_WARPS>(a, s);                                 \
        return true;                                                                  \
    }
    VERB_FRW(1, 1) VERB_FRW(2, 1) VERB_FRW(3, 2) VERB_FRW(4, 2) VERB_FRW(5, 3) VERB_FRW(6, 3)
    VERB_FRW(7, 4) VERB_FRW(8, 4) VERB_FRW(9, 5) VERB_FRW(10, 5) VERB_FRW(11, 6) VERB_FRW(12, 6)
    VERB_FRW(13, 7) VERB_FRW(14, 7)
#undef VERB_FRW
    return false;
}

}  // namespace

int launch_local_factor(const LocalArgs& a, cudaStream_t s)
{
    if (a.factors32 ? launch_factor_rw_t<float>(a, s) : launch_factor_rw_t<double>(a, s)) return 2;
    const size_t smem = local_factor_smem(a.d.V);
    if (a.factors32) {
        allow_max_dynamic_smem((const void*)local_factor_kernel<float>);
        local_factor_kernel<float><<<a.d.P * a.d.R, FACT_THREADS, smem, s>>>(a);
    } else {
        allow_max_dynamic_smem((const void*)local_factor_kernel<double>);
        local_factor_kernel<double><<<a.d.P * a.d.R, FACT_THREADS, smem, s>>>(a);
    }
    return 1;
}

void launch_local_rhs(const LocalArgs& a, bool from_work, cudaStream_t s)
{
    dim3 grid((a.d.K + 31) / 32, (a.d.V + 31) / 32, a.d.P * a.d.R);
    local_rhs_kernel<<<grid, dim3(32, 8), 0, s>>>(a, from_work ? 1 : 0);
}

void launch_local_store(const LocalArgs& a, cudaStream_t s)
{
    dim3 grid((a.d.K + 31) / 32, (a.d.V + 31) / 32, a.d.P * a.d.R);
    local_store_kernel<<<grid, dim3(32, 8), 0, s>>>(a);
}

namespace {

template <typename T, int W, int FD, int BD, int RW, int MB>
void launch_solve_t(const LocalArgs& a, const size_t kl_p, const size_t kv_p, cudaStream_t s)
{
    const int nsys = a.d.P * a.d.R;
    const int grid = (nsys + W - 1) / W;
    if (RW) {
        // slots of the register window: 32 FS > kl, 32 BS > kv
        const int fs = (a.kl + 1 + 31) / 32, bs = (a.kv + 1 + 31) / 32;
        constexpr int STAGE = (FD > BD ? FD : BD) + 1 & ~1;
        const size_t smem =
            (size_t)W * (STAGE + solve_ring_doubles((int)kl_p, (int)kv_p, sizeof(T), FD, BD)) *
            sizeof(double);
#define VERB_RW(F, B)                                                                         \
    if (fs <= F && bs <= B) {                                                                 \
        allow_max_dynamic_smem((const void*)local_solve_rw_kernel<T, W, FD, BD, F, B, MB>);   \
        local_solve_rw_kernel<T, W, FD, BD, F, B, MB><<<grid, W * 32, smem, s>>>(a, nsys);    \
        return;                                                                               \
    }
        VERB_RW(1, 1)
        VERB_RW(1, 2)
        VERB_RW(2, 3)
        VERB_RW(2, 4)
        VERB_RW(3, 5)
        VERB_RW(3, 6)
        VERB_RW(4, 7)
        VERB_RW(4, 8)
#undef VERB_RW
        // wider bands than the register window holds: the shared-memory window
    }
    const size_t smem =
        (size_t)W * (BWD_WIN + solve_ring_doubles((int)kl_p, (int)kv_p, sizeof(T), FD, BD)) *
        sizeof(double);
    allow_max_dynamic_smem((const void*)local_solve_kernel<T, W, FD, BD>);
    local_solve_kernel<T, W, FD, BD><<<grid, W * 32, smem, s>>>(a, nsys);
}

template <typename T>
void launch_solve_v(const LocalArgs& a, int v, size_t klp, size_t kvp, cudaStream_t s)
{
    switch (v) {
#define VERB_SOLVE_CASE(i)                                                                \
    case i:                                                                               \
        launch_solve_t<T, SOLVE_SHAPES[i].warps, SOLVE_SHAPES[i].fwd, SOLVE_SHAPES[i].bwd, \
                       SOLVE_SHAPES[i].rw, SOLVE_SHAPES[i].minb>(a, klp, kvp, s);         \
        break;
        VERB_SOLVE_CASE(1)
        VERB_SOLVE_CASE(2)
        VERB_SOLVE_CASE(3)
        VERB_SOLVE_CASE(4)
        VERB_SOLVE_CASE(5)
        VERB_SOLVE_CASE(6)
        VERB_SOLVE_CASE(7)
        VERB_SOLVE_CASE(8)
        VERB_SOLVE_CASE(9)
        VERB_SOLVE_CASE(10)
        VERB_SOLVE_CASE(11)
        VERB_SOLVE_CASE(12)
        VERB_SOLVE_CASE(13)
        VERB_SOLVE_CASE(14)
        VERB_SOLVE_CASE(15)
        VERB_SOLVE_CASE(16)
        VERB_SOLVE_CASE(17)
#undef VERB_SOLVE_CASE
        default:
            launch_solve_t<T, SOLVE_SHAPES[0].warps, SOLVE_SHAPES[0].fwd, SOLVE_SHAPES[0].bwd,
                           SOLVE_SHAPES[0].rw, 1>(a, klp, kvp, s);
    }
}

}  // namespace

static_assert(N_SOLVE_SHAPES == 18, "launch_solve_v lists every shape");

int local_solve_variants() { return N_SOLVE_SHAPES; }

void local_solve_variant_shape(int v, int* warps, int* fwd, int* bwd, int* rw)
{
    const SolveShape& sh = SOLVE_SHAPES[v >= 0 && v < N_SOLVE_SHAPES ? v : 0];
    *warps = sh.warps;
    *fwd = sh.fwd;
    *bwd = sh.bwd;
    if (rw) *rw = sh.rw;
}

void launch_local_solve(const LocalArgs& a, cudaStream_t s)
{
    if (a.factors32)
        launch_solve_v<float>(a, a.solve_variant, a.klp32, a.kvp32, s);
    else
        launch_solve_v<double>(a, a.solve_variant, a.klp, a.kvp, s);
}

}  // namespace verb
