// Convection in (MLT, L): Convection_2D + ULTIMATE-QUICKEST on every (V,K) slice.
//
// Reference: src/Convection_2D.cpp:36-169 and
// src/Convection_1D_ULTIMATE_QUICKEST6.cpp:22-482.  Compiled with -fmad=false
// and written with the reference's operation order, so the limiter and
// discriminator comparisons see bit-identical values and the result is
// bit-identical to the reference (exp() of non-zero loss rates aside, which
// may differ by one ulp from the host libm).
//
// Layout: one persistent CTA works on one [P][R] slice at a time; the slice
// stays in shared memory for all of its CFL sub-steps (up to several hundred
// at the high-energy end).  Shared memory holds five P*R double planes: the
// PSD (S), the unlimited result (U), face values (F) and the Courant numbers
// of the P-lines (CP) and R-lines (CR).  Slices are taken highest energy
// first from a ticket counter, as the reference's OpenMP loop does
// (src/VERB4D_Solver.cpp:885-889), which balances the very uneven sub-step
// counts across SMs.
//
// A 1-D pass over a set of lines runs in four block-synchronous phases:
// unlimited faces -> unlimited cells (+BC rewrite) -> limited faces ->
// limited cells (+BC rewrite).  Every face and cell is independent within a
// phase, so the sequential loops of the reference become parallel loops over
// (line, index) with identical arithmetic.
//
// The file is compiled twice: as above (-fmad=false), and with
// -DVERB_BUILD_CONV_FMA -fmad=true, which lets the compiler contract multiply-add
// pairs into fused multiply-adds (one rounding instead of two).  That variant
// runs about 10 % faster and differs from the reference by a few units in the
// last place per step (launch_convection_fma); it also takes the Courant
// factors as products with rounded reciprocals instead of exactly rounded
// quotients, and runs nine warps per CTA instead of eight.
#include "verb_internal.cuh"

#ifdef VERB_BUILD_CONV_FMA
#define VERB_CONV_NS conv_fma
#else
#define VERB_CONV_NS conv_exact
#endif

namespace verb {
namespace VERB_CONV_NS {  // the two compilations keep their kernels apart
namespace {

constexpr int CONV_THREADS = 512;
// Sub-step counts above this are treated as a Courant failure: the reference
// would sub-cycle (practically) forever, and a kernel must never spin unbounded.
constexpr double MAX_SUBSTEPS = 1.0e6;

// 9th-order face value, src/Convection_1D_ULTIMATE_QUICKEST6.cpp:162-241.
__device__ __forceinline__ double quickest_face(double U1, double U2, double U3, double U4, double C,
                                                double D1, double D2v, double D3v, double D4v,
                                                double D5v, double cr)
{
    const double cs = cr * cr;
    const double ca = fabs(cr);
    double f = 0.5 * (C + D1);
    const double d1 = C - D1;
    f += 0.5 * ca * d1;
    const double D2 = (U1 - C - D1 + D2v) / 2;
    const double d3 = U1 - 3 * C + 3 * D1 - D2v;
    f += (cs - 1) / 6.0 * (D2 + ca / 4 * d3);
    const double D4 = (U2 - 3 * U1 + 2 * C + 2 * D1 - 3 * D2v + D3v) / 2;
    const double d5 = U2 - 5 * U1 + 10 * C - 10 * D1 + 5 * D2v - D3v;
    f += (cs - 1) * (cs - 4) / 120.0 * (D4 + ca / 6 * d5);
    const double D6 = (U3 - 5 * U2 + 9 * U1 - 5 * C - 5 * D1 + 9 * D2v - 5 * D3v + D4v) / 2;
    const double d7 = U3 - 7 * U2 + 21 * U1 - 35 * C + 35 * D1 - 21 * D2v + 7 * D3v - D4v;
    f += (cs - 1) * (cs - 4) * (cs - 9) / 5040.0 * (D6 + ca / 8 * d7);
    const double D8 = (U4 - 7 * U3 + 20 * U2 - 28 * U1 + 14 * C + 14 * D1 - 28 * D2v + 20 * D3v -
                       7 * D4v + D5v) /
                      2;
    const double d9 = U4 - 9 * U3 + 36 * U2 - 84 * U1 + 126 * C - 126 * D1 + 84 * D2v - 36 * D3v +
                      9 * D4v - D5v;
    f += (cs - 1) * (cs - 4) * (cs - 9) * (cs - 16) / 362880.0 * (D8 + d9 / 2);
    return f;
}

// Courant-number factors of the face polynomial (QUICKEST6.cpp:209-238); they
// depend only on the face Courant number, which is constant over a slice's
// sub-steps, so they are computed once per slice with the same expressions.
struct FaceCoef {
    double k3, c6, k5, k7, k9;
};

__device__ __forceinline__ FaceCoef face_coef(double cr)
{
    const double cs = cr * cr;
    const double ca = fabs(cr);
    FaceCoef k;
    k.k3 = (cs - 1) / 6.0;
    k.c6 = ca / 6;
    k.k5 = (cs - 1) * (cs - 4) / 120.0;
    k.k7 = (cs - 1) * (cs - 4) * (cs - 9) / 5040.0;
    k.k9 = (cs - 1) * (cs - 4) * (cs - 9) * (cs - 16) / 362880.0;
    return k;
}

// quickest_face with the Courant factors supplied: the same operations in the
// same order, the factor sub-expressions taken from the table.
__device__ __forceinline__ double quickest_face_k(double U1, double U2, double U3, double U4,
                                                  double C, double D1, double D2v, double D3v,
                                                  double D4v, double D5v, double cr,
                                                  const FaceCoef& k)
{
    const double ca = fabs(cr);
    double f = 0.5 * (C + D1);
    const double d1 = C - D1;
    f += 0.5 * ca * d1;
    const double D2 = (U1 - C - D1 + D2v) / 2;
    const double d3 = U1 - 3 * C + 3 * D1 - D2v;
    f += k.k3 * (D2 + ca / 4 * d3);
    const double D4 = (U2 - 3 * U1 + 2 * C + 2 * D1 - 3 * D2v + D3v) / 2;
    const double d5 = U2 - 5 * U1 + 10 * C - 10 * D1 + 5 * D2v - D3v;
    f += k.k5 * (D4 + k.c6 * d5);
    const double D6 = (U3 - 5 * U2 + 9 * U1 - 5 * C - 5 * D1 + 9 * D2v - 5 * D3v + D4v) / 2;
    const double d7 = U3 - 7 * U2 + 21 * U1 - 35 * C + 35 * D1 - 21 * D2v + 7 * D3v - D4v;
    f += k.k7 * (D6 + ca / 8 * d7);
    const double D8 = (U4 - 7 * U3 + 20 * U2 - 28 * U1 + 14 * C + 14 * D1 - 28 * D2v + 20 * D3v -
                       7 * D4v + D5v) /
                      2;
    const double d9 = U4 - 9 * U3 + 36 * U2 - 84 * U1 + 126 * C - 126 * D1 + 84 * D2v - 36 * D3v +
                      9 * D4v - D5v;
    f += k.k9 * (D8 + d9 / 2);
    return f;
}

#ifdef VERB_BUILD_CONV_FMA
// quickest_face_k regrouped for the contracted form: the D terms are symmetric
// and the d terms antisymmetric in the pairs (U_k, D_k+1) (upwind point k
// cells behind the centre, downwind point k+1 cells ahead), so they are
// formed from the pair sums s_k and differences t_k, with the same
// polynomial in the Courant factors.  Fewer operations and shorter
// dependency chains; the rounding differs from the reference order by a few
// units in the last place.
__device__ __forceinline__ double quickest_face_sym(double U1, double U2, double U3, double U4,
                                                    double C, double D1, double D2v, double D3v,
                                                    double D4v, double D5v, double cr,
                                                    const FaceCoef& k)
{
    const double ca = fabs(cr);
    const double s0 = C + D1, t0 = C - D1;
    const double s1 = U1 + D2v, t1 = U1 - D2v;
    const double s2 = U2 + D3v, t2 = U2 - D3v;
    const double s3 = U3 + D4v, t3 = U3 - D4v;
    const double s4 = U4 + D5v, t4 = U4 - D5v;
    const double D2 = (s1 - s0) * 0.5;
    const double d3 = t1 - 3 * t0;
    const double D4 = ((s2 - 3 * s1) + 2 * s0) * 0.5;
    const double d5 = (t2 - 5 * t1) + 10 * t0;
    const double D6 = ((s3 - 5 * s2) + (9 * s1 - 5 * s0)) * 0.5;
    const double d7 = (t3 - 7 * t2) + (21 * t1 - 35 * t0);
    const double D8 = ((s4 - 7 * s3) + (20 * s2 - 28 * s1) + 14 * s0) * 0.5;
    const double d9 = (t4 - 9 * t3) + (36 * t2 - 84 * t1) + 126 * t0;
    double f = 0.5 * s0;
    f += 0.5 * ca * t0;
    f += k.k3 * (D2 + ca * 0.25 * d3);
    f += k.k5 * (D4 + k.c6 * d5);
    f += k.k7 * (D6 + ca * 0.125 * d7);
    f += k.k9 * (D8 + d9 * 0.5);
    return f;
}
#define QUICKEST_FACE quickest_face_sym
#else
#define QUICKEST_FACE quickest_face_k
#endif

// Limiter of src/Convection_1D_ULTIMATE_QUICKEST6.cpp:394-447 applied to the
// unlimited face value f.
__device__ __forceinline__ double quickest_limit(double f, double cr, double ou, double oc,
                                                 double od, double UU1, double UU2, double UU3,
                                                 double UC, double UD1, double UD2, double UD3)
{
    const double ca = fabs(cr);
    const double DEL = od - ou;
    const double CURV = od - 2 * oc + ou;
    const double ADEL = fabs(DEL);
    const double ACURV = fabs(CURV);
    const double dif1 = UD2 - UD3;
    const double dif2 = UD1 - UD2;
    const double dif3 = UC - UD1;
    const double dif4 = UU1 - UC;
    const double dif5 = UU2 - UU1;
    const double dif6 = UU3 - UU2;
    const bool peak_dw = dif1 > 0 && dif2 > 0 && dif3 < 0 && dif4 < 0 && dif2 < dif1 && dif3 > dif4;
    const bool peak_c = dif2 > 0 && dif3 > 0 && dif4 < 0 && dif5 < 0 && dif3 < dif2 && dif4 > dif5;
    const bool peak_u = dif3 > 0 && dif4 > 0 && dif5 < 0 && dif6 < 0 && dif4 < dif3 && dif5 > dif6;
    if (!(peak_dw || peak_c || peak_u)) {
        if (ACURV >= ADEL) {
            f = oc;
        } else if (ca > 1e-31) {
            const double ref = ou + (oc - ou) / ca;
            if (DEL > 0) {
                f = fmax(f, oc);
                f = fmin(f, fmin(ref, od));
            } else if (DEL < 0) {
                f = fmin(f, oc);
                f = fmax(f, fmax(ref, od));
            }
        }
    }
    return f;
}

// Per-line description of a 1-D sweep.
struct Line {
    int base, stride;   // element ix of the line is at base + ix*stride in a plane
    double lbc, ubc;    // boundary values
    double dxl, dxu;    // x[1]-x[0] and x[n-1]-x[n-2] (ConstantDerivative ghosts)
};

struct Sweep {
    int n;              // points per line
    int lt, ut;         // lower / upper BC types
};

// Value t[k] of a line extended by GST ghost cells per side
// (src/Convection_1D_ULTIMATE_QUICKEST6.cpp:89-143 and 277-330): `lo` feeds
// the low ghosts and `in`/`hi` the interior and high ghosts.
__device__ __forceinline__ double ext(const double* in, const double* lo, const double* hi,
                                      const Line& L, const Sweep& w, int k)
{
    if (k >= 0 && k < w.n) return in[L.base + k * L.stride];
    if (k < 0) {
        const int ig = -k;
        if (w.lt == VERB_BC_PERIODIC) return lo[L.base + ((w.n - 1) - ig) * L.stride];
        if (w.lt == VERB_BC_CONSTANT_VALUE) return L.lbc;
        double g = lo[L.base] - L.lbc * L.dxl;
        for (int i = 2; i <= ig; i++) g = g - L.lbc * L.dxl;
        return g;
    }
    const int ig = k - (w.n - 1);
    if (w.ut == VERB_BC_PERIODIC) return hi[L.base + ig * L.stride];
    if (w.ut == VERB_BC_CONSTANT_VALUE) return L.ubc;
    double g = hi[L.base + (w.n - 1) * L.stride] + L.ubc * L.dxu;
    for (int i = 2; i <= ig; i++) g = g + L.ubc * L.dxu;
    return g;
}

// Courant number of face ix (between cells ix-1 and ix), :150-160.
__device__ __forceinline__ double face_cr(const double* cour, const Line& L, const Sweep& w, int ix)
{
    if (ix == 0) return (cour[L.base + (w.n - 2) * L.stride] + cour[L.base]) / 2;
    return (cour[L.base + (ix - 1) * L.stride] + cour[L.base + ix * L.stride]) / 2;
}

// Flux difference update of cell c (:245-249 / 448-452); face 0 of a
// non-periodic line carries zero flux (courant_left = psd_face_left = 0).
__device__ __forceinline__ double cell_raw(const double* S, const double* F, const double* cour,
                                           const Line& L, const Sweep& w, int c)
{
    const double cr = face_cr(cour, L, w, c + 1);
    const double fr = F[L.base + (c + 1) * L.stride];
    double cl = 0.0, fl = 0.0;
    if (c > 0 || w.lt == VERB_BC_PERIODIC) {
        cl = face_cr(cour, L, w, c);
        fl = F[L.base + c * L.stride];
    }
    return S[L.base + c * L.stride] - (cr * fr - cl * fl);
}

// Final value of cell c after the boundary rewrite of :257-272 / 457-477.
__device__ __forceinline__ double cell_final(const double* S, const double* F, const double* cour,
                                             const Line& L, const Sweep& w, int c)
{
    if (c == w.n - 1) {
        if (w.ut == VERB_BC_CONSTANT_VALUE) return L.ubc;
        if (w.ut == VERB_BC_CONSTANT_DERIVATIVE) return cell_raw(S, F, cour, L, w, w.n - 2);
        return cell_raw(S, F, cour, L, w, 0);  // periodic: f[n-1] = f[0]
    }
    if (c == 0) {
        if (w.lt == VERB_BC_CONSTANT_VALUE) return L.lbc;
        if (w.lt == VERB_BC_CONSTANT_DERIVATIVE) return cell_raw(S, F, cour, L, w, 1);
    }
    return cell_raw(S, F, cour, L, w, c);
}

// One inner sub-step of Convection_1D_ULTIMATE_QUICKEST6 on every active line.
// Lines are described by `line(l)`; `active(l)` masks lines whose own CFL
// sub-cycle is already complete.  The new values land in U (inactive lines are
// copied), so the caller swaps S and U afterwards.
template <class LineFn, class ActiveFn>
__device__ void quickest_pass(const double* S, double* U, double* F, const double* cour, int nlines,
                              const Sweep& w, bool line_major, LineFn line, ActiveFn active)
{
    const int n = w.n;
    const int total = nlines * n;
    const int ix0 = (w.lt == VERB_BC_PERIODIC) ? 0 : 1;
    auto split = [&](int i, int& l, int& ix) {
        if (line_major) {
            l = i / n;
            ix = i - l * n;
        } else {
            ix = i / nlines;
            l = i - ix * nlines;
        }
    };
    // A: unlimited faces (:148-256)
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        int l, ix;
        split(i, l, ix);
        if (ix < ix0 || !active(l)) continue;
        const Line L = line(l);
        const double cr = face_cr(cour, L, w, ix);
        double U1, U2, U3, U4, C, D1, D2, D3, D4, D5;
        if (cr >= 0) {
            const int c = ix - 1;
            U1 = ext(S, S, S, L, w, c - 1);
            U2 = ext(S, S, S, L, w, c - 2);
            U3 = ext(S, S, S, L, w, c - 3);
            U4 = ext(S, S, S, L, w, c - 4);
            C = ext(S, S, S, L, w, c);
            D1 = ext(S, S, S, L, w, c + 1);
            D2 = ext(S, S, S, L, w, c + 2);
            D3 = ext(S, S, S, L, w, c + 3);
            D4 = ext(S, S, S, L, w, c + 4);
            D5 = ext(S, S, S, L, w, c + 5);
        } else {
            D1 = ext(S, S, S, L, w, ix - 1);
            D2 = ext(S, S, S, L, w, ix - 2);
            D3 = ext(S, S, S, L, w, ix - 3);
            D4 = ext(S, S, S, L, w, ix - 4);
            D5 = ext(S, S, S, L, w, ix - 5);
            C = ext(S, S, S, L, w, ix);
            U1 = ext(S, S, S, L, w, ix + 1);
            U2 = ext(S, S, S, L, w, ix + 2);
            U3 = ext(S, S, S, L, w, ix + 3);
            U4 = ext(S, S, S, L, w, ix + 4);
        }
        F[L.base + ix * L.stride] = quickest_face(U1, U2, U3, U4, C, D1, D2, D3, D4, D5, cr);
    }
    __syncthreads();
    // B: unlimited cells with the boundary rewrite (:245-272)
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        int l, ix;
        split(i, l, ix);
        if (!active(l)) continue;
        const Line L = line(l);
        U[L.base + ix * L.stride] = cell_final(S, F, cour, L, w, ix);
    }
    __syncthreads();
    // C: limited faces (:332-447); orig values from S, unlimited from U with the
    // low ghosts taken from the pre-step S (:283-302) and high ones from U.
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        int l, ix;
        split(i, l, ix);
        if (ix < ix0 || !active(l)) continue;
        const Line L = line(l);
        const double cr = face_cr(cour, L, w, ix);
        double ou, oc, od, UU1, UU2, UU3, UC, UD1, UD2, UD3;
        if (cr >= 0) {
            const int c = ix - 1;
            UU1 = ext(U, S, U, L, w, c - 1);
            UU2 = ext(U, S, U, L, w, c - 2);
            UU3 = ext(U, S, U, L, w, c - 3);
            ou = ext(S, S, S, L, w, c - 1);
            UC = ext(U, S, U, L, w, c);
            oc = ext(S, S, S, L, w, c);
            UD1 = ext(U, S, U, L, w, c + 1);
            UD2 = ext(U, S, U, L, w, c + 2);
            UD3 = ext(U, S, U, L, w, c + 3);
            od = ext(S, S, S, L, w, c + 1);
        } else {
            UD1 = ext(U, S, U, L, w, ix - 1);
            UD2 = ext(U, S, U, L, w, ix - 2);
            UD3 = ext(U, S, U, L, w, ix - 3);
            od = ext(S, S, S, L, w, ix - 1);
            UC = ext(U, S, U, L, w, ix);
            oc = ext(S, S, S, L, w, ix);
            UU1 = ext(U, S, U, L, w, ix + 1);
            UU2 = ext(U, S, U, L, w, ix + 2);
            UU3 = ext(U, S, U, L, w, ix + 3);
            ou = ext(S, S, S, L, w, ix + 1);
        }
        double* fp = &F[L.base + ix * L.stride];
        *fp = quickest_limit(*fp, cr, ou, oc, od, UU1, UU2, UU3, UC, UD1, UD2, UD3);
    }
    __syncthreads();
    // D: limited cells with the boundary rewrite (:448-477), into U.
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        int l, ix;
        split(i, l, ix);
        const Line L = line(l);
        const int a = L.base + ix * L.stride;
        U[a] = active(l) ? cell_final(S, F, cour, L, w, ix) : S[a];
    }
    __syncthreads();
}

__device__ __forceinline__ double block_max(double v, double* red)
{
    for (int o = 16; o > 0; o >>= 1) {
        double t = __shfl_xor_sync(0xffffffffu, v, o);
        v = (v < t) ? t : v;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double m = red[0];
    for (int i = 1; i < nw; i++) m = (m < red[i]) ? red[i] : m;
    __syncthreads();
    return m;
}

// ---------------------------------------------------------------------------
// Slice kernel.
//
// A CTA of C3_WARPS warps owns one [P][R] slice at a time; the slice stays in
// shared memory (plane S) for all of its CFL sub-steps.  A sweep is a set of
// independent lines (P-lines: fixed L, R-lines: fixed MLT).  A warp takes
// 32/lpl lines per job with lpl lanes per line, and lane j of a line owns the
// cells x = j + lpl*t, t < T = ceil(n/lpl): at every step of a phase the lanes
// of a line touch consecutive shared-memory words.  A job copies its lines
// into per-warp buffers extended by the GST = 5 ghost cells of
// QUICKEST6.cpp:89-143, stages the lines' face Courant numbers next to them,
// and runs the four phases of one ULTIMATE-QUICKEST sub-step with warp
// synchronisation only:
//   A  unlimited face values into F                    (QUICKEST6.cpp:148-241)
//   B  unlimited cells + boundary rewrite into UE      (:243-272)
//   C  limited face values into F                      (:277-447)
//   D  final cells + rewrite; into S on the last sub-step (:448-477)
// The Courant factors of the face polynomial are recomputed from the face
// Courant number with exactly rounded divisions by the constant denominators
// (div_const).  All faces of a job usually have
// the same upwind direction (the drift velocities are smooth along MLT and the
// radial velocity depends on MLT only), so a job is dispatched to a
// direction-specialised body in which the upwind stencil roles are fixed
// registers; jobs with mixed directions select the roles per face.
//
// The radial sweep works on PSD*G: a pass over the plane multiplies by G
// before it, and the epilogue pass /G, *exp(Loss dt), +S dt (interior L)
// follows it, in the reference's order (src/Convection_2D.cpp:122-165).  The
// per-slice planes G, exp(Loss dt), S dt and the face Courant tables live in a
// per-CTA scratch region that stays resident in L2.

// Warps per CTA (two CTAs per SM).  The contracted build needs fewer
// registers (113 fit), so nine warps per CTA fit beside the exact build's
// eight in the same shared memory and register file.
#ifdef VERB_BUILD_CONV_FMA
constexpr int C3_WARPS = 9;
#else
constexpr int C3_WARPS = 8;
#endif
constexpr int C3_THREADS = C3_WARPS * 32;
constexpr int TMAX = 16;  // cells per lane: lines of up to 32*TMAX points

// a / b rounded to nearest, for the constants b = 6, 120, 5040 and 362880 with
// y = RN(1/b) (Markstein's correction step: P. Markstein, IBM J. Res. Dev.
// 34(1), 1990).  q = RN(a*y) is within 1.5 ulp of a/b, so the residual a - b*q
// is a representable number (at most 6B units of 2^(e_b+e_q-1), B <= 2835 the
// odd part of b) and the fused multiply-add returns it exactly.  q + r*y then
// differs from a/b by |r|*|y - 1/b| < 1.5*2^-53 ulp, whereas a/b lies at
// least ulp/(2B) away from every rounding midpoint (b's odd part B >= 3 makes
// a midpoint times b need more than 53 significant bits), so a single
// rounding of q + r*y gives RN(a/b).  A zero residual returns q, which keeps
// the sign that division gives to a zero quotient.
__device__ __forceinline__ double div_const(double a, double b, double y)
{
    const double q = __dmul_rn(a, y);
    const double r = __fma_rn(-q, b, a);
    return r == 0.0 ? q : __fma_rn(r, y, q);
}

// The same for a dividend that is never -0 (then a zero residual needs no
// special case: q + 0*y = q for every q but -0).
__device__ __forceinline__ double div_const_nz(double a, double b, double y)
{
    const double q = __dmul_rn(a, y);
    return __fma_rn(__fma_rn(-q, b, a), y, q);
}

// Courant factors of the face polynomial (QUICKEST6.cpp:209-238), the same
// expressions as face_coef().
__device__ __forceinline__ FaceCoef face_coef_exact(double cr)
{
    const double cs = cr * cr;
    const double ca = fabs(cr);
    const double t1 = cs - 1;
    const double p2 = t1 * (cs - 4);
    const double p3 = p2 * (cs - 9);
    const double p4 = p3 * (cs - 16);
    // t1 = cs - 1 and ca = |cr| are never -0, nor is p3 = p2*(cs-9) (p2 = -0
    // only when cs = 1, and then p3 = +0); p2 and p4 are -0 when |cr| = 1
    FaceCoef k;
#ifdef VERB_BUILD_CONV_FMA
    // contracted form: a product with the rounded reciprocal (within an ulp
    // of the quotient) instead of the exactly rounded division
    k.k3 = t1 * (1.0 / 6.0);
    k.c6 = ca * (1.0 / 6.0);
    k.k5 = p2 * (1.0 / 120.0);
    k.k7 = p3 * (1.0 / 5040.0);
    k.k9 = p4 * (1.0 / 362880.0);
#else
    k.k3 = div_const_nz(t1, 6.0, 1.0 / 6.0);
    k.c6 = div_const_nz(ca, 6.0, 1.0 / 6.0);
    k.k5 = div_const(p2, 120.0, 1.0 / 120.0);
    k.k7 = div_const_nz(p3, 5040.0, 1.0 / 5040.0);
    k.k9 = div_const(p4, 362880.0, 1.0 / 362880.0);
#endif
    return k;
}

enum { DIR_POS = 0, DIR_NEG = 1, DIR_MIX = 2 };

// Face value of face x from w[k] = E[x-5+k].  Courant >= 0: upwind centre
// x-1, U_k = E[x-1-k], D_k = E[x-1+k]; Courant < 0: centre x, U_k = E[x+k],
// D_k = E[x-k] (QUICKEST6.cpp:169-186).
template <int DIR>
__device__ __forceinline__ double face3(const double (&w)[10], double cr)
{
    const FaceCoef k = face_coef_exact(cr);
    if (DIR == DIR_POS)
        return QUICKEST_FACE(w[3], w[2], w[1], w[0], w[4], w[5], w[6], w[7], w[8], w[9], cr, k);
    if (DIR == DIR_NEG)
        return QUICKEST_FACE(w[6], w[7], w[8], w[9], w[5], w[4], w[3], w[2], w[1], w[0], cr, k);
    const bool up = cr >= 0;
    return QUICKEST_FACE(up ? w[3] : w[6], up ? w[2] : w[7], up ? w[1] : w[8], up ? w[0] : w[9],
                           up ? w[4] : w[5], up ? w[5] : w[4], up ? w[6] : w[3], up ? w[7] : w[2],
                           up ? w[8] : w[1], up ? w[9] : w[0], cr, k);
}

// quickest_limit with the branches turned into selects: the same comparisons
// and the same fmax/fmin sequence pick the same value; only the division for
// the reference value stays behind a branch.
__device__ __forceinline__ double quickest_limit_sel(double f, double cr, double ou, double oc,
                                                     double od, double UU1, double UU2, double UU3,
                                                     double UC, double UD1, double UD2, double UD3)
{
    const double ca = fabs(cr);
    const double DEL = od - ou;
    const double CURV = od - 2 * oc + ou;
    const double ADEL = fabs(DEL);
    const double ACURV = fabs(CURV);
    const double dif1 = UD2 - UD3;
    const double dif2 = UD1 - UD2;
    const double dif3 = UC - UD1;
    const double dif4 = UU1 - UC;
    const double dif5 = UU2 - UU1;
    const double dif6 = UU3 - UU2;
    const bool peak_dw = dif1 > 0 && dif2 > 0 && dif3 < 0 && dif4 < 0 && dif2 < dif1 && dif3 > dif4;
    const bool peak_c = dif2 > 0 && dif3 > 0 && dif4 < 0 && dif5 < 0 && dif3 < dif2 && dif4 > dif5;
    const bool peak_u = dif3 > 0 && dif4 > 0 && dif5 < 0 && dif6 < 0 && dif4 < dif3 && dif5 > dif6;
    const bool mono = !(peak_dw || peak_c || peak_u);
    const bool flat = ACURV >= ADEL;
    const bool rise = DEL > 0, fall = DEL < 0;
    const bool useref = mono && !flat && ca > 1e-31 && (rise || fall);
    double ref = 0.0;
    if (useref) ref = ou + (oc - ou) / ca;
    const double fr = fmin(fmax(f, oc), fmin(ref, od));
    const double ff = fmax(fmin(f, oc), fmax(ref, od));
    double res = useref ? (rise ? fr : ff) : f;
    if (mono && flat) res = oc;
    return res;
}

// Limited face value of face x from u[k] = UE[x-4+k] and ev[k] = E[x-2+k].
template <int DIR>
__device__ __forceinline__ double limit3(double f, double cr, const double (&u)[8],
                                         const double (&ev)[4])
{
    if (DIR == DIR_POS)
        return quickest_limit_sel(f, cr, ev[0], ev[1], ev[2], u[2], u[1], u[0], u[3], u[4], u[5], u[6]);
    if (DIR == DIR_NEG)
        return quickest_limit_sel(f, cr, ev[3], ev[2], ev[1], u[5], u[6], u[7], u[4], u[3], u[2], u[1]);
    const bool up = cr >= 0;
    return quickest_limit_sel(f, cr, up ? ev[0] : ev[3], up ? ev[1] : ev[2], up ? ev[2] : ev[1],
                              up ? u[2] : u[5], up ? u[1] : u[6], up ? u[0] : u[7],
                              up ? u[3] : u[4], up ? u[4] : u[3], up ? u[5] : u[2],
                              up ? u[6] : u[1]);
}

// 8-byte asynchronous global->shared copy (cp.async, sm_80+).
__device__ __forceinline__ void cp_async8(double* dst, const double* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Work split of one sweep: nlines lines of n points, lpl lanes per line, T
// cells per lane.  The choice models a job's cost as a fixed part (line
// set-up, boundary cells, ghost cells, barriers: about 400 warp instructions)
// plus about 330 per cell step, and counts half of the idle warp slots of the
// last round (the other CTA on the SM fills the rest).
struct SweepCfg {
    int lpl, T, nlw, njobs, nb;  // nb: doubles per line buffer (E, UE, F and CR each)
};

__host__ __device__ inline SweepCfg sweep_cfg(int n, int nlines)
{
    SweepCfg best{0, 0, 0, 0, 0};
    double bc = 0.0;
    for (int lpl = 32; lpl >= 8; lpl >>= 1) {
        const int T = (n + lpl - 1) / lpl;
        if (T > TMAX) continue;
        const int nlw = 32 / lpl;
        const int jobs = (nlines + nlw - 1) / nlw;
        const int rounds = (jobs + C3_WARPS - 1) / C3_WARPS;
        const double job = 400.0 + 330.0 * T;
        const double cost = job * (jobs + 0.5 * (rounds * C3_WARPS - jobs));
        if (best.lpl == 0 || cost < bc - 1e-9) {
            bc = cost;
            best = SweepCfg{lpl, T, nlw, jobs, lpl * T + 10};
        }
    }
    return best;  // lpl == 0: lines longer than 32*TMAX points
}

// per-warp buffer size in doubles (both sweeps share it)
__host__ __device__ inline int conv_wstride(int P, int R)
{
    int w = 0;
    if (P >= 3) {
        const SweepCfg c = sweep_cfg(P, R - 1);
        w = c.nlw * 4 * c.nb;
    }
    if (R >= 3) {
        const SweepCfg c = sweep_cfg(R, P);
        if (c.nlw * 4 * c.nb > w) w = c.nlw * 4 * c.nb;
    }
    return (w + 1) & ~1;  // keep every warp's buffer 16-byte aligned
}

// One job's lines as seen by one lane.
struct LineJob {
    double *E, *UE, *F, *CR;  // the lane's line buffers; E/UE slot x+5 holds cell x,
                              // F and CR slot x hold face x and its Courant number
    int n, lpl, T, j;         // line length, lanes per line, cells per lane, lane in line
    int li;                   // line index (P-sweep: iR, R-sweep: iP)
    int lt, ut;               // boundary types
    int ns, nsmax;            // the line's sub-steps; the maximum over the warp
    int R;                    // row length of the plane S
    bool lv;                  // the lane's line exists
    double lbc, ubc, dxl, dxu;
};

// Flux update of cell k, E[k] - (cr[k+1]*F[k+1] - cr[k]*F[k]) (:245-249,
// 448-452).  A non-periodic line's cell 0 is always rewritten, so its left
// flux (zero in the reference) is never used.
__device__ __forceinline__ double cell_raw3(const LineJob& J, int k)
{
    return J.E[k + 5] - (J.CR[k + 1] * J.F[k + 1] - J.CR[k] * J.F[k]);
}

// End cell of a line after the boundary rewrite (:257-272 / 457-477): lane 0
// of a line computes cell 0 and lane 1 cell n-1, with the same code; cells
// 1..n-2 keep their flux update.
__device__ __forceinline__ double edge_cell3(const LineJob& J)
{
    const bool hi = J.j == 1;
    const int type = hi ? J.ut : J.lt;
    const int k = type == VERB_BC_CONSTANT_DERIVATIVE ? (hi ? J.n - 2 : 1) : 0;
    const double raw = cell_raw3(J, k);
    return type == VERB_BC_CONSTANT_VALUE ? (hi ? J.ubc : J.lbc) : raw;
}

__device__ __forceinline__ void store_plane(double* S, const LineJob& J, bool RS, int x, double v)
{
    if (RS) S[J.li * J.R + x] = v;
    else S[x * J.R + J.li] = v;
}

// Ghost cells of the extended line X from its interior (QUICKEST6.cpp:94-140
// for E; :281-326 for UE).  Ghost gi < 5 is low ghost gi+1, gi >= 5 high
// ghost gi-4; the lanes of a line take the ten of them in turn, with the same
// code at both ends.  With low unset only the high ghosts are filled (UE's low
// ghosts are copies of E's); constant-value ghosts are written only when cv is
// set (they do not change within a job).
__device__ __forceinline__ void fill_ghosts3(double* X, const LineJob& J, bool low, bool cv)
{
    const int n = J.n;
    for (int gi = J.j; gi < 10; gi += J.lpl) {
        if (!low && gi < 5) continue;
        const bool hi = gi >= 5;
        const int ig = hi ? gi - 4 : gi + 1;
        const int type = hi ? J.ut : J.lt;
        double g;
        if (type == VERB_BC_PERIODIC) {
            g = X[hi ? 5 + ig : 5 + (n - 1) - ig];
        } else if (type == VERB_BC_CONSTANT_VALUE) {
            if (!cv) continue;
            g = hi ? J.ubc : J.lbc;
        } else {
            const double c = hi ? J.ubc * J.dxu : J.lbc * J.dxl;
            g = hi ? X[5 + n - 1] + c : X[5] - c;
            for (int i = 2; i <= ig; i++) g = hi ? g + c : g - c;
        }
        X[hi ? 5 + (n - 1) + ig : 5 - ig] = g;
    }
}

// All sub-steps of one job (QUICKEST6.cpp:37-52 sub-cycle, one pass per
// sub-step).  The loops over a lane's cells stay rolled (one copy of the face
// code per phase keeps the kernel small enough for the instruction caches);
// the per-cell state between phases lives in the line buffers.  Cell loops
// cover cells 0..n-2 (lane 0 rewrites cell 0); lane 1 of a line writes cell
// n-1 with its boundary rewrite; lanes 0-9 then fill the ghost cells.
template <bool RS, int DIR>
__device__ __forceinline__ void job_substeps(double* S, const LineJob& J)
{
    const int L = J.lpl;
    const bool edge = J.lv && J.j < 2;      // lanes 0 and 1: cells 0 and n-1
    const int ecell = J.j == 1 ? J.n - 1 : 0;
    const int nc = J.lv ? J.n - 1 : 0;
    // the lane's first cell in every buffer; loops advance them by L cells
    const double* const E0 = J.E + J.j;
    double* const UE0 = J.UE + J.j;
    double* const F0 = J.F + J.j;
    const double* const CR0 = J.CR + J.j;
    double* const SP0 = RS ? S + J.li * J.R + J.j : S + J.j * J.R + J.li;
    const int sstep = RS ? L : L * J.R;
    for (int sub = 0; sub < J.nsmax; sub++) {
        // A: unlimited faces
        {
            const double* e = E0;
            const double* c = CR0;
            double* f = F0;
#pragma unroll 1
            for (int t = 0; t < J.T; t++, e += L, c += L, f += L) {
                double w[10];
#pragma unroll
                for (int k = 0; k < 10; k++) w[k] = e[k];
                *f = face3<DIR>(w, *c);
            }
        }
        __syncwarp();
        // B: unlimited cells into UE
        {
            const double* e = E0;
            const double* c = CR0;
            const double* f = F0;
            double* u = UE0;
#pragma unroll 2
            for (int x = J.j; x < nc; x += L, e += L, c += L, f += L, u += L)
                u[5] = e[5] - (c[1] * f[1] - c[0] * f[0]);
        }
        if (edge) J.UE[ecell + 5] = edge_cell3(J);
        __syncwarp();
        if (J.lv) {
            if (J.j < 5) J.UE[J.j] = J.E[J.j];  // low ghosts: the pre-step ones of E
            fill_ghosts3(J.UE, J, false, false);
        }
        __syncwarp();
        // C: limited faces, in place (each lane reads only its own faces)
        {
            const double* e = E0;
            const double* c = CR0;
            double* f = F0;
            const double* u = UE0;
#pragma unroll 1
            for (int t = 0; t < J.T; t++, e += L, c += L, f += L, u += L) {
                double uu[8], ev[4];
#pragma unroll
                for (int k = 0; k < 8; k++) uu[k] = u[1 + k];
#pragma unroll
                for (int k = 0; k < 4; k++) ev[k] = e[3 + k];
                *f = limit3<DIR>(*f, *c, uu, ev);
            }
        }
        __syncwarp();
        // D: final cells.  On a line's last sub-step they go to the plane;
        // otherwise they are staged in UE (free after phase C) and copied into
        // E once every lane is done reading E.
        const bool last = sub == J.ns - 1;
        {
            const double* e = E0;
            const double* c = CR0;
            const double* f = F0;
            double* u = UE0;
            double* sp = SP0;
#pragma unroll 2
            for (int x = J.j; x < nc; x += L, e += L, c += L, f += L, u += L, sp += sstep) {
                const double v = e[5] - (c[1] * f[1] - c[0] * f[0]);
                if (last) *sp = v;
                else u[5] = v;
            }
        }
        if (edge) {
            const double v = edge_cell3(J);
            if (last) store_plane(S, J, RS, ecell, v);
            else J.UE[ecell + 5] = v;
        }
        if (sub + 1 < J.nsmax) {
            __syncwarp();
            {
                const double* u = UE0;
                double* e = J.E + J.j;
                const int ncf = J.lv ? J.n : 0;
#pragma unroll 2
                for (int x = J.j; x < ncf; x += L, u += L, e += L) e[5] = u[5];
            }
            __syncwarp();
            if (J.lv) fill_ghosts3(J.E, J, true, false);
            __syncwarp();
        }
    }
    __syncwarp();  // the warp's next job overwrites the buffers read in phase D
}

struct LineArrays {
    const double *lb, *ub, *dxl, *dxu;
    const int *ns, *dir;
};

// One job of a sweep: load the lines into the warp's buffers, pick the
// direction-specialised body, run the line sub-steps.
template <bool RS>
__device__ __forceinline__ void sweep_job(double* S, double* wb, const SweepCfg& c, int job, int n,
                                          int nlines, int R, int lt, int ut, const double* crtab,
                                          const LineArrays& la)
{
    const int lane = threadIdx.x & 31;
    const int q = lane / c.lpl;
    LineJob J;
    J.n = n;
    J.lpl = c.lpl;
    J.T = c.T;
    J.j = lane - q * c.lpl;
    J.li = job * c.nlw + q;
    J.lv = J.li < nlines;
    J.lt = lt;
    J.ut = ut;
    J.R = R;
    J.E = wb + (size_t)q * 4 * c.nb;
    J.UE = J.E + c.nb;
    J.F = J.UE + c.nb;
    J.CR = J.F + c.nb;
    const int L = c.lpl;
    // the lines' face Courant numbers: asynchronous copies from the per-CTA
    // table (L2), in flight while the lines are copied out of the plane
    {
        const double* src = crtab + (size_t)J.li * n + J.j;
        double* dst = J.CR + J.j;
        const int nv = J.lv ? n : 0;
        int x = J.j;
        for (; x < nv; x += L, src += L, dst += L) cp_async8(dst, src);
        for (; x <= L * c.T; x += L, dst += L) *dst = 0.0;
        cp_async_commit();
    }
    J.lbc = J.lv ? la.lb[J.li] : 0.0;
    J.ubc = J.lv ? la.ub[J.li] : 0.0;
    J.dxl = J.lv ? la.dxl[J.li] : 0.0;
    J.dxu = J.lv ? la.dxu[J.li] : 0.0;
    J.ns = J.lv ? la.ns[J.li] : 0;
    J.nsmax = __reduce_max_sync(0xffffffffu, J.ns);
    const unsigned dir = __reduce_or_sync(0xffffffffu, J.lv ? (unsigned)la.dir[J.li] : 0u);
    // E (QUICKEST6.cpp:89-91), then its ghost cells
    {
        const double* sp = RS ? S + J.li * R + J.j : S + J.j * R + J.li;
        const int sstep = RS ? L : L * R;
        double* e = J.E + 5 + J.j;
        const int nv = J.lv ? n : 0;
#pragma unroll 2
        for (int x = J.j; x < nv; x += L, sp += sstep, e += L) *e = *sp;
    }
    __syncwarp();
    if (J.lv) {
        fill_ghosts3(J.E, J, true, true);
        if (ut == VERB_BC_CONSTANT_VALUE)
            for (int gi = J.j; gi < 10; gi += L)
                if (gi >= 5) J.UE[n + gi] = J.ubc;
    }
    cp_async_wait_all();
    __syncwarp();
    if (dir == 2u) job_substeps<RS, DIR_NEG>(S, J);
    else if (dir == 3u) job_substeps<RS, DIR_MIX>(S, J);
    else job_substeps<RS, DIR_POS>(S, J);
}

// offset (doubles) of the warp buffers in the dynamic shared memory: plane,
// per-line arrays, reduction slots and the int sub-step counts, rounded up to
// 16 bytes
__host__ __device__ inline int conv_wall_offset(int P, int R)
{
    const int o = P * R + 4 * R + 4 * P + 32 + (R + P);
    return (o + 1) & ~1;
}

__host__ __device__ inline size_t conv_scratch_per_cta(int P, int R)
{
    return (size_t)(R > 1 ? R - 1 : 1) * P + 4 * (size_t)P * R;
}

__global__ void __launch_bounds__(C3_THREADS, 2) convection_kernel(ConvArgs a)
{
    extern __shared__ double sm[];
    const Dims d = a.d;
    const int P = d.P, R = d.R, V = d.V, K = d.K;
    const int PR = P * R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* S = sm;                // [P][R]
    double* lbP = S + PR;          // per P-line (index iR): lbc, ubc, dxl, dxu
    double* ubP = lbP + R;
    double* dxP = ubP + R;
    double* dxPu = dxP + R;
    double* lbR = dxPu + R;        // per R-line (index iP)
    double* ubR = lbR + P;
    double* dxR = ubR + P;
    double* dxRu = dxR + P;
    double* red = dxRu + P;        // [32]
    int* nsP = (int*)(red + 32);   // [R] per-line sub-steps
    int* nsR = nsP + R;            // [P]
    int* dirP = nsR + P;           // [R] per-line face directions: bit 0 some Courant >= 0,
    int* dirR = dirP + R;          // [P]                           bit 1 some Courant < 0
    const int wstride = conv_wstride(P, R);
    double* wall = sm + conv_wall_offset(P, R);  // pointer arithmetic on sm keeps LDS/STS
    double* wb = wall + (size_t)warp * wstride;
    __shared__ int s_ticket;

    // line buffers start as zeros: ghost slots that a sweep never writes are
    // read only by padding lanes, whose results are discarded
    for (int i = threadIdx.x; i < C3_WARPS * wstride; i += blockDim.x) wall[i] = 0.0;

    const SweepCfg cP = sweep_cfg(P, R - 1), cR = sweep_cfg(R, P);
    const size_t VK = (size_t)V * K;
    double* crP = a.scratch + (size_t)blockIdx.x * conv_scratch_per_cta(P, R);  // [R-1][P]
    double* crR = crP + (size_t)(R > 1 ? R - 1 : 1) * P;                       // [P][R]
    double* gpl = crR + PR;    // G of the slice
    double* lexp = gpl + PR;   // exp(Loss dt)
    double* spl = lexp + PR;   // Sources dt
    const int nslices = V * K;
    const LineArrays laP{lbP, ubP, dxP, dxPu, nsP, dirP};
    const LineArrays laR{lbR, ubR, dxR, dxRu, nsR, dirR};
    // first face of a line that the reference sweeps (face 0 only when periodic)
    const int ixP0 = a.Pl_t == VERB_BC_PERIODIC ? 0 : 1;
    const int ixR0 = a.Rl_t == VERB_BC_PERIODIC ? 0 : 1;
    // the thread's first L index and its advance per C3_THREADS cells
    const int iR0 = threadIdx.x % R, iRstep = C3_THREADS % R;

    for (;;) {
        if (threadIdx.x == 0) s_ticket = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int t = s_ticket;
        __syncthreads();
        if (t >= nslices) break;
        const int iV = V - 1 - t / K;
        const int iK = t - (t / K) * K;
        const size_t off = (size_t)iV * K + iK;
        auto g = [&](int iP, int iR) { return ((size_t)iP * R + iR) * VK + off; };

        // slice load and slice-level sub-step count (src/Convection_2D.cpp:57-86)
        double vpm = 0.0, vrm = 0.0;
        for (int i = threadIdx.x; i < PR; i += blockDim.x) {
            const int iP = i / R, iR = i - iP * R;
            const size_t gi = g(iP, iR);
            S[i] = a.psd[gi];
            const double vp = fabs(a.VP[gi]), vr = fabs(a.VR[gi]);
            vpm = (vpm < vp) ? vp : vpm;
            vrm = (vrm < vr) ? vr : vrm;
        }
        vpm = block_max(vpm, red);
        vrm = block_max(vrm, red);
        double nsp = 1, nsr = 1;
        if (P >= 3) {
            const double dP = a.Pg[g(1, 0)] - a.Pg[g(0, 0)];
            const double x = (double)a.dt * vpm / dP / 0.25;
            nsp = x <= 1 ? 1 : ceil(x);
        }
        if (R >= 3) {
            const double dR = a.Rg[g(0, 1)] - a.Rg[g(0, 0)];
            const double x = (double)a.dt * vrm / dR / 0.25;
            nsr = x <= 1 ? 1 : ceil(x);
        }
        const double num_steps = (nsp < nsr) ? nsr : nsp;
        if (!(num_steps <= MAX_SUBSTEPS)) {  // also catches inf / NaN
            if (threadIdx.x == 0) {
                a.substeps[off] = -1;
                set_error(a.status, VERB_ERR_CFL);
            }
            __syncthreads();
            continue;
        }
        const double dtc = a.dt / num_steps;
        if (threadIdx.x == 0) a.substeps[off] = (int)num_steps;
        for (int i = threadIdx.x; i < PR; i += blockDim.x) {
            const int iP = i / R, iR = i - iP * R;
            const size_t gi = g(iP, iR);
            lexp[i] = exp(a.loss[gi] * dtc);
            gpl[i] = a.G[gi];
            spl[i] = a.S[gi] * dtc;
        }

        // per-line CFL sub-cycles and face Courant numbers (QUICKEST6.cpp:37-52,
        // 150-160), one warp per line
        if (P >= 3) {
            for (int iR = warp; iR < R - 1; iR += C3_WARPS) {
                double m = -INFINITY;
                for (int iP = lane; iP < P; iP += 32) {
                    const double v = fabs(a.VP[g(iP, iR)]);
                    m = (m > v) ? m : v;
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const double q = __shfl_xor_sync(0xffffffffu, m, o);
                    m = (m > q) ? m : q;
                }
                const double dx = a.Pg[g(1, iR)] - a.Pg[g(0, iR)];
                const double sd = (double)dtc * m / dx / 1.0;
                int ns = 1;
                if (!(sd <= MAX_SUBSTEPS)) set_error(a.status, VERB_ERR_CFL);
                else if (sd > 1) ns = (int)ceil(sd);
                const double dtl = dtc / ns;
                if (fabs(m / dx * dtl) > 1) set_error(a.status, VERB_ERR_CFL);
                unsigned dir = 0;
                for (int ix = lane; ix < P; ix += 32) {
                    const int i0 = ix == 0 ? P - 2 : ix - 1;
                    const double c0 = a.VP[g(i0, iR)] / dx * dtl;
                    const double c1 = a.VP[g(ix, iR)] / dx * dtl;
                    const double cr = (c0 + c1) / 2;
                    crP[(size_t)iR * P + ix] = cr;
                    if (ix >= ixP0) dir |= cr >= 0 ? 1u : (cr < 0 ? 2u : 0u);
                }
                dir = __reduce_or_sync(0xffffffffu, dir);
                if (lane == 0) {
                    dirP[iR] = (int)dir;
                    nsP[iR] = ns;
                    dxP[iR] = dx;
                    dxPu[iR] = a.Pg[g(P - 1, iR)] - a.Pg[g(P - 2, iR)];
                    const size_t bo = ((size_t)iR * V + iV) * K + iK;
                    lbP[iR] = a.Pl[bo];
                    ubP[iR] = a.Pu[bo];
                }
            }
        }
        if (R >= 3) {
            for (int iP = warp; iP < P; iP += C3_WARPS) {
                double m = -INFINITY;
                for (int iR = lane; iR < R; iR += 32) {
                    const double v = fabs(a.VR[g(iP, iR)]);
                    m = (m > v) ? m : v;
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const double q = __shfl_xor_sync(0xffffffffu, m, o);
                    m = (m > q) ? m : q;
                }
                const double dx = a.Rg[g(iP, 1)] - a.Rg[g(iP, 0)];
                const double sd = (double)dtc * m / dx / 1.0;
                int ns = 1;
                if (!(sd <= MAX_SUBSTEPS)) set_error(a.status, VERB_ERR_CFL);
                else if (sd > 1) ns = (int)ceil(sd);
                const double dtl = dtc / ns;
                if (fabs(m / dx * dtl) > 1) set_error(a.status, VERB_ERR_CFL);
                unsigned dir = 0;
                for (int ix = lane; ix < R; ix += 32) {
                    const int i0 = ix == 0 ? R - 2 : ix - 1;
                    const double c0 = a.VR[g(iP, i0)] / dx * dtl;
                    const double c1 = a.VR[g(iP, ix)] / dx * dtl;
                    const double cr = (c0 + c1) / 2;
                    crR[(size_t)iP * R + ix] = cr;
                    if (ix >= ixR0) dir |= cr >= 0 ? 1u : (cr < 0 ? 2u : 0u);
                }
                dir = __reduce_or_sync(0xffffffffu, dir);
                if (lane == 0) {
                    dirR[iP] = (int)dir;
                    nsR[iP] = ns;
                    dxR[iP] = dx;
                    dxRu[iP] = a.Rg[g(iP, R - 1)] - a.Rg[g(iP, R - 2)];
                    const size_t bo = ((size_t)iP * V + iV) * K + iK;
                    lbR[iP] = a.Rl[bo] * a.G[g(iP, 0)];
                    ubR[iP] = a.Ru[bo] * a.G[g(iP, R - 1)];
                }
            }
        }
        __syncthreads();

        for (int it = 0; it < num_steps; it++) {
            if (P >= 3) {
                // P-lines iR = 0 .. R-2 (the last R row is not swept, :104)
                for (int job = warp; job < cP.njobs; job += C3_WARPS)
                    sweep_job<false>(S, wb, cP, job, P, R - 1, R, a.Pl_t, a.Pu_t, crP, laP);
                __syncthreads();
            }
            if (R >= 3) {
#pragma unroll 4
                for (int i = threadIdx.x; i < PR; i += C3_THREADS) S[i] = S[i] * gpl[i];
                __syncthreads();
                for (int job = warp; job < cR.njobs; job += C3_WARPS)
                    sweep_job<true>(S, wb, cR, job, R, P, R, a.Rl_t, a.Ru_t, crR, laR);
                __syncthreads();
                int iR = iR0;
#pragma unroll 4
                for (int i = threadIdx.x; i < PR; i += C3_THREADS) {
                    double x = S[i] / gpl[i];
                    x = x * lexp[i];
                    if (iR >= 1 && iR < R - 1) x = x + spl[i];
                    S[i] = x;
                    iR += iRstep;
                    if (iR >= R) iR -= R;
                }
                __syncthreads();
            } else {
                // no R-sweep: exp(loss dt) and sources only (:147-165)
                int iR = iR0;
                for (int i = threadIdx.x; i < PR; i += C3_THREADS) {
                    double x = S[i] * lexp[i];
                    if (iR >= 1 && iR < R - 1) x = x + spl[i];
                    S[i] = x;
                    iR += iRstep;
                    if (iR >= R) iR -= R;
                }
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < PR; i += blockDim.x) {
            const int iP = i / R, iR = i - iP * R;
            a.psd[g(iP, iR)] = S[i];
        }
        __syncthreads();
    }
}

// Convection_1D_ULTIMATE_QUICKEST6 on one line (per-slice entry point).
__global__ void __launch_bounds__(CONV_THREADS)
    convection_line_kernel(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                           int ubc_t, const double* ux, double dt_total, int* status)
{
    extern __shared__ double sm[];
    double* S = sm;
    double* U = sm + n;
    double* F = sm + 2 * n;
    double* CO = sm + 3 * n;
    double* red = sm + 4 * n;
    double m = -INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        S[i] = psd[i];
        const double v = fabs(ux[i]);
        m = (m > v) ? m : v;
    }
    m = block_max(m, red);
    const double dx = x[1] - x[0];
    const double sd = (double)dt_total * m / dx / 1.0;
    int ns = 1;
    if (!(sd <= MAX_SUBSTEPS)) {
        if (threadIdx.x == 0) set_error(status, VERB_ERR_CFL);
        return;
    }
    if (sd > 1) ns = (int)ceil(sd);
    const double dt = dt_total / ns;
    for (int i = threadIdx.x; i < n; i += blockDim.x) CO[i] = ux[i] / dx * dt;
    if (threadIdx.x == 0 && fabs(m / dx * dt) > 1) set_error(status, VERB_ERR_CFL);
    __syncthreads();
    const Sweep w{n, lbc_t, ubc_t};
    Line L0;
    L0.base = 0;
    L0.stride = 1;
    L0.lbc = lbc;
    L0.ubc = ubc;
    L0.dxl = dx;
    L0.dxu = x[n - 1] - x[n - 2];
    for (int it = 0; it < ns; it++) {
        quickest_pass(S, U, F, CO, 1, w, true, [&](int) { return L0; }, [&](int) { return true; });
        double* t = S;
        S = U;
        U = t;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) psd[i] = S[i];
}

}  // namespace
}  // namespace VERB_CONV_NS
using namespace VERB_CONV_NS;

#ifdef VERB_BUILD_CONV_FMA

size_t conv_smem_bytes_fma(int P, int R)
{
    return ((size_t)conv_wall_offset(P, R) + (size_t)C3_WARPS * conv_wstride(P, R)) * sizeof(double);
}

int conv_check_fma(int P, int R)
{
    if ((P >= 3 && sweep_cfg(P, R - 1).lpl == 0) || (R >= 3 && sweep_cfg(R, P).lpl == 0))
        return VERB_ERR_SIZE;
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (conv_smem_bytes_fma(P, R) > (size_t)maxsm) return VERB_ERR_SIZE;
    return VERB_OK;
}

int conv_ctas_fma(int P, int R)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = conv_smem_bytes_fma(P, R);
    allow_max_dynamic_smem((const void*)convection_kernel);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, convection_kernel, C3_THREADS, smem);
    if (per < 1) per = 1;
    return sms * per;
}

void launch_convection_fma(const ConvArgs& a, int nctas, cudaStream_t s)
{
    const size_t smem = conv_smem_bytes_fma(a.d.P, a.d.R);
    allow_max_dynamic_smem((const void*)convection_kernel);
    convection_kernel<<<nctas, C3_THREADS, smem, s>>>(a);
}

#else

size_t conv_smem_bytes(int P, int R)
{
    return ((size_t)conv_wall_offset(P, R) + (size_t)C3_WARPS * conv_wstride(P, R)) * sizeof(double);
}

size_t conv_scratch_doubles(int P, int R) { return conv_scratch_per_cta(P, R); }

int conv_check(int P, int R)
{
    if ((P >= 3 && sweep_cfg(P, R - 1).lpl == 0) || (R >= 3 && sweep_cfg(R, P).lpl == 0))
        return VERB_ERR_SIZE;
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (conv_smem_bytes(P, R) > (size_t)maxsm) return VERB_ERR_SIZE;
    return VERB_OK;
}

int conv_ctas(int P, int R)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = conv_smem_bytes(P, R);
    allow_max_dynamic_smem((const void*)convection_kernel);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, convection_kernel, C3_THREADS, smem);
    if (per < 1) per = 1;
    return sms * per;
}

void launch_convection(const ConvArgs& a, int nctas, cudaStream_t s)
{
    const size_t smem = conv_smem_bytes(a.d.P, a.d.R);
    allow_max_dynamic_smem((const void*)convection_kernel);
    convection_kernel<<<nctas, C3_THREADS, smem, s>>>(a);
}

void launch_convection_line(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                            int ubc_t, const double* ux, double dt, int* status, cudaStream_t s)
{
    const size_t smem = (size_t)(4 * n + 32) * sizeof(double);
    allow_max_dynamic_smem((const void*)convection_line_kernel);
    convection_line_kernel<<<1, CONV_THREADS, smem, s>>>(psd, x, n, lbc, ubc, lbc_t, ubc_t, ux, dt,
                                                        status);
}

#endif  // VERB_BUILD_CONV_FMA

}  // namespace verb
