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
// shared memory for all of its CFL sub-steps, in a plane X of (P + 2 GST) x RS
// doubles with GST = 5 ghost rows above and below and GST ghost columns left
// and right of the P x R interior (QUICKEST6.cpp:89-143 extends every 1-D line
// by five ghost cells per side).  A sweep is a set of independent lines
// (P-lines: one per L index, along MLT; R-lines: one per MLT index, along L).
// A warp takes 32/lpl lines per job with lpl lanes per line, and lane j of a
// line owns the T consecutive cells jT .. jT+T-1 of the line, and their left
// faces, for the whole job: their values live in registers.  A sub-step of a
// job:
//   ghosts of E          from the line's boundary types, into the plane's
//                        ghost slots of the line (lanes 0..9 of the line)
//   A  window W = E[jT-5 .. jT+T+3] from the plane (T+9 shared loads); the
//      lane's T unlimited face values from it (QUICKEST6.cpp:148-241)
//   B  unlimited cells UE = E - (c F)_right + (c F)_left with the right
//      neighbour's first face by a shuffle; written over E in the plane,
//      then the boundary rewrite of cells 0 and n-1 and UE's high ghosts
//      (the low ghosts stay E's, as the reference takes them from the
//      pre-step PSD, :283-302)                              (:243-272, 277-330)
//   C  window UE[jT-4 .. jT+T+2] from the plane; the limited face values from
//      it and from E's window (registers)                   (:332-447)
//   D  final cells into the plane and their boundary rewrite (:448-477)
// with warp synchronisation only; the CTA synchronises between sweeps.  A
// lane thus reads T+9 + T+7 and writes about 2T doubles of shared memory per
// sub-step for its T faces, and the face arithmetic runs on registers.
//
// The face Courant numbers of every line are computed once per slice into a
// per-CTA table in global memory (L2-resident), laid out [line][t][lane] so
// that the lanes of a warp load them with contiguous accesses.  The Courant
// factors of the face polynomial are recomputed per face from the Courant
// number with exactly rounded divisions by the constant denominators
// (div_const).  All faces of a job usually have the same upwind direction
// (the drift velocities are smooth along MLT and the radial velocity depends
// on MLT only), so a job is dispatched to a direction-specialised body in
// which the upwind stencil roles are fixed registers; jobs with mixed
// directions select the roles per face.
//
// The radial sweep works on PSD*G: with G not identically 1 on the slice a
// pass over the plane multiplies by G before it, and a pass /G, *exp(Loss dt),
// +S dt (interior L) follows it, in the reference's order
// (src/Convection_2D.cpp:122-165).  With G = 1 and exp(Loss dt) = 1 on the
// whole slice those factors are exact identities, and the sources are added by
// the R-sweep itself after its boundary rewrite.

// Warps per CTA (two CTAs per SM).  The contracted build needs fewer
// registers, so nine warps per CTA fit beside the exact build's eight in the
// same register file.  Nine warps split the 25 MLT-sweep jobs and the 24
// L-sweep jobs of a 48 x 101 slice into three rounds each.
#if defined(VERB_CONV_WARPS)
constexpr int C3_WARPS = VERB_CONV_WARPS;
#else
constexpr int C3_WARPS = 8;
#endif
constexpr int C3_THREADS = C3_WARPS * 32;
constexpr int GST = 5;  // ghost cells per side
constexpr unsigned FULL = 0xffffffffu;

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

// Face value of face x from w_k = E[x-5+k].  Courant >= 0: upwind centre
// x-1, U_k = E[x-1-k], D_k = E[x-1+k]; Courant < 0: centre x, U_k = E[x+k],
// D_k = E[x-k] (QUICKEST6.cpp:169-186).
template <int DIR>
__device__ __forceinline__ double face10(double w0, double w1, double w2, double w3, double w4,
                                         double w5, double w6, double w7, double w8, double w9,
                                         double cr)
{
    const FaceCoef k = face_coef_exact(cr);
    if (DIR == DIR_POS) return QUICKEST_FACE(w3, w2, w1, w0, w4, w5, w6, w7, w8, w9, cr, k);
    if (DIR == DIR_NEG) return QUICKEST_FACE(w6, w7, w8, w9, w5, w4, w3, w2, w1, w0, cr, k);
    const bool up = cr >= 0;
    return QUICKEST_FACE(up ? w3 : w6, up ? w2 : w7, up ? w1 : w8, up ? w0 : w9, up ? w4 : w5,
                         up ? w5 : w4, up ? w6 : w3, up ? w7 : w2, up ? w8 : w1, up ? w9 : w0, cr,
                         k);
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

// Limited face value of face x from u_k = UE[x-4+k] (k = 0..7) and
// e_k = E[x-2+k] (k = 0..3).
template <int DIR>
__device__ __forceinline__ double limit12(double f, double cr, double u0, double u1, double u2,
                                          double u3, double u4, double u5, double u6, double u7,
                                          double e0, double e1, double e2, double e3)
{
    if (DIR == DIR_POS) return quickest_limit_sel(f, cr, e0, e1, e2, u2, u1, u0, u3, u4, u5, u6);
    if (DIR == DIR_NEG) return quickest_limit_sel(f, cr, e3, e2, e1, u5, u6, u7, u4, u3, u2, u1);
    const bool up = cr >= 0;
    return quickest_limit_sel(f, cr, up ? e0 : e3, up ? e1 : e2, up ? e2 : e1, up ? u2 : u5,
                              up ? u1 : u6, up ? u0 : u7, up ? u3 : u4, up ? u4 : u3,
                              up ? u5 : u2, up ? u6 : u1);
}

// Cells per lane the kernel is compiled for; a sweep's shape uses the
// smallest of them that covers its lines.  Up to 8 with every direction
// body, 10, 12 and 16 (lines of up to 512 points) with the mixed-direction
// body only.
__host__ __device__ inline int t_allowed(int t)
{
    if (t <= 3) return 3;
    if (t <= 8) return t;
    if (t <= 10) return 10;
    if (t <= 12) return 12;
    if (t <= 16) return 16;
    return 0;
}

// Work split of one sweep: nlines lines of n points, lpl lanes per line, T
// cells per lane.  The choice models a job's cost as a fixed part (line
// set-up, ghost cells, loads of the windows, synchronisation) plus a part per
// cell, and counts half of the idle warp slots of the last round (the other
// CTA on the SM fills the rest).
struct SweepCfg {
    int lpl, T, nlw, njobs;
};

__host__ __device__ inline SweepCfg sweep_cfg(int n, int nlines)
{
    SweepCfg best{0, 0, 0, 0};
    double bc = 0.0;
    // shapes with at most 8 cells per lane (every direction body) first; ties
    // go to fewer lanes per line (less padding)
    for (int pass = 0; pass < 2 && best.lpl == 0; pass++) {
        for (int lpl = 4; lpl <= 32; lpl <<= 1) {
            const int T = t_allowed((n + lpl - 1) / lpl);
            if (T == 0 || (T > 8) != (pass == 1)) continue;
            const int nlw = 32 / lpl;
            const int jobs = (nlines + nlw - 1) / nlw;
            const int rounds = (jobs + C3_WARPS - 1) / C3_WARPS;
            const double job = 300.0 + 200.0 * T;
            const double cost = job * (jobs + 0.5 * (rounds * C3_WARPS - jobs));
            if (best.lpl == 0 || cost < bc - 1e-9) {
                bc = cost;
                best = SweepCfg{lpl, T, nlw, jobs};
            }
        }
    }
    return best;  // lpl == 0: lines longer than 32*16 points
}

// row stride of the plane: R + 2 GST, odd, so that the MLT sweep's strided
// accesses (stride T*RS between lanes) fall on distinct banks
__host__ __device__ inline int plane_stride(int R)
{
    const int rs = R + 2 * GST;
    return rs | 1;
}

__host__ __device__ inline int plane_doubles(int P, int R) { return (P + 2 * GST) * plane_stride(R); }

// offset (doubles) of the per-line arrays after the plane
__host__ __device__ inline size_t conv_table_doubles(int P, int R, size_t* off_r);

__host__ __device__ inline int conv_smem_doubles(int P, int R)
{
    const int base = plane_doubles(P, R) + 4 * R + 4 * P + 32 + (R + P) + 2;
#ifdef VERB_CONV_CR_SMEM
    return base + (int)conv_table_doubles(P, R, nullptr);  // Courant tables in shared memory
#else
    return base;
#endif
}

// per-CTA scratch: the Courant tables of both sweeps ([line][T][lpl]) and
// the G, exp(Loss dt) and Sources dt planes
__host__ __device__ inline size_t conv_table_doubles(int P, int R, size_t* off_r)
{
    size_t tp = 0, tr = 0;
    if (P >= 3) {
        const SweepCfg c = sweep_cfg(P, R - 1);
        tp = (size_t)(R > 1 ? R - 1 : 1) * c.T * c.lpl;
    }
    if (R >= 3) {
        const SweepCfg c = sweep_cfg(R, P);
        tr = (size_t)P * c.T * c.lpl;
    }
    if (off_r) *off_r = tp;
    return tp + tr;
}

__host__ __device__ inline size_t conv_scratch_per_cta(int P, int R)
{
    return conv_table_doubles(P, R, nullptr) + 3 * (size_t)P * R;
}

// One sweep as the jobs of a warp see it.
struct SweepRun {
    double* X;                  // the plane
    int RS;                     // its row stride
    bool rsw;                   // R-sweep (lines are rows) or MLT sweep (lines are columns)
    int n, nlines, lt, ut, lpl, T;
    const double* crtab;        // [line][T][lpl] face Courant numbers
    const double *lb, *ub, *dxl, *dxu;  // per line
    const int *ns, *dir;
    // R-sweep with G = 1 and exp(Loss dt) = 1: Sources*dt of interior cells
    // added after the line's last sub-step ([P][R], or +0 everywhere)
    bool fuse_src;
    const double* spl;
    bool spl_zero;
    int R;
};

// All sub-steps of one job (QUICKEST6.cpp:37-52 sub-cycle, one pass per
// sub-step), with T cells per lane and the stencil roles of direction DIR.
template <int T, int DIR>
__device__ __forceinline__ void sweep_job(const SweepRun& s, int job)
{
    const int lane = threadIdx.x & 31;
    const int lpl = s.lpl;
    const int q = lane / lpl;
    const int j = lane - q * lpl;
    const int n = s.n;
    int li = job * (32 / lpl) + q;
    const bool lv = li < s.nlines;
    if (!lv) li = s.nlines - 1;  // a line to read from; nothing is written
    const int xs = s.rsw ? 1 : s.RS;
    double* const X0 = s.X + (s.rsw ? (li + GST) * s.RS + GST : GST * s.RS + li + GST);
    const int c0 = j * T;
    const int xmax = n - 1 + GST;  // last ghost slot
    const int lt = s.lt, ut = s.ut;
    const double lbc = s.lb[li], ubc = s.ub[li], dxl = s.dxl[li], dxu = s.dxu[li];
    const int ns = lv ? s.ns[li] : 0;
    const int nsmax = __reduce_max_sync(FULL, ns);
    const int jl = (n - 1) / T;  // the lane that owns cell n-1

    // Courant numbers of the lane's faces and of the right neighbour's first
    // face
    const double* const ct0 = s.crtab + (size_t)li * T * lpl + j;
#ifdef VERB_CONV_CR_REG
    double crr[T];
#pragma unroll
    for (int t = 0; t < T; t++) crr[t] = ct0[t * lpl];
#define CT(t) crr[t]
#else
#define CT(t) ct0[(t) * lpl]
#endif
    const double crn = __shfl_down_sync(FULL, CT(0), 1, lpl);

    // ghost cells of E (QUICKEST6.cpp:94-140): ghost gi < 5 is low ghost
    // gi+1, gi >= 5 high ghost gi-4; the lanes of a line take the ten in turn
    auto fill_ghosts = [&](bool low) {
        for (int gi = j; gi < 2 * GST; gi += lpl) {
            const bool hi = gi >= GST;
            if (!low && !hi) continue;
            const int ig = hi ? gi - GST + 1 : gi + 1;
            const int type = hi ? ut : lt;
            double g;
            if (type == VERB_BC_PERIODIC) {
                g = X0[(hi ? ig : (n - 1) - ig) * xs];
            } else if (type == VERB_BC_CONSTANT_VALUE) {
                g = hi ? ubc : lbc;
            } else {
                const double c = hi ? ubc * dxu : lbc * dxl;
                g = hi ? X0[(n - 1) * xs] + c : X0[0] - c;
                for (int i = 2; i <= ig; i++) g = hi ? g + c : g - c;
            }
            X0[(hi ? (n - 1) + ig : -ig) * xs] = g;
        }
    };
    // boundary rewrite of cells 0 and n-1 (:257-272 / 457-477)
    auto edge_fix = [&]() {
        if (j == 0 && lt != VERB_BC_PERIODIC)
            X0[0] = lt == VERB_BC_CONSTANT_VALUE ? lbc : X0[xs];
        if (j == jl) {
            double v;
            if (ut == VERB_BC_CONSTANT_VALUE) v = ubc;
            else if (ut == VERB_BC_CONSTANT_DERIVATIVE) v = X0[(n - 2) * xs];
            else v = X0[0];  // periodic: f[n-1] = f[0]
            X0[(n - 1) * xs] = v;
        }
    };

    if (lv) fill_ghosts(true);
    for (int sub = 0; sub < nsmax; sub++) {
        const bool act = lv && sub < ns;
        __syncwarp();
        // A: the window of E and the unlimited faces
        double W[T + 9];
#pragma unroll
        for (int i = 0; i < T + 9; i++) W[i] = X0[min(c0 - GST + i, xmax) * xs];
        double F[T];
#pragma unroll
        for (int t = 0; t < T; t++)
            F[t] = face10<DIR>(W[t], W[t + 1], W[t + 2], W[t + 3], W[t + 4], W[t + 5], W[t + 6],
                               W[t + 7], W[t + 8], W[t + 9], CT(t));
        // B: unlimited cells (:245-249); cell 0 of a non-periodic line is
        // rewritten below, so its left flux (zero in the reference) is unused
        double fn = __shfl_down_sync(FULL, F[0], 1, lpl);
        double C[T];
#pragma unroll
        for (int t = 0; t < T; t++) {
            const double fr = t + 1 < T ? F[t + 1] : fn;
            const double cg = t + 1 < T ? CT(t + 1) : crn;
            C[t] = W[GST + t] - (cg * fr - CT(t) * F[t]);
        }
        __syncwarp();  // every lane has its window of E
        if (act) {
#pragma unroll
            for (int t = 0; t < T; t++)
                if (c0 + t <= n - 2) X0[(c0 + t) * xs] = C[t];
        }
        __syncwarp();
        if (act) edge_fix();
        __syncwarp();
        // UE's high ghosts from UE; its low ghosts stay E's (:283-326)
        if (act && ut != VERB_BC_CONSTANT_VALUE) fill_ghosts(false);
        __syncwarp();
        // C: the window of UE and the limited faces
        {
            double Uw[T + 7];
#pragma unroll
            for (int i = 0; i < T + 7; i++) Uw[i] = X0[min(c0 - 4 + i, xmax) * xs];
#pragma unroll
            for (int t = 0; t < T; t++)
                F[t] = limit12<DIR>(F[t], CT(t), Uw[t], Uw[t + 1], Uw[t + 2], Uw[t + 3], Uw[t + 4],
                                    Uw[t + 5], Uw[t + 6], Uw[t + 7], W[t + 3], W[t + 4], W[t + 5],
                                    W[t + 6]);
        }
        // D: final cells (:448-452)
        fn = __shfl_down_sync(FULL, F[0], 1, lpl);
#pragma unroll
        for (int t = 0; t < T; t++) {
            const double fr = t + 1 < T ? F[t + 1] : fn;
            const double cg = t + 1 < T ? CT(t + 1) : crn;
            C[t] = W[GST + t] - (cg * fr - CT(t) * F[t]);
        }
        __syncwarp();  // every lane has its window of UE
        if (act) {
#pragma unroll
            for (int t = 0; t < T; t++)
                if (c0 + t <= n - 2) X0[(c0 + t) * xs] = C[t];
        }
        __syncwarp();
        if (act) edge_fix();
        __syncwarp();
        if (act && sub + 1 < ns) {
            fill_ghosts(true);  // the next sub-step's ghosts of E
        } else if (act && s.fuse_src) {
            // the line's last sub-step: + Sources*dt on interior cells
            // (src/Convection_2D.cpp:156-165; /G and *exp(Loss dt) are
            // identities here).  Cells 1..n-2 still hold C.
            const double* sp = s.spl + (size_t)li * s.R;
#pragma unroll
            for (int t = 0; t < T; t++) {
                const int c = c0 + t;
                if (c >= 1 && c <= n - 2) X0[c * xs] = C[t] + (s.spl_zero ? 0.0 : sp[c]);
            }
        }
    }
    __syncwarp();  // the warp's next job overwrites what phase D wrote last
#undef CT
}

// One job: the body for the sweep's cells per lane and the job's directions
// (bit 0: some face Courant number >= 0, bit 1: some < 0).
__device__ __forceinline__ void run_job(const SweepRun& s, int job)
{
    const int lane = threadIdx.x & 31;
    const int li = job * (32 / s.lpl) + lane / s.lpl;
    const unsigned d = __reduce_or_sync(FULL, li < s.nlines ? (unsigned)s.dir[li] : 0u);
    const int dir = d == 2u ? DIR_NEG : (d == 3u ? DIR_MIX : DIR_POS);
#define VERB_JOB3(TT)                                              \
    case TT:                                                       \
        if (dir == DIR_POS) sweep_job<TT, DIR_POS>(s, job);        \
        else if (dir == DIR_NEG) sweep_job<TT, DIR_NEG>(s, job);   \
        else sweep_job<TT, DIR_MIX>(s, job);                       \
        break;
    switch (s.T) {
        VERB_JOB3(3)
        VERB_JOB3(4)
        VERB_JOB3(5)
        VERB_JOB3(6)
        VERB_JOB3(7)
        VERB_JOB3(8)
        case 10: sweep_job<10, DIR_MIX>(s, job); break;
        case 12: sweep_job<12, DIR_MIX>(s, job); break;
        default: sweep_job<16, DIR_MIX>(s, job); break;
    }
#undef VERB_JOB3
}

#ifndef VERB_CONV_MINB
#define VERB_CONV_MINB 2
#endif
__global__ void __launch_bounds__(C3_THREADS, VERB_CONV_MINB) convection_kernel(ConvArgs a)
{
    extern __shared__ double sm[];
    const Dims d = a.d;
    const int P = d.P, R = d.R, V = d.V, K = d.K;
    const int PR = P * R;
    const int RS = plane_stride(R);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* X = sm;                          // [P + 2 GST][RS]
    double* lbP = X + plane_doubles(P, R);   // per P-line (index iR): lbc, ubc, dxl, dxu
    double* ubP = lbP + R;
    double* dxP = ubP + R;
    double* dxPu = dxP + R;
    double* lbR = dxPu + R;                  // per R-line (index iP)
    double* ubR = lbR + P;
    double* dxR = ubR + P;
    double* dxRu = dxR + P;
    double* red = dxRu + P;                  // [32]
    int* nsP = (int*)(red + 32);             // [R] per-line sub-steps
    int* nsR = nsP + R;                      // [P]
    int* dirP = nsR + P;                     // [R] per-line face directions: bit 0 some Courant >= 0,
    int* dirR = dirP + R;                    // [P]                           bit 1 some Courant < 0
    __shared__ int s_ticket, s_flags;
    auto xi = [&](int iP, int iR) { return (iP + GST) * RS + iR + GST; };

    const SweepCfg cP = sweep_cfg(P, R - 1), cR = sweep_cfg(R, P);
    const size_t VK = (size_t)V * K;
    size_t offR = 0;
    const size_t ntab = conv_table_doubles(P, R, &offR);
    double* crP = a.scratch + (size_t)blockIdx.x * conv_scratch_per_cta(P, R);  // [R-1][TP][lplP]
    double* gpl = crP + ntab;  // G of the slice
#ifdef VERB_CONV_CR_SMEM
    crP = (double*)(dirR + P) + 1;  // after the int arrays, 8-byte aligned (+1 for odd P+R)
    crP = (double*)(((size_t)crP + 7) & ~(size_t)7);
#endif
    double* crR = crP + offR;                                                  // [P][TR][lplR]
    double* lexp = gpl + PR;   // exp(Loss dt)
    double* spl = lexp + PR;   // Sources dt
    const int nslices = V * K;
    // first face of a line that the reference sweeps (face 0 only when periodic)
    const int ixP0 = a.Pl_t == VERB_BC_PERIODIC ? 0 : 1;
    const int ixR0 = a.Rl_t == VERB_BC_PERIODIC ? 0 : 1;

    SweepRun sP{};
    sP.X = X;
    sP.RS = RS;
    sP.rsw = false;
    sP.n = P;
    sP.nlines = R - 1;  // the last R row is not swept (src/Convection_2D.cpp:104)
    sP.lt = a.Pl_t;
    sP.ut = a.Pu_t;
    sP.lpl = cP.lpl;
    sP.T = cP.T;
    sP.crtab = crP;
    sP.lb = lbP;
    sP.ub = ubP;
    sP.dxl = dxP;
    sP.dxu = dxPu;
    sP.ns = nsP;
    sP.dir = dirP;
    sP.fuse_src = false;
    SweepRun sR{};
    sR.X = X;
    sR.RS = RS;
    sR.rsw = true;
    sR.n = R;
    sR.nlines = P;
    sR.lt = a.Rl_t;
    sR.ut = a.Ru_t;
    sR.lpl = cR.lpl;
    sR.T = cR.T;
    sR.crtab = crR;
    sR.lb = lbR;
    sR.ub = ubR;
    sR.dxl = dxR;
    sR.dxu = dxRu;
    sR.ns = nsR;
    sR.dir = dirR;
    sR.spl = spl;
    sR.R = R;

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
            X[xi(iP, iR)] = a.psd[gi];
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
        if (threadIdx.x == 0) {
            a.substeps[off] = (int)num_steps;
            s_flags = 7;
        }
        __syncthreads();
        // G, exp(Loss dt), Sources dt of the slice; flags: bit 0 G == 1
        // everywhere, bit 1 exp(Loss dt) == 1 everywhere, bit 2 Sources dt
        // is +0 everywhere
        {
            int fl = 7;
            for (int i = threadIdx.x; i < PR; i += blockDim.x) {
                const int iP = i / R, iR = i - iP * R;
                const size_t gi = g(iP, iR);
                const double le = exp(a.loss[gi] * dtc);
                const double gg = a.G[gi];
                const double sd = a.S[gi] * dtc;
                lexp[i] = le;
                gpl[i] = gg;
                spl[i] = sd;
                if (!(gg == 1.0)) fl &= ~1;
                if (!(le == 1.0)) fl &= ~2;
                if (__double_as_longlong(sd) != 0) fl &= ~4;
            }
            fl = __reduce_and_sync(FULL, fl);
            if (lane == 0 && fl != 7) atomicAnd(&s_flags, fl);
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
                    const double q = __shfl_xor_sync(FULL, m, o);
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
                double* tab = crP + (size_t)iR * cP.T * cP.lpl;
                for (int ix = lane; ix < cP.T * cP.lpl; ix += 32) {
                    double cr = 0.0;
                    if (ix < P) {
                        const int i0 = ix == 0 ? P - 2 : ix - 1;
                        const double c0 = a.VP[g(i0, iR)] / dx * dtl;
                        const double c1 = a.VP[g(ix, iR)] / dx * dtl;
                        cr = (c0 + c1) / 2;
                        if (ix >= ixP0) dir |= cr >= 0 ? 1u : (cr < 0 ? 2u : 0u);
                    }
                    const int jj = ix / cP.T;
                    tab[(ix - jj * cP.T) * cP.lpl + jj] = cr;
                }
                dir = __reduce_or_sync(FULL, dir);
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
                    const double q = __shfl_xor_sync(FULL, m, o);
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
                double* tab = crR + (size_t)iP * cR.T * cR.lpl;
                for (int ix = lane; ix < cR.T * cR.lpl; ix += 32) {
                    double cr = 0.0;
                    if (ix < R) {
                        const int i0 = ix == 0 ? R - 2 : ix - 1;
                        const double c0 = a.VR[g(iP, i0)] / dx * dtl;
                        const double c1 = a.VR[g(iP, ix)] / dx * dtl;
                        cr = (c0 + c1) / 2;
                        if (ix >= ixR0) dir |= cr >= 0 ? 1u : (cr < 0 ? 2u : 0u);
                    }
                    const int jj = ix / cR.T;
                    tab[(ix - jj * cR.T) * cR.lpl + jj] = cr;
                }
                dir = __reduce_or_sync(FULL, dir);
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
        const int flags = s_flags;
        const bool fused = (flags & 3) == 3;  // G = 1 and exp(Loss dt) = 1
        sR.fuse_src = fused;
        sR.spl_zero = (flags & 4) != 0;

        for (int it = 0; it < num_steps; it++) {
            if (P >= 3) {
                // P-lines iR = 0 .. R-2 (the last R row is not swept, :104)
                for (int job = warp; job < cP.njobs; job += C3_WARPS) run_job(sP, job);
                __syncthreads();
            }
            if (R >= 3) {
                if (!(flags & 1)) {
                    for (int i = threadIdx.x; i < PR; i += C3_THREADS) {
                        const int iP = i / R, iR = i - iP * R;
                        X[xi(iP, iR)] = X[xi(iP, iR)] * gpl[i];
                    }
                    __syncthreads();
                }
                for (int job = warp; job < cR.njobs; job += C3_WARPS) run_job(sR, job);
                __syncthreads();
                if (!fused) {
                    for (int i = threadIdx.x; i < PR; i += C3_THREADS) {
                        const int iP = i / R, iR = i - iP * R;
                        double x = X[xi(iP, iR)] / gpl[i];
                        x = x * lexp[i];
                        if (iR >= 1 && iR < R - 1) x = x + spl[i];
                        X[xi(iP, iR)] = x;
                    }
                    __syncthreads();
                }
            } else {
                // no R-sweep: exp(loss dt) and sources only (:147-165)
                for (int i = threadIdx.x; i < PR; i += C3_THREADS) {
                    const int iP = i / R, iR = i - iP * R;
                    double x = X[xi(iP, iR)] * lexp[i];
                    if (iR >= 1 && iR < R - 1) x = x + spl[i];
                    X[xi(iP, iR)] = x;
                }
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < PR; i += blockDim.x) {
            const int iP = i / R, iR = i - iP * R;
            a.psd[g(iP, iR)] = X[xi(iP, iR)];
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

size_t conv_smem_bytes_fma(int P, int R) { return (size_t)conv_smem_doubles(P, R) * sizeof(double); }

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

size_t conv_smem_bytes(int P, int R) { return (size_t)conv_smem_doubles(P, R) * sizeof(double); }

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
