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
#include "verb_internal.cuh"

namespace verb {

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
// Slice kernel: warp-per-line 1-D passes.
//
// A warp owns whole lines (two P-lines or one R-line at a time).  It copies a
// line into a per-warp buffer E with its GST ghost cells materialised (so the
// 10-point stencils are branch-free shared-memory loads), runs the four phases
// of one ULTIMATE-QUICKEST sub-step with warp-level synchronisation only,
// and writes the result back into the slice plane S.  Block barriers remain
// only between the P-sweep and the R-sweep.  Face Courant numbers are
// precomputed once per slice (they are constant over its sub-steps) with the
// reference's expression (Ux[i-1]/dx*dt + Ux[i]/dx*dt)/2.  The R-sweep folds
// PSD*G into its load and /G, *exp(Loss dt), +S dt into its store, in the
// reference's order (src/Convection_2D.cpp:122-165).

constexpr int NW = CONV_THREADS / 32;

struct WLine {
    int base, stride;    // element ix of the line is S[base + ix*stride]
    const double* cf;    // face Courant numbers of the line, [n]
    const double* co;    // face coefficient table of the line (5 planes, stride nf) or nullptr
    double lbc, ubc, dxl, dxu;
    int ns;              // the line's own CFL sub-steps (QUICKEST6.cpp:37-52)
    int row;             // R-sweep: the MLT row iP
};

// per-line buffer: E [n+10] (orig values + ghosts), UE [n+10] (unlimited +
// ghosts), F [n] (face values)
__device__ __forceinline__ int line_buf(int n) { return 3 * n + 20; }

// Ghost cells t[k], k in [-GST,-1] and [n, n+GST-1], of an extended line whose
// interior sits at X[5..n+4] (QUICKEST6.cpp:92-143, 281-330).  Lane l < 5
// fills low ghost l+1, lanes 5..9 fill high ghost l-4.
__device__ __forceinline__ void fill_ghosts(double* X, const double* lowsrc, int n, int lt, int ut,
                                            const WLine& L, int lane)
{
    if (lane < 5) {
        const int ig = lane + 1;
        double g;
        if (lt == VERB_BC_PERIODIC) {
            g = lowsrc[5 + (n - 1) - ig];
        } else if (lt == VERB_BC_CONSTANT_VALUE) {
            g = L.lbc;
        } else {
            g = lowsrc[5] - L.lbc * L.dxl;
            for (int i = 2; i <= ig; i++) g = g - L.lbc * L.dxl;
        }
        X[5 - ig] = g;
    } else if (lane < 10) {
        const int ig = lane - 4;
        double g;
        if (ut == VERB_BC_PERIODIC) {
            g = X[5 + ig];
        } else if (ut == VERB_BC_CONSTANT_VALUE) {
            g = L.ubc;
        } else {
            g = X[5 + n - 1] + L.ubc * L.dxu;
            for (int i = 2; i <= ig; i++) g = g + L.ubc * L.dxu;
        }
        X[5 + (n - 1) + ig] = g;
    }
}

__device__ __forceinline__ double wcell_raw(const double* E, const double* F, const double* cf,
                                            int lt, int c)
{
    const double cr = cf[c + 1];
    const double fr = F[c + 1];
    double cl = 0.0, fl = 0.0;
    if (c > 0 || lt == VERB_BC_PERIODIC) {
        cl = cf[c];
        fl = F[c];
    }
    return E[5 + c] - (cr * fr - cl * fl);
}

__device__ __forceinline__ double wcell_final(const double* E, const double* F, const WLine& L, int n,
                                              int lt, int ut, int c)
{
    if (c == n - 1) {
        if (ut == VERB_BC_CONSTANT_VALUE) return L.ubc;
        if (ut == VERB_BC_CONSTANT_DERIVATIVE) return wcell_raw(E, F, L.cf, lt, n - 2);
        return wcell_raw(E, F, L.cf, lt, 0);
    }
    if (c == 0) {
        if (lt == VERB_BC_CONSTANT_VALUE) return L.lbc;
        if (lt == VERB_BC_CONSTANT_DERIVATIVE) return wcell_raw(E, F, L.cf, lt, 1);
    }
    return wcell_raw(E, F, L.cf, lt, c);
}

struct SliceIO {
    const double* G;     // global G_conv
    const double* src;   // global Sources
    const double* lexp;  // per-CTA exp(Loss dt) plane [P][R]
    const double* gpl;   // per-CTA G plane [P][R] (PRE only)
    const double* spl;   // per-CTA Sources*dt plane [P][R] (PRE only)
    size_t VK, off;
    int R;
    double dtc;
};

// Face value of face ix of an extended line E (QUICKEST6.cpp:162-241).  The
// upwind side comes from the sign of the Courant number: centre c and
// direction s give U_k = E[c - s k], D_k = E[c + s k] (:169-186).
template <bool PRE>
__device__ __forceinline__ double face_at(const double* E, const double* cf, const double* co,
                                          int nf, int ix)
{
    const double cr = cf[ix];
    const int up = cr >= 0 ? 1 : 0;
    const int c = 5 + ix - up;
    const int s = up ? 1 : -1;
    const double U1 = E[c - s], U2 = E[c - 2 * s], U3 = E[c - 3 * s], U4 = E[c - 4 * s];
    const double C = E[c];
    const double D1 = E[c + s], D2 = E[c + 2 * s], D3 = E[c + 3 * s], D4 = E[c + 4 * s],
                 D5 = E[c + 5 * s];
    if (PRE) {
        FaceCoef fk;
        fk.k3 = co[ix];
        fk.c6 = co[nf + ix];
        fk.k5 = co[2 * nf + ix];
        fk.k7 = co[3 * nf + ix];
        fk.k9 = co[4 * nf + ix];
        return quickest_face_k(U1, U2, U3, U4, C, D1, D2, D3, D4, D5, cr, fk);
    }
    return quickest_face(U1, U2, U3, U4, C, D1, D2, D3, D4, D5, cr);
}

// Limited face value (QUICKEST6.cpp:357-447) from the original line E, the
// unlimited line UE and the unlimited face value f.
__device__ __forceinline__ double limit_at(const double* E, const double* UE, const double* cf,
                                           double f, int ix)
{
    const double cr = cf[ix];
    const int up = cr >= 0 ? 1 : 0;
    const int c = 5 + ix - up;
    const int s = up ? 1 : -1;
    return quickest_limit(f, cr, E[c - s], E[c], E[c + s], UE[c - s], UE[c - 2 * s], UE[c - 3 * s],
                          UE[c], UE[c + s], UE[c + 2 * s], UE[c + 3 * s]);
}

// One group of nl (1 or 2) lines of length n through all of their CFL
// sub-steps.  RS: R-line (load *G, store /G *lexp +src dt).
template <bool RS, bool PRE>
__device__ void warp_lines(double* S, double* buf, const WLine L0, const WLine L1, int nl, int n,
                           int lt, int ut, int lane, const SliceIO& io, int nf)
{
    // the two line descriptors stay in registers: fields are selected, never indexed
#define LQ(q) ((q) ? L1 : L0)
    const int lb = line_buf(n);
    const int ix0 = (lt == VERB_BC_PERIODIC) ? 0 : 1;
    auto gidx = [&](int row, int c) { return ((size_t)row * io.R + c) * io.VK + io.off; };
    for (int q = 0; q < nl; q++) {
        double* E = buf + q * lb;
        for (int k = lane; k < n; k += 32) {
            const double v = S[LQ(q).base + k * LQ(q).stride];
            if (RS) E[5 + k] = v * (PRE ? io.gpl[LQ(q).row * io.R + k] : io.G[gidx(LQ(q).row, k)]);
            else E[5 + k] = v;
        }
    }
    __syncwarp();
    for (int q = 0; q < nl; q++) fill_ghosts(buf + q * lb, buf + q * lb, n, lt, ut, LQ(q), lane);
    __syncwarp();
    int nsmax = L0.ns;
    if (nl > 1 && L1.ns > nsmax) nsmax = L1.ns;
    const int tot = nl * n;
    for (int sub = 0; sub < nsmax; sub++) {
        // A: unlimited faces (QUICKEST6.cpp:148-256), two faces per lane and
        // iteration so that their FP64 chains interleave
        for (int f0 = lane; f0 < tot; f0 += 64) {
            const int f1 = f0 + 32;
            int qa = f0 >= n ? 1 : 0, ia = f0 - qa * n;
            int qb = f1 >= n ? 1 : 0, ib = f1 - qb * n;
            const bool va = ia >= ix0 && sub < LQ(qa).ns;
            const bool vb = f1 < tot && ib >= ix0 && sub < LQ(qb).ns;
            if (!va && !vb) continue;
            if (!vb) { qb = qa; ib = ia; }
            if (!va) { qa = qb; ia = ib; }
            const double fa = face_at<PRE>(buf + qa * lb, LQ(qa).cf, LQ(qa).co, nf, ia);
            const double fbv = face_at<PRE>(buf + qb * lb, LQ(qb).cf, LQ(qb).co, nf, ib);
            if (va) buf[qa * lb + 2 * (n + 10) + ia] = fa;
            if (vb) buf[qb * lb + 2 * (n + 10) + ib] = fbv;
        }
        __syncwarp();
        // B: unlimited cells + boundary rewrite (:243-272) into UE
        for (int f = lane; f < tot; f += 32) {
            const int q = f >= n ? 1 : 0;
            const int c = f - q * n;
            if (sub >= LQ(q).ns) continue;
            const double* E = buf + q * lb;
            double* UE = buf + q * lb + (n + 10);
            const double* F = buf + q * lb + 2 * (n + 10);
            UE[5 + c] = wcell_final(E, F, LQ(q), n, lt, ut, c);
        }
        __syncwarp();
        // UE ghosts: low ones from the pre-step PSD (= E's), high ones from UE
        for (int q = 0; q < nl; q++) {
            if (sub >= LQ(q).ns) continue;
            double* E = buf + q * lb;
            double* UE = E + (n + 10);
            if (lane < 5) UE[lane] = E[lane];
            fill_ghosts(UE, E, n, lt, ut, LQ(q), lane < 5 ? 32 : lane);
        }
        __syncwarp();
        // C: limited faces, in place (:332-455), two per lane and iteration
        for (int f0 = lane; f0 < tot; f0 += 64) {
            const int f1 = f0 + 32;
            int qa = f0 >= n ? 1 : 0, ia = f0 - qa * n;
            int qb = f1 >= n ? 1 : 0, ib = f1 - qb * n;
            const bool va = ia >= ix0 && sub < LQ(qa).ns;
            const bool vb = f1 < tot && ib >= ix0 && sub < LQ(qb).ns;
            if (!va && !vb) continue;
            if (!vb) { qb = qa; ib = ia; }
            if (!va) { qa = qb; ia = ib; }
            const double* Ea = buf + qa * lb;
            const double* Eb = buf + qb * lb;
            double* Fa = buf + qa * lb + 2 * (n + 10);
            double* Fb = buf + qb * lb + 2 * (n + 10);
            const double la = limit_at(Ea, Ea + (n + 10), LQ(qa).cf, Fa[ia], ia);
            const double lbv = limit_at(Eb, Eb + (n + 10), LQ(qb).cf, Fb[ib], ib);
            if (va) Fa[ia] = la;
            if (vb) Fb[ib] = lbv;
        }
        __syncwarp();
        // D: final cells + rewrite (:448-477)
        for (int f = lane; f < tot; f += 32) {
            const int q = f >= n ? 1 : 0;
            const int c = f - q * n;
            if (sub >= LQ(q).ns) continue;
            const double* E = buf + q * lb;
            double* UE = buf + q * lb + (n + 10);
            const double* F = buf + q * lb + 2 * (n + 10);
            const double v = wcell_final(E, F, LQ(q), n, lt, ut, c);
            if (sub == LQ(q).ns - 1) {
                if (RS && PRE) {
                    const int pi = LQ(q).row * io.R + c;
                    double x = v / io.gpl[pi];
                    x = x * io.lexp[pi];
                    if (c >= 1 && c < io.R - 1) x = x + io.spl[pi];
                    S[LQ(q).base + c * LQ(q).stride] = x;
                } else if (RS) {
                    const size_t gi = gidx(LQ(q).row, c);
                    double x = v / io.G[gi];
                    x = x * io.lexp[LQ(q).row * io.R + c];
                    if (c >= 1 && c < io.R - 1) x = x + io.src[gi] * io.dtc;
                    S[LQ(q).base + c * LQ(q).stride] = x;
                } else {
                    S[LQ(q).base + c * LQ(q).stride] = v;
                }
            } else {
                UE[5 + c] = v;
            }
        }
        __syncwarp();
        if (sub + 1 < nsmax) {
            // lines that continue: the new values become E (ghosts rebuilt from them)
            for (int q = 0; q < nl; q++) {
                if (sub + 1 >= LQ(q).ns) continue;
                double* E = buf + q * lb;
                const double* UE = E + (n + 10);
                for (int k = lane; k < n; k += 32) E[5 + k] = UE[5 + k];
            }
            __syncwarp();
            for (int q = 0; q < nl; q++)
                if (sub + 1 < LQ(q).ns) fill_ghosts(buf + q * lb, buf + q * lb, n, lt, ut, LQ(q), lane);
            __syncwarp();
        }
    }
#undef LQ
}

template <bool PRE>
__global__ void __launch_bounds__(CONV_THREADS) convection_kernel(ConvArgs a)
{
    extern __shared__ double sm[];
    const Dims d = a.d;
    const int P = d.P, R = d.R, V = d.V, K = d.K;
    const int PR = P * R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* S = sm;                                   // [P][R]
    double* CFP = S + PR;                             // P-line face Courants [R-1][P]
    double* CFR = CFP + (size_t)(R > 1 ? R - 1 : 1) * P;  // R-line face Courants [P][R]
    double* lbP = CFR + PR;                           // per P-line [R]: lbc, ubc, dxl, dxu
    double* ubP = lbP + R;
    double* dxP = ubP + R;
    double* dxPu = dxP + R;
    double* lbR = dxPu + R;                           // per R-line [P]
    double* ubR = lbR + P;
    double* dxR = ubR + P;
    double* dxRu = dxR + P;
    double* red = dxRu + P;                           // [32]
    int* nsP = (int*)(red + 32);                      // [R]
    int* nsR = nsP + R;                               // [P]
    const int wbuf = 2 * line_buf(P) > line_buf(R) ? 2 * line_buf(P) : line_buf(R);
    double* wb = (double*)(((uintptr_t)(nsR + P) + 15) & ~(uintptr_t)15) + (size_t)warp * wbuf;
    __shared__ int s_ticket;

    const size_t VK = (size_t)V * K;
    double* lexp = a.scratch + (size_t)blockIdx.x * PR;
    // face coefficient table: P-line faces [R-1][P] then R-line faces [P][R], 5 planes
    const int nfP = (R > 1 ? R - 1 : 1) * P;
    const int nf = nfP + PR;
    double* coef = PRE ? a.coef + (size_t)blockIdx.x * (5 * (size_t)nf + 2 * (size_t)PR) : nullptr;
    double* gpl = PRE ? coef + 5 * (size_t)nf : nullptr;     // G of the slice
    double* spl = PRE ? gpl + PR : nullptr;                  // Sources*dt of the slice
    const int nslices = V * K;
    const int nw = blockDim.x >> 5;

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
            lexp[i] = exp(a.loss[g(iP, iR)] * dtc);
            if (PRE) {
                gpl[i] = a.G[g(iP, iR)];
                spl[i] = a.S[g(iP, iR)] * dtc;
            }
        }

        // per-line CFL sub-cycles and face Courant numbers (QUICKEST6.cpp:37-52,
        // 150-160), one warp per line
        if (P >= 3) {
            for (int iR = warp; iR < R - 1; iR += nw) {
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
                for (int ix = lane; ix < P; ix += 32) {
                    const int i0 = ix == 0 ? P - 2 : ix - 1;
                    const double c0 = a.VP[g(i0, iR)] / dx * dtl;
                    const double c1 = a.VP[g(ix, iR)] / dx * dtl;
                    const double cr = (c0 + c1) / 2;
                    CFP[iR * P + ix] = cr;
                    if (PRE) {
                        const FaceCoef fk = face_coef(cr);
                        double* co = coef + iR * P + ix;
                        co[0] = fk.k3;
                        co[nf] = fk.c6;
                        co[2 * nf] = fk.k5;
                        co[3 * nf] = fk.k7;
                        co[4 * nf] = fk.k9;
                    }
                }
                if (lane == 0) {
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
            for (int iP = warp; iP < P; iP += nw) {
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
                for (int ix = lane; ix < R; ix += 32) {
                    const int i0 = ix == 0 ? R - 2 : ix - 1;
                    const double c0 = a.VR[g(iP, i0)] / dx * dtl;
                    const double c1 = a.VR[g(iP, ix)] / dx * dtl;
                    const double cr = (c0 + c1) / 2;
                    CFR[iP * R + ix] = cr;
                    if (PRE) {
                        const FaceCoef fk = face_coef(cr);
                        double* co = coef + nfP + iP * R + ix;
                        co[0] = fk.k3;
                        co[nf] = fk.c6;
                        co[2 * nf] = fk.k5;
                        co[3 * nf] = fk.k7;
                        co[4 * nf] = fk.k9;
                    }
                }
                if (lane == 0) {
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

        SliceIO io;
        io.G = a.G;
        io.src = a.S;
        io.lexp = lexp;
        io.VK = VK;
        io.off = off;
        io.R = R;
        io.dtc = dtc;
        io.gpl = gpl;
        io.spl = spl;
        const int npairs = (R - 1 + 1) / 2;
        for (int it = 0; it < num_steps; it++) {
            if (P >= 3) {
                // P-lines iR = 0 .. R-2 in pairs (the last R row is not swept, :104)
                for (int gp = warp; gp < npairs; gp += nw) {
                    WLine L[2];
                    const int nl = (2 * gp + 1 < R - 1) ? 2 : 1;
                    for (int q = 0; q < nl; q++) {
                        const int iR = 2 * gp + q;
                        L[q].base = iR;
                        L[q].stride = R;
                        L[q].cf = CFP + iR * P;
                        L[q].co = PRE ? coef + iR * P : nullptr;
                        L[q].lbc = lbP[iR];
                        L[q].ubc = ubP[iR];
                        L[q].dxl = dxP[iR];
                        L[q].dxu = dxPu[iR];
                        L[q].ns = nsP[iR];
                        L[q].row = 0;
                    }
                    warp_lines<false, PRE>(S, wb, L[0], L[1], nl, P, a.Pl_t, a.Pu_t, lane, io, nf);
                }
                __syncthreads();
            }
            if (R >= 3) {
                for (int iP = warp; iP < P; iP += nw) {
                    WLine L[2];
                    L[0].base = iP * R;
                    L[0].stride = 1;
                    L[0].cf = CFR + iP * R;
                    L[0].co = PRE ? coef + nfP + iP * R : nullptr;
                    L[0].lbc = lbR[iP];
                    L[0].ubc = ubR[iP];
                    L[0].dxl = dxR[iP];
                    L[0].dxu = dxRu[iP];
                    L[0].ns = nsR[iP];
                    L[0].row = iP;
                    warp_lines<true, PRE>(S, wb, L[0], L[0], 1, R, a.Rl_t, a.Ru_t, lane, io, nf);
                }
                __syncthreads();
            } else {
                // no R-sweep: exp(loss dt) and sources only (:147-165)
                for (int i = threadIdx.x; i < PR; i += blockDim.x) {
                    const int iP = i / R, iR = i - iP * R;
                    double x = S[i] * lexp[i];
                    if (iR >= 1 && iR < R - 1) x = x + a.S[g(iP, iR)] * dtc;
                    S[i] = x;
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

size_t conv_smem_bytes(int P, int R)
{
    const size_t PR = (size_t)P * R;
    const size_t lbP = 3 * (size_t)P + 20, lbR = 3 * (size_t)R + 20;
    const size_t wbuf = 2 * lbP > lbR ? 2 * lbP : lbR;
    return (PR + (size_t)(R > 1 ? R - 1 : 1) * P + PR + 4 * (size_t)R + 4 * (size_t)P + 32) *
               sizeof(double) +
           (size_t)(R + P) * sizeof(int) + 16 + (size_t)(CONV_THREADS / 32) * wbuf * sizeof(double);
}

size_t conv_coef_doubles(int P, int R)
{
    return 5 * ((size_t)(R > 1 ? R - 1 : 1) * P + (size_t)P * R) + 2 * (size_t)P * R;
}

int conv_ctas(int P, int R)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = conv_smem_bytes(P, R);
    cudaFuncSetAttribute(convection_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, convection_kernel<true>, CONV_THREADS, smem);
    if (per < 1) per = 1;
    return sms * per;
}

void launch_convection(const ConvArgs& a, int nctas, cudaStream_t s)
{
    const size_t smem = conv_smem_bytes(a.d.P, a.d.R);
    if (a.coef) {
        cudaFuncSetAttribute(convection_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        convection_kernel<true><<<nctas, CONV_THREADS, smem, s>>>(a);
    } else {
        cudaFuncSetAttribute(convection_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        convection_kernel<false><<<nctas, CONV_THREADS, smem, s>>>(a);
    }
}

void launch_convection_line(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                            int ubc_t, const double* ux, double dt, int* status, cudaStream_t s)
{
    const size_t smem = (size_t)(4 * n + 32) * sizeof(double);
    cudaFuncSetAttribute(convection_line_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    convection_line_kernel<<<1, CONV_THREADS, smem, s>>>(psd, x, n, lbc, ubc, lbc_t, ubc_t, ux, dt,
                                                        status);
}

}  // namespace verb
