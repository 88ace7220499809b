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

__global__ void __launch_bounds__(CONV_THREADS) convection_kernel(ConvArgs a)
{
    extern __shared__ double sm[];
    const Dims d = a.d;
    const int P = d.P, R = d.R, V = d.V, K = d.K;
    const int PR = P * R;
    double* S = sm;
    double* U = sm + PR;
    double* F = sm + 2 * PR;
    double* CP = sm + 3 * PR;
    double* CR = sm + 4 * PR;
    int* nsP = (int*)(sm + 5 * PR);       // inner steps of P-lines [R]
    int* nsR = nsP + R;                   // inner steps of R-lines [P]
    // per-line boundary values and spacings: P-lines [R], R-lines [P]
    double* lbP = (double*)(((uintptr_t)(nsR + P) + 15) & ~(uintptr_t)15);
    double* ubP = lbP + R;
    double* dxP = ubP + R;
    double* dxPu = dxP + R;
    double* lbR = dxPu + R;
    double* ubR = lbR + P;
    double* dxR = ubR + P;
    double* dxRu = dxR + P;
    double* red = dxRu + P;               // [32]
    __shared__ int s_ticket;
    __shared__ int s_maxP, s_maxR;

    const size_t VK = (size_t)V * K;
    double* lexp = a.scratch + (size_t)blockIdx.x * PR;
    const int nslices = V * K;

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

        // slice load and slice-level maxima (src/Convection_2D.cpp:57-86)
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
        if (threadIdx.x == 0) {
            a.substeps[off] = (int)num_steps;
            s_maxP = 1;
            s_maxR = 1;
        }
        for (int i = threadIdx.x; i < PR; i += blockDim.x) {
            const int iP = i / R, iR = i - iP * R;
            lexp[i] = exp(a.loss[g(iP, iR)] * dtc);
        }
        __syncthreads();

        // per-line CFL sub-cycle and Courant numbers (QUICKEST6.cpp:37-52), one warp per line
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
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
                for (int iP = lane; iP < P; iP += 32) CP[iP * R + iR] = a.VP[g(iP, iR)] / dx * dtl;
                if (lane == 0) {
                    nsP[iR] = ns;
                    dxP[iR] = dx;
                    dxPu[iR] = a.Pg[g(P - 1, iR)] - a.Pg[g(P - 2, iR)];
                    const size_t bo = ((size_t)iR * V + iV) * K + iK;
                    lbP[iR] = a.Pl[bo];
                    ubP[iR] = a.Pu[bo];
                    if (ns > 1) atomicMax(&s_maxP, ns);
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
                for (int iR = lane; iR < R; iR += 32) CR[iP * R + iR] = a.VR[g(iP, iR)] / dx * dtl;
                if (lane == 0) {
                    nsR[iP] = ns;
                    dxR[iP] = dx;
                    dxRu[iP] = a.Rg[g(iP, R - 1)] - a.Rg[g(iP, R - 2)];
                    const size_t bo = ((size_t)iP * V + iV) * K + iK;
                    lbR[iP] = a.Rl[bo] * a.G[g(iP, 0)];
                    ubR[iP] = a.Ru[bo] * a.G[g(iP, R - 1)];
                    if (ns > 1) atomicMax(&s_maxR, ns);
                }
            }
        }
        __syncthreads();
        const int maxP = s_maxP, maxR = s_maxR;

        const Sweep wP{P, a.Pl_t, a.Pu_t};
        const Sweep wR{R, a.Rl_t, a.Ru_t};
        for (int it = 0; it < num_steps; it++) {
            if (P >= 3) {
                // P-lines iR = 0 .. R-2 (the last R row is not swept, :104)
                for (int sub = 0; sub < maxP; sub++) {
                    auto line = [&](int l) {
                        Line L;
                        L.base = l;
                        L.stride = R;
                        L.lbc = lbP[l];
                        L.ubc = ubP[l];
                        L.dxl = dxP[l];
                        L.dxu = dxPu[l];
                        return L;
                    };
                    auto active = [&](int l) { return sub < nsP[l]; };
                    quickest_pass(S, U, F, CP, R - 1, wP, false, line, active);
                    double* tmp = S;
                    S = U;
                    U = tmp;
                }
                // the untouched last R row lives in the old buffer: carry it over
                if (maxP & 1) {
                    for (int iP = threadIdx.x; iP < P; iP += blockDim.x)
                        S[iP * R + (R - 1)] = U[iP * R + (R - 1)];
                    __syncthreads();
                }
            }
            if (R >= 3) {
                // PSD * G, then R-lines with BC*G (:122-145)
                for (int i = threadIdx.x; i < PR; i += blockDim.x) {
                    const int iP = i / R, iR = i - iP * R;
                    S[i] = S[i] * a.G[g(iP, iR)];
                }
                __syncthreads();
                for (int sub = 0; sub < maxR; sub++) {
                    auto line = [&](int l) {
                        Line L;
                        L.base = l * R;
                        L.stride = 1;
                        L.lbc = lbR[l];
                        L.ubc = ubR[l];
                        L.dxl = dxR[l];
                        L.dxu = dxRu[l];
                        return L;
                    };
                    auto active = [&](int l) { return sub < nsR[l]; };
                    quickest_pass(S, U, F, CR, P, wR, true, line, active);
                    double* tmp = S;
                    S = U;
                    U = tmp;
                }
            }
            // /G, exp(loss dt), sources on interior R (:141-165)
            for (int i = threadIdx.x; i < PR; i += blockDim.x) {
                const int iP = i / R, iR = i - iP * R;
                const size_t gi = g(iP, iR);
                double x = S[i];
                if (R >= 3) x = x / a.G[gi];
                x = x * lexp[i];
                if (iR >= 1 && iR < R - 1) x = x + a.S[gi] * dtc;
                S[i] = x;
            }
            __syncthreads();
        }
        for (int i = threadIdx.x; i < PR; i += blockDim.x) {
            const int iP = i / R, iR = i - iP * R;
            a.psd[g(iP, iR)] = S[i];
        }
        // the S/U roles may have swapped an odd number of times; the next
        // slice simply starts from the canonical order again
        S = sm;
        U = sm + PR;
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
    return 5 * PR * sizeof(double) + (size_t)(P + R) * sizeof(int) + 16 +
           (size_t)(4 * R + 4 * P) * sizeof(double) + 32 * sizeof(double);
}

int conv_ctas(int P, int R)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = conv_smem_bytes(P, R);
    cudaFuncSetAttribute(convection_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, convection_kernel, CONV_THREADS, smem);
    if (per < 1) per = 1;
    return sms * per;
}

void launch_convection(const ConvArgs& a, int nctas, cudaStream_t s)
{
    const size_t smem = conv_smem_bytes(a.d.P, a.d.R);
    cudaFuncSetAttribute(convection_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    convection_kernel<<<nctas, CONV_THREADS, smem, s>>>(a);
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
