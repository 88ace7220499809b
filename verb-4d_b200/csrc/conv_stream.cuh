// Streaming form of one Convection_1D_ULTIMATE_QUICKEST6 pass over a line
// (src/Convection_1D_ULTIMATE_QUICKEST6.cpp:22-482), one thread per line (or
// per segment of a line).  Shared by the device kernel (convection_stream.cu)
// and compiled for the host by the tests' algorithm check.
//
// The reference's pass is four sequential loops over the line: unlimited
// faces (:148-241), unlimited cells with the boundary rewrite (:243-272),
// limited faces (:277-447) and final cells with the rewrite (:448-477).  Every
// stage at position p only needs the previous stage within a few cells of p,
// so one loop runs all four at once with fixed lags: at step j it loads cell
// j+4, forms unlimited face j, unlimited cell j-2, the limiter's peak flag of
// cell j-6, limited face j-5 and final cell j-7.  The values in flight live in
// register windows; nothing but the final cells is written back.
//
// Two rearrangements of the reference's arithmetic (both exact in IEEE
// arithmetic, since negation and commutation are exact):
//  * the face polynomial is written for the positive Courant direction with
//    the signed Courant number in place of |c| (QUICKEST6.cpp:169-186 swap
//    the upwind and downwind points with the sign, which negates every odd
//    difference and leaves every even one as it is, so c * odd-part is the
//    same value either way; the ninth-order odd term, which has no |c|
//    factor, takes the sign explicitly);
//  * the limiter's three peak tests (:394-447) are differences of the
//    unlimited line taken from upwind to downwind; with e_k = U[k+1] - U[k]
//    each test is the same predicate M of four consecutive e's at a position
//    that depends on the direction only by one cell, so M is formed once per
//    cell and each face ORs three of them.
// The file is compiled with multiply-add contraction, and ref = ou + (oc -
// ou) / |c| uses the rounded reciprocal of |c|: results stay within a few
// units in the last place of the reference per pass.
#pragma once
#include <math.h>

#include "verb4d_b200.h"

#if defined(__CUDACC__)
#define CS_FN __host__ __device__ __forceinline__
#else
#define CS_FN inline
#endif

namespace verb {
namespace cstream {

// Values a thread saves for itself: slots 0-8 are line values it reads but
// cannot take from the plane (the periodic high ghosts E[1..9], or the halo
// of a segment, which the neighbouring segment overwrites), 9-13 the
// periodic line's unlimited cells 0-4 (the unlimited line's high ghosts) and
// 14 its final cell 0 (the periodic rewrite of cell n-1).
constexpr int NSLOT = 15;

// A thread's line (or segment) in a sweep.
struct LineDesc {
    double* pl;        // cell k of the line at pl[k * st]
    int st;
    int a, own, n;     // first cell this thread finalises, cells it finalises, line length
    int lt, ut;        // boundary types
    double lbc, ubc;   // boundary values
    double dxl, dxu;   // x[1] - x[0], x[n-1] - x[n-2]
    const double* cr;  // Courant number of face k (between cells k-1 and k) at cr[k * crs]
    int crs;
    double* sl;        // slot k at sl[k * sls]
    int sls;
    const double* e1;  // store epilogue: factor of cell k at e1[k * es]
    const double* e2;  // added term of cell k at e2[k * es] (cells 1..n-2)
    int es;
};

// Uniform description of a sweep's step range: steps jb .. je (local index),
// unlimited faces needed for steps [f0, f1], limited faces for [l0, l1],
// blocks whose steps lie in the fast range need no boundary logic.
struct StepRange {
    int jb, je;
    int f0, f1, l0, l1;
    int own_min;
};

CS_FN double rcp_rn(double x)
{
#if defined(__CUDA_ARCH__)
    return __drcp_rn(x);
#else
    return 1.0 / x;
#endif
}

// E[-ig] (QUICKEST6.cpp:89-143 for the low side); ig >= 1
CS_FN double ghost_lo(const LineDesc& L, int ig)
{
    if (L.lt == VERB_BC_PERIODIC) return L.pl[(L.n - 1 - ig) * L.st];
    if (L.lt == VERB_BC_CONSTANT_VALUE) return L.lbc;
    double g = L.pl[0] - L.lbc * L.dxl;
    for (int i = 2; i <= ig; i++) g = g - L.lbc * L.dxl;
    return g;
}

// E[n-1+ig]; ig >= 1 (periodic: the saved E[ig])
CS_FN double ghost_hi(const LineDesc& L, int ig)
{
    if (L.ut == VERB_BC_PERIODIC) return L.sl[(ig - 1) * L.sls];
    if (L.ut == VERB_BC_CONSTANT_VALUE) return L.ubc;
    double g = L.pl[(L.n - 1) * L.st] + L.ubc * L.dxu;
    for (int i = 2; i <= ig; i++) g = g + L.ubc * L.dxu;
    return g;
}

// Line value at local position j (cell a + j), -9 <= j < own + 9.
CS_FN double getE(const LineDesc& L, int j)
{
    if (j >= 0 && j < L.own) return L.pl[(L.a + j) * L.st];
    if (j < 0) {
        if (L.a > 0) return L.sl[(9 + j) * L.sls];
        return ghost_lo(L, -j);
    }
    if (L.a + L.own < L.n) return L.sl[(j - L.own) * L.sls];
    return ghost_hi(L, L.a + j - (L.n - 1));
}

CS_FN double getC(const LineDesc& L, int j)
{
    const int p = L.a + j;
    return (p >= 0 && p < L.n) ? L.cr[p * L.crs] : 0.0;
}

// Saves what the pass will read but cannot find in the plane.  For a segment
// this must happen before the neighbouring segment starts writing.
CS_FN void fill_slots(const LineDesc& L)
{
    if (L.a > 0) {
        for (int k = 0; k < 9; k++) L.sl[k * L.sls] = L.pl[(L.a - 9 + k) * L.st];
    } else if (L.a + L.own < L.n) {
        for (int k = 0; k < 9; k++) L.sl[k * L.sls] = L.pl[(L.a + L.own + k) * L.st];
    } else if (L.ut == VERB_BC_PERIODIC) {
        for (int k = 0; k < 9; k++) L.sl[k * L.sls] = L.pl[(1 + k) * L.st];
    }
}

// Unlimited face value from w[k] = E[x-5+k], signed Courant number c
// (QUICKEST6.cpp:162-241 in the positive orientation, pair sums s_k and
// differences t_k of the points k cells behind and k+1 cells ahead of face x).
CS_FN double face_df(const double* w, double c)
{
    // factors of the even and odd difference pairs, each with the 1/2 of
    // the even differences folded in: k3 (D2 + c/4 d3) = K3 ((2 D2) + c/2 d3)
    const double cs = c * c;
    const double q1 = cs - 1;
    const double p2 = q1 * (cs - 4);
    const double p3 = p2 * (cs - 9);
    const double p4 = p2 * ((cs - 9) * (cs - 16));
    const double K3 = q1 * (1.0 / 12.0);
    const double K5 = p2 * (1.0 / 240.0);
    const double K7 = p3 * (1.0 / 10080.0);
    const double K9 = p4 * (1.0 / 725760.0);
    const double s0 = w[4] + w[5], t0 = w[4] - w[5];
    const double s1 = w[3] + w[6], t1 = w[3] - w[6];
    const double s2 = w[2] + w[7], t2 = w[2] - w[7];
    const double s3 = w[1] + w[8], t3 = w[1] - w[8];
    const double s4 = w[0] + w[9], t4 = w[0] - w[9];
    const double E2 = s1 - s0;                                      // 2 D2
    const double d3 = t1 - 3 * t0;
    const double E4 = (s2 - 3 * s1) + 2 * s0;                      // 2 D4
    const double d5 = (t2 - 5 * t1) + 10 * t0;
    const double E6 = (s3 - 5 * s2) + (9 * s1 - 5 * s0);           // 2 D6
    const double d7 = (t3 - 7 * t2) + (21 * t1 - 35 * t0);
    const double E8 = (s4 - 7 * s3) + ((20 * s2 - 28 * s1) + 14 * s0);  // 2 D8
    const double d9 = (t4 - 9 * t3) + ((36 * t2 - 84 * t1) + 126 * t0);
    // the ninth-order odd term carries 1/2 instead of |c|/2k: its sign follows
    // the direction explicitly (c = -0 counts as positive, as in :169)
    const double g3 = K3 * (E2 + (c * 0.5) * d3);
    const double g5 = K5 * (E4 + (c * (1.0 / 3.0)) * d5);
    const double g7 = K7 * (E6 + (c * 0.25) * d7);
    const double g9 = K9 * (E8 + (c >= 0 ? d9 : -d9));
    return 0.5 * (s0 + c * t0) + ((g3 + g5) + (g7 + g9));
}

// Peak test of the unlimited line at four consecutive differences (a,b,c,d)
// = (e_k .. e_k+3): rising twice then falling twice with a bend at both ends.
CS_FN bool peak4(double a, double b, double c, double d)
{
    return (a > 0) & (b > 0) & (c < 0) & (d < 0) & (b < a) & (c > d);
}

// Limited face value (QUICKEST6.cpp:394-447) of face x from its unlimited
// value f, Courant number c, the pre-step cells E[x-2..x+1] and the peak
// flags m0..m3 of positions x-4..x-1.  The falling case (6) is the rising
// case (5) on the negated values (sg = -1; negation is exact), so one chain
// of max/min serves both.
CS_FN double limit_df(double f, double c, double em2, double em1, double e0, double ep1, bool m0,
                      bool m1, bool m2, bool m3)
{
    const bool pos = c >= 0;
    const double ou = pos ? em2 : ep1;
    const double oc = pos ? em1 : e0;
    const double od = pos ? e0 : em1;
    const bool peak = m1 | m2 | (pos ? m0 : m3);
    const double ca = fabs(c);
    const double DEL = od - ou;
    const double CURV = od - 2 * oc + ou;
    const bool flat = fabs(CURV) >= fabs(DEL);
    const bool rise = DEL > 0, fall = DEL < 0;
    const bool useref = !peak & !flat & (ca > 1e-31) & (rise | fall);
    const double ref = ou + (oc - ou) * rcp_rn(ca);
    const double sg = rise ? 1.0 : -1.0;
    const double a = sg * f, lo = sg * oc, h1 = sg * ref, h2 = sg * od;
    // fmax/fmin as selects: the same values unless the second operand is NaN
    // (then the select keeps it where fmax/fmin would drop it); a NaN PSD is
    // reported by the step's NaN check either way
    double t = a > lo ? a : lo;               // fmax(f, oc)
    const double hi = h1 < h2 ? h1 : h2;      // fmin(ref, od)
    t = t < hi ? t : hi;                      // fmin(., .)
    double res = useref ? sg * t : f;
    if (!peak & flat) res = oc;
    return res;
}

// Register windows of a block of U steps starting at step b (index k of
// each array holds the quantity at the position given beside it).
template <int U>
struct Win {
    double E[11 + U];  // E[b-7+k]
    double F[5 + U];   // unlimited face b-5+k
    double C[5 + U];   // Courant number of face b-5+k
    double Q[1 + U];   // C*F of face b-1+k
    double UR[3 + U];  // unlimited cell b-4+k before the boundary rewrite
    double UU[1 + U];  // unlimited cell b-3+k after it (ghosts past the ends)
    double EE[3 + U];  // e_{b-6+k} = UU[b-5+k] - UU[b-6+k]
    bool M[3 + U];     // peak flag of position b-9+k
    double RR[1 + U];  // C * limited face of face b-6+k
    double OR[2 + U];  // final cell b-8+k before the boundary rewrite
};

// Store epilogue factors of local cell c: v * f1 + f2 (epi 0: 1, 0; epi 1:
// e1, 0; epi 2: e1, e2 on interior cells).
CS_FN void load_epi(const LineDesc& L, int epi, int c, bool checked, double& f1, double& f2)
{
    f1 = 1.0;
    f2 = 0.0;
    if (epi == 0) return;
    const int p = L.a + c;
    if (checked && (c < 0 || c >= L.own)) return;
    f1 = L.e1[p * L.es];
    if (epi == 2 && (!checked || (p >= 1 && p <= L.n - 2))) f2 = L.e2[p * L.es];
}

// One step (local index j = b + s) of the pipeline.  `edge` (uniform over
// the block) selects the boundary logic: reads past the thread's range,
// rewrites at the line ends, stage ranges and store bounds.
template <int U, bool edge>
CS_FN void step(const LineDesc& L, const StepRange& R, Win<U>& w, int b, int s,
                const double (&PC)[U], const double (&P1)[U], const double (&P2)[U],
                double* blk)
{
    // blk: cell b-7 of the line (fast blocks address the plane from it)
    const int j = b + s;
    const bool lo_end = L.a == 0, hi_end = L.a + L.own == L.n;
    // front: cell j+4
    double e;
    if (edge) e = (j + 4 < L.own + 9) ? getE(L, j + 4) : 0.0;
    else e = blk[(s + 11) * L.st];
    w.E[11 + s] = e;
    w.C[5 + s] = PC[s];
    // unlimited face j
    double F = 0.0;
    if (!edge || (j >= R.f0 && j <= R.f1)) F = face_df(&w.E[s + 2], w.C[5 + s]);
    w.F[5 + s] = F;
    w.Q[1 + s] = w.C[5 + s] * F;
    // unlimited cell j-1 (raw), then cell j-2 with the rewrite (:243-272)
    w.UR[3 + s] = w.E[s + 6] - (w.Q[1 + s] - w.Q[s]);
    double u = w.UR[2 + s];
    if (edge) {
        const int uj = j - 2;
        if (lo_end && uj <= 0) {
            if (uj < 0) u = w.E[s + 5];  // the unlimited line's low ghosts are E's (:283-302)
            else if (L.lt == VERB_BC_CONSTANT_VALUE) u = L.lbc;
            else if (L.lt == VERB_BC_CONSTANT_DERIVATIVE) u = w.UR[3 + s];
            if (L.lt == VERB_BC_PERIODIC && uj == 0) L.sl[9 * L.sls] = u;
        }
        if (hi_end && uj >= L.own - 1) {
            if (uj == L.own - 1) {
                if (L.ut == VERB_BC_PERIODIC) u = L.sl[9 * L.sls];
                else if (L.ut == VERB_BC_CONSTANT_VALUE) u = L.ubc;
                else u = w.UR[1 + s];
            } else {
                if (L.ut == VERB_BC_PERIODIC)
                    u = (uj - L.own + 1 <= 4) ? L.sl[(9 + uj - L.own + 1) * L.sls] : 0.0;
                else if (L.ut == VERB_BC_CONSTANT_VALUE) u = L.ubc;
                else u = w.UU[s] + L.ubc * L.dxu;
            }
        }
        if (lo_end && L.lt == VERB_BC_PERIODIC && uj >= 1 && uj <= 4 && uj < L.own - 1)
            L.sl[(9 + uj) * L.sls] = u;
    }
    w.UU[1 + s] = u;
    w.EE[3 + s] = w.UU[1 + s] - w.UU[s];
    w.M[3 + s] = peak4(w.EE[s], w.EE[s + 1], w.EE[s + 2], w.EE[s + 3]);
    // limited face j-5
    double fl = 0.0;
    if (!edge || (j >= R.l0 && j <= R.l1))
        fl = limit_df(w.F[s], w.C[s], w.E[s], w.E[s + 1], w.E[s + 2], w.E[s + 3], w.M[s], w.M[s + 1],
                      w.M[s + 2], w.M[s + 3]);
    w.RR[1 + s] = w.C[s] * fl;
    // final cell j-6 (raw), cell j-7 with the rewrite (:448-477)
    w.OR[2 + s] = w.E[s + 1] - (w.RR[1 + s] - w.RR[s]);
    double o = w.OR[1 + s];
    const int oj = j - 7;
    bool store = true;
    if (edge) {
        if (lo_end && oj == 0) {
            if (L.lt == VERB_BC_CONSTANT_VALUE) o = L.lbc;
            else if (L.lt == VERB_BC_CONSTANT_DERIVATIVE) o = w.OR[2 + s];
            else L.sl[14 * L.sls] = o;
        }
        if (hi_end && oj == L.own - 1) {
            if (L.ut == VERB_BC_PERIODIC) o = L.sl[14 * L.sls];
            else if (L.ut == VERB_BC_CONSTANT_VALUE) o = L.ubc;
            else o = w.OR[s];
        }
        store = oj >= 0 && oj < L.own;
    }
    if (edge) {
        if (store) L.pl[(L.a + oj) * L.st] = o * P1[s] + P2[s];
    } else {
        blk[s * L.st] = o * P1[s] + P2[s];
    }
}

template <int U>
CS_FN void shift(Win<U>& w)
{
#pragma unroll
    for (int k = 0; k < 11; k++) w.E[k] = w.E[k + U];
#pragma unroll
    for (int k = 0; k < 5; k++) {
        w.F[k] = w.F[k + U];
        w.C[k] = w.C[k + U];
    }
    w.Q[0] = w.Q[U];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        w.UR[k] = w.UR[k + U];
        w.EE[k] = w.EE[k + U];
        w.M[k] = w.M[k + U];
    }
    w.UU[0] = w.UU[U];
    w.RR[0] = w.RR[U];
#pragma unroll
    for (int k = 0; k < 2; k++) w.OR[k] = w.OR[k + U];
}

// One pass over the thread's line or segment, stored as v * f1 + f2 (epi).
// Steps run from R.jb to R.je in blocks of U; a block is on the fast path (no
// boundary logic, no range checks) when all of its steps read plane cells of
// the thread's own range and write cells away from the line ends.
template <int U>
CS_FN void stream_pass(const LineDesc& L, const StepRange& R, int epi)
{
    Win<U> w;
#pragma unroll
    for (int k = 0; k < 11 + U; k++) w.E[k] = 0.0;
    for (int k = 2; k < 11; k++) w.E[k] = (R.jb - 7 + k >= -9) ? getE(L, R.jb - 7 + k) : 0.0;
#pragma unroll
    for (int k = 0; k < 5 + U; k++) {
        w.F[k] = 0.0;
        w.C[k] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < 3 + U; k++) {
        w.UR[k] = 0.0;
        w.EE[k] = 0.0;
        w.M[k] = false;
    }
#pragma unroll
    for (int k = 0; k < 1 + U; k++) {
        w.Q[k] = 0.0;
        w.UU[k] = 0.0;
        w.RR[k] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < 2 + U; k++) w.OR[k] = 0.0;
    if (R.jb == 0) {
        // a whole line starts at face 0: the unlimited line's ghosts left of
        // cell -2 (E's ghosts) enter the windows here instead of by steps
        w.UU[0] = getE(L, -3);
        w.EE[2] = w.UU[0] - getE(L, -4);
    }
    // Courant numbers are loaded one block ahead (a face needs its own at
    // the start of its step); epilogue factors at the start of the block
    // that stores with them (the stores come last in each step)
    double PC[U];
#pragma unroll
    for (int s = 0; s < U; s++) PC[s] = getC(L, R.jb + s);
    // fast block: the front (cell j+4) stays inside the thread's range,
    // cells and rewrites stay clear of the line ends, and the next block's
    // Courant numbers lie inside the range too.  The fast blocks form one
    // run in the middle of the pass; they run without any boundary logic.
    auto fast = [&](int b) { return b >= 8 && b + (2 * U > U + 4 ? 2 * U : U + 4) <= R.own_min; };
    int b = R.jb;
    // one block of the fast run: Courant numbers of the next block and the
    // epilogue factors of this one from running pointers, then the steps
    auto fast_block = [&](const double*& cp, const double*& e1p, const double*& e2p, double*& bp) {
        double NC[U], P1[U], P2[U];
#pragma unroll
        for (int s = 0; s < U; s++) {
            NC[s] = cp[s * L.crs];
            P1[s] = epi ? e1p[s * L.es] : 1.0;
            P2[s] = epi == 2 ? e2p[s * L.es] : 0.0;
        }
#pragma unroll
        for (int s = 0; s < U; s++) step<U, false>(L, R, w, b, s, PC, P1, P2, bp);
        shift<U>(w);
#pragma unroll
        for (int s = 0; s < U; s++) PC[s] = NC[s];
        b += U;
        cp += U * L.crs;
        e1p += U * L.es;
        e2p += U * L.es;
        bp += U * L.st;
    };
    while (b <= R.je) {
        if (fast(b)) {
            const double* cp = L.cr + (L.a + b + U) * L.crs;
            const double* e1p = epi ? L.e1 + (L.a + b - 7) * L.es : nullptr;
            const double* e2p = epi == 2 ? L.e2 + (L.a + b - 7) * L.es : nullptr;
            double* bp = L.pl + (L.a + b - 7) * L.st;
            do {
                fast_block(cp, e1p, e2p, bp);
            } while (b <= R.je && fast(b));
        } else {
            double NC[U], P1[U], P2[U];
#pragma unroll
            for (int s = 0; s < U; s++) {
                NC[s] = getC(L, b + U + s);
                load_epi(L, epi, b + s - 7, true, P1[s], P2[s]);
            }
#pragma unroll
            for (int s = 0; s < U; s++) step<U, true>(L, R, w, b, s, PC, P1, P2, nullptr);
            shift<U>(w);
#pragma unroll
            for (int s = 0; s < U; s++) PC[s] = NC[s];
            b += U;
        }
    }
}

// Step range of a sweep whose threads finalise own_min..own_max cells each;
// whole: every thread owns a whole line (a = 0, own = n), periodic lines
// included; otherwise the line is split into two segments.
CS_FN StepRange step_range(int own_min, int own_max, bool whole, bool periodic)
{
    StepRange r;
    // a whole line needs no unlimited face left of face 0 (its unlimited
    // cells there are ghosts); a segment starts 4 faces left of its range
    r.jb = whole ? 0 : -4;
    r.je = own_max + 6;
    if (whole) {
        r.f0 = periodic ? 0 : 1;
        r.f1 = own_max - 1;
        r.l0 = 5 + (periodic ? 0 : 1);
        r.l1 = own_max - 1 + 5;
    } else {
        r.f0 = -4;
        r.f1 = own_max + 4;
        r.l0 = 5;
        r.l1 = own_max + 5;
    }
    r.own_min = own_min;
    return r;
}

}  // namespace cstream
}  // namespace verb
