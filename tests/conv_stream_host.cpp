// The streaming convection algorithm of conv_stream.cuh compiled for the host:
// one [P][R] slice through the same slice tables, sweeps, segments and slots
// as convection_stream_kernel, its threads run one after another (in order or
// in reverse, which checks that the segments' halo slots make the in-place L
// sweep independent of thread order).  Test infrastructure only: built by
// tests/test_conv_stream_host.py and compared there with the oracle.
#include <cmath>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include "conv_stream.cuh"

using namespace verb::cstream;

extern "C" int host_stream_convection_2d(double* psd, const double* Pg, const double* Rg, int P,
                                         int R, const double* pl, const double* pu,
                                         const double* rl, const double* ru, int pl_t, int pu_t,
                                         int rl_t, int ru_t, const double* VP, const double* VR,
                                         const double* Sv, const double* loss, const double* Gv,
                                         double dt, int* substeps, int force_whole, int order)
{
    const int NT = 128;
    const int Rs = R | 1;
    const int PR = P * R;
    std::vector<double> S((size_t)P * Rs), slots(NSLOT * NT), crP((size_t)P * (R - 1)),
        crR((size_t)R * P), Gp(PR), hqT(PR), spT(PR), lnP(4 * (R - 1)), lnR(4 * P);
    std::vector<int> nsP(R), nsR(P);
    double vpm = 0, vrm = 0;
    for (int i = 0; i < PR; i++) {
        int iP = i / R, iR = i % R;
        S[iP * Rs + iR] = psd[i];
        vpm = std::max(vpm, std::fabs(VP[i]));
        vrm = std::max(vrm, std::fabs(VR[i]));
    }
    double nsp, nsr;
    {
        double dP = Pg[1 * R] - Pg[0];
        double x = dt * vpm / dP / 0.25;
        nsp = x <= 1 ? 1 : ceil(x);
        double dR = Rg[1] - Rg[0];
        x = dt * vrm / dR / 0.25;
        nsr = x <= 1 ? 1 : ceil(x);
    }
    double num_steps = std::max(nsp, nsr);
    double dtc = dt / num_steps;
    *substeps = (int)num_steps;
    for (int i = 0; i < PR; i++) {
        int iP = i / R, iR = i % R;
        Gp[i] = Gv[i];
        hqT[iR * P + iP] = std::exp(loss[i] * dtc) / Gv[i];
        spT[iR * P + iP] = Sv[i] * dtc;
    }
    for (int iR = 0; iR < R - 1; iR++) {
        double m = -INFINITY;
        for (int iP = 0; iP < P; iP++) m = std::max(m, std::fabs(VP[iP * R + iR]));
        double dx = Pg[1 * R + iR] - Pg[iR];
        double sd = dtc * m / dx / 1.0;
        int ns = sd > 1 ? (int)ceil(sd) : 1;
        double dtl = dtc / ns;
        for (int ix = 0; ix < P; ix++) {
            int i0 = ix == 0 ? P - 2 : ix - 1;
            double c0 = VP[i0 * R + iR] / dx * dtl, c1 = VP[ix * R + iR] / dx * dtl;
            crP[ix * (R - 1) + iR] = (c0 + c1) / 2;
        }
        nsP[iR] = ns;
        lnP[iR] = pl[iR];
        lnP[(R - 1) + iR] = pu[iR];
        lnP[2 * (R - 1) + iR] = dx;
        lnP[3 * (R - 1) + iR] = Pg[(P - 1) * R + iR] - Pg[(P - 2) * R + iR];
    }
    for (int iP = 0; iP < P; iP++) {
        double m = -INFINITY;
        for (int iR = 0; iR < R; iR++) m = std::max(m, std::fabs(VR[iP * R + iR]));
        double dx = Rg[iP * R + 1] - Rg[iP * R];
        double sd = dtc * m / dx / 1.0;
        int ns = sd > 1 ? (int)ceil(sd) : 1;
        double dtl = dtc / ns;
        for (int ix = 0; ix < R; ix++) {
            int i0 = ix == 0 ? R - 2 : ix - 1;
            double c0 = VR[iP * R + i0] / dx * dtl, c1 = VR[iP * R + ix] / dx * dtl;
            crR[ix * P + iP] = (c0 + c1) / 2;
        }
        nsR[iP] = ns;
        lnR[iP] = rl[iP] * Gv[iP * R];
        lnR[P + iP] = ru[iP] * Gv[iP * R + R - 1];
        lnR[2 * P + iP] = dx;
        lnR[3 * P + iP] = Rg[iP * R + R - 1] - Rg[iP * R + R - 2];
    }
    const bool pper = pl_t == VERB_BC_PERIODIC, rper = rl_t == VERB_BC_PERIODIC;
    const int m0 = (R + 1) / 2;
    bool seg = !rper && 2 * P <= NT && R >= 32 && !force_whole;
    for (int iP = 0; iP < P; iP++) seg = seg && nsR[iP] == 1;
    const StepRange rgP = step_range(P, P, true, pper);
    const StepRange rgRw = step_range(R, R, true, rper);
    const StepRange rgRs = step_range(R - m0, m0, false, false);
    auto run_line = [&](LineDesc& D, const StepRange& rg, int ns, int epi) {
        for (int k = 0; k < ns; k++) {
            fill_slots(D);
            stream_pass<2>(D, rg, k == ns - 1 ? epi : 0);
        }
    };
    for (int it = 0; it < num_steps; it++) {
        for (int tt = 0; tt < R - 1; tt++) {
            int iR = order ? (R - 2 - tt) : tt;
            int tid = iR % NT;
            LineDesc D;
            D.pl = S.data() + iR;
            D.st = Rs;
            D.a = 0;
            D.own = P;
            D.n = P;
            D.lt = pl_t;
            D.ut = pu_t;
            D.lbc = lnP[iR];
            D.ubc = lnP[(R - 1) + iR];
            D.dxl = lnP[2 * (R - 1) + iR];
            D.dxu = lnP[3 * (R - 1) + iR];
            D.cr = crP.data() + iR;
            D.crs = R - 1;
            D.sl = slots.data() + tid;
            D.sls = NT;
            D.e1 = Gp.data() + iR;
            D.e2 = nullptr;
            D.es = R;
            run_line(D, rgP, nsP[iR], 1);
        }
        for (int iP = 0; iP < P; iP++) S[iP * Rs + R - 1] *= Gp[iP * R + R - 1];
        auto descR = [&](LineDesc& D, int iP, int tid, int a0, int own) {
            D.pl = S.data() + (size_t)iP * Rs;
            D.st = 1;
            D.a = a0;
            D.own = own;
            D.n = R;
            D.lt = rl_t;
            D.ut = ru_t;
            D.lbc = lnR[iP];
            D.ubc = lnR[P + iP];
            D.dxl = lnR[2 * P + iP];
            D.dxu = lnR[3 * P + iP];
            D.cr = crR.data() + iP;
            D.crs = P;
            D.sl = slots.data() + tid;
            D.sls = NT;
            D.e1 = hqT.data() + iP;
            D.e2 = spT.data() + iP;
            D.es = P;
        };
        if (seg) {
            std::vector<LineDesc> Ds(2 * P);
            for (int tid = 0; tid < 2 * P; tid++) {
                int iP = tid < P ? tid : tid - P;
                int sg = tid < P ? 0 : 1;
                descR(Ds[tid], iP, tid, sg ? m0 : 0, sg ? R - m0 : m0);
                fill_slots(Ds[tid]);
            }
            for (int tt = 0; tt < 2 * P; tt++) {
                int tid = order ? (2 * P - 1 - tt) : tt;
                stream_pass<2>(Ds[tid], rgRs, 2);
            }
        } else {
            for (int iP = 0; iP < P; iP++) {
                LineDesc D;
                descR(D, iP, iP, 0, R);
                run_line(D, rgRw, nsR[iP], 2);
            }
        }
    }
    for (int i = 0; i < PR; i++) psd[i] = S[(i / R) * Rs + i % R];
    return 0;
}

extern "C" void host_line_pass(double* psd, int n, double lbc, double ubc, int lt, int ut,
                               const double* cr, double dxl, double dxu, int a, int own, int whole)
{
    std::vector<double> slots(NSLOT);
    LineDesc D;
    D.pl = psd; D.st = 1; D.a = a; D.own = own; D.n = n; D.lt = lt; D.ut = ut;
    D.lbc = lbc; D.ubc = ubc; D.dxl = dxl; D.dxu = dxu; D.cr = cr; D.crs = 1;
    D.sl = slots.data(); D.sls = 1; D.e1 = nullptr; D.e2 = nullptr; D.es = 1;
    fill_slots(D);
    StepRange rg = step_range(own, own, whole != 0, lt == VERB_BC_PERIODIC);
    stream_pass<2>(D, rg, 0);
}
