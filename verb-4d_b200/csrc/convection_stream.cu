// Convection in (MLT, L) on every (V,K) slice with one thread per line:
// Convection_2D (src/Convection_2D.cpp:36-169) over the streaming
// ULTIMATE-QUICKEST pass of conv_stream.cuh (QUICKEST6.cpp:22-482).
//
// A persistent CTA of CS_THREADS threads owns one [P][R] slice at a time and
// keeps it in shared memory for all of its CFL sub-steps, taking slices
// highest energy first from a ticket counter like the other convection
// kernels.  Per sub-step:
//   * MLT sweep: thread t streams P-line iR = t (R-1 lines); its final cells
//     are stored already multiplied by G, which is the reference's PSD*G pass
//     before the L sweep (:122-126); the last L row, which the MLT sweep does
//     not touch (:104), is multiplied by the threads once their lines are done;
//   * L sweep: thread t streams half of R-line iP (two segments per line, so
//     2P threads work; each saves the 9 cells of the other half it reads
//     before the segments start writing), and stores the final cells as
//     v * exp(Loss dt)/G + S dt (the epilogue of :126-165; S dt for interior
//     L only).  Lines with their own CFL sub-cycles, and periodic L, run
//     whole, one thread per line.
// Both sweeps go through a single call of the pass: the kernel then holds one
// copy of its (unrolled) code, which keeps it in the instruction cache.
// Slice tables (face Courant numbers, G, exp(Loss dt)/G, S dt, boundary data)
// are formed once per slice into a per-CTA region that stays in L2, laid out
// line-fastest so that a sweep's loads are coalesced across its threads.
// The shared plane has an odd row stride, so the L sweep's column-strided
// accesses are free of bank conflicts.
//
// Compiled with multiply-add contraction: a step is within a few units in
// the last place of the reference's (not bit-identical), like the contracted
// form of convection.cu.
#include "conv_stream.cuh"
#include "verb_internal.cuh"

namespace verb {
namespace {

using cstream::LineDesc;
using cstream::StepRange;

constexpr int CS_THREADS = 128;
constexpr double CS_MAX_SUBSTEPS = 1.0e6;

__host__ __device__ inline int cs_rs(int R) { return R | 1; }

__host__ __device__ inline size_t cs_scratch(int P, int R)
{
    return (size_t)P * (R - 1) + 4 * (size_t)P * R + 4 * (size_t)(R - 1) + 4 * (size_t)P;
}

__host__ __device__ inline size_t cs_smem(int P, int R)
{
    return ((size_t)P * cs_rs(R) + (size_t)cstream::NSLOT * CS_THREADS + 32) * sizeof(double) +
           (size_t)(R + P) * sizeof(int);
}

__device__ __forceinline__ double cs_block_max(double v, double* red)
{
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, v, o);
        v = (v < t) ? t : v;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double m = red[0];
    for (int i = 1; i < CS_THREADS / 32; i++) m = (m < red[i]) ? red[i] : m;
    __syncthreads();
    return m;
}

// CS_U: steps per unrolled block; CS_MINB: resident CTAs per SM the
// registers are capped for
template <int CS_U, int CS_MINB>
__global__ void __launch_bounds__(CS_THREADS, CS_MINB) convection_stream_kernel(ConvArgs a)
{
    extern __shared__ double sm[];
    const Dims d = a.d;
    const int P = d.P, R = d.R, V = d.V, K = d.K;
    const int PR = P * R, Rs = cs_rs(R);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int NW = CS_THREADS / 32;
    double* S = sm;                                    // [P][Rs]
    double* slots = S + (size_t)P * Rs;                // [NSLOT][CS_THREADS]
    double* red = slots + cstream::NSLOT * CS_THREADS;  // [32]
    int* nsP = (int*)(red + 32);                       // [R] sub-cycles of P-line iR
    int* nsR = nsP + R;                                // [P] sub-cycles of R-line iP
    __shared__ int s_ticket;

    const size_t VK = (size_t)V * K;
    double* crP = a.scratch + (size_t)blockIdx.x * cs_scratch(P, R);  // [P faces][R-1 lines]
    double* crR = crP + (size_t)P * (R - 1);                          // [R faces][P lines]
    double* Gp = crR + (size_t)R * P;                                 // [P][R]
    double* hqT = Gp + (size_t)PR;                                    // [R][P] exp(Loss dt)/G
    double* spT = hqT + (size_t)PR;                                   // [R][P] S dt
    double* lnP = spT + (size_t)PR;                                   // [4][R-1]
    double* lnR = lnP + 4 * (size_t)(R - 1);                          // [4][P]
    const int nslices = V * K;
    const bool pper = a.Pl_t == VERB_BC_PERIODIC, rper = a.Rl_t == VERB_BC_PERIODIC;
    // L sweep in two segments of m0 and R - m0 cells
    const int m0 = (R + 1) / 2;
    const bool seg_shape = !rper && 2 * P <= CS_THREADS && R >= 32;
    const StepRange rgP = cstream::step_range(P, P, true, pper);
    const StepRange rgRw = cstream::step_range(R, R, true, rper);
    const StepRange rgRs = cstream::step_range(R - m0, m0, false, false);

    for (;;) {
        if (tid == 0) s_ticket = atomicAdd(a.ticket, 1);
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
        for (int i = tid; i < PR; i += CS_THREADS) {
            const int iP = i / R, iR = i - iP * R;
            const size_t gi = g(iP, iR);
            S[iP * Rs + iR] = a.psd[gi];
            const double vp = fabs(a.VP[gi]), vr = fabs(a.VR[gi]);
            vpm = (vpm < vp) ? vp : vpm;
            vrm = (vrm < vr) ? vr : vrm;
        }
        vpm = cs_block_max(vpm, red);
        vrm = cs_block_max(vrm, red);
        double nsp, nsr;
        {
            const double dP = a.Pg[g(1, 0)] - a.Pg[g(0, 0)];
            const double x = (double)a.dt * vpm / dP / 0.25;
            nsp = x <= 1 ? 1 : ceil(x);
        }
        {
            const double dR = a.Rg[g(0, 1)] - a.Rg[g(0, 0)];
            const double x = (double)a.dt * vrm / dR / 0.25;
            nsr = x <= 1 ? 1 : ceil(x);
        }
        const double num_steps = (nsp < nsr) ? nsr : nsp;
        if (!(num_steps <= CS_MAX_SUBSTEPS)) {  // also catches inf / NaN
            if (tid == 0) {
                a.substeps[off] = -1;
                set_error(a.status, VERB_ERR_CFL);
            }
            __syncthreads();
            continue;
        }
        const double dtc = a.dt / num_steps;
        if (tid == 0) a.substeps[off] = (int)num_steps;
        for (int i = tid; i < PR; i += CS_THREADS) {
            const int iP = i / R, iR = i - iP * R;
            const size_t gi = g(iP, iR);
            const double G = a.G[gi];
            Gp[i] = G;
            hqT[(size_t)iR * P + iP] = exp(a.loss[gi] * dtc) / G;
            spT[(size_t)iR * P + iP] = a.S[gi] * dtc;
        }
        // per-line CFL sub-cycles and face Courant numbers (QUICKEST6.cpp:37-52,
        // 150-160), one warp per line
        for (int iR = warp; iR < R - 1; iR += NW) {
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
            if (!(sd <= CS_MAX_SUBSTEPS)) set_error(a.status, VERB_ERR_CFL);
            else if (sd > 1) ns = (int)ceil(sd);
            const double dtl = dtc / ns;
            if (fabs(m / dx * dtl) > 1) set_error(a.status, VERB_ERR_CFL);
            for (int ix = lane; ix < P; ix += 32) {
                const int i0 = ix == 0 ? P - 2 : ix - 1;
                const double c0 = a.VP[g(i0, iR)] / dx * dtl;
                const double c1 = a.VP[g(ix, iR)] / dx * dtl;
                crP[(size_t)ix * (R - 1) + iR] = (c0 + c1) / 2;
            }
            if (lane == 0) {
                nsP[iR] = ns;
                const size_t bo = ((size_t)iR * V + iV) * K + iK;
                lnP[iR] = a.Pl[bo];
                lnP[(R - 1) + iR] = a.Pu[bo];
                lnP[2 * (R - 1) + iR] = dx;
                lnP[3 * (R - 1) + iR] = a.Pg[g(P - 1, iR)] - a.Pg[g(P - 2, iR)];
            }
        }
        for (int iP = warp; iP < P; iP += NW) {
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
            if (!(sd <= CS_MAX_SUBSTEPS)) set_error(a.status, VERB_ERR_CFL);
            else if (sd > 1) ns = (int)ceil(sd);
            const double dtl = dtc / ns;
            if (fabs(m / dx * dtl) > 1) set_error(a.status, VERB_ERR_CFL);
            for (int ix = lane; ix < R; ix += 32) {
                const int i0 = ix == 0 ? R - 2 : ix - 1;
                const double c0 = a.VR[g(iP, i0)] / dx * dtl;
                const double c1 = a.VR[g(iP, ix)] / dx * dtl;
                crR[(size_t)ix * P + iP] = (c0 + c1) / 2;
            }
            if (lane == 0) {
                nsR[iP] = ns;
                const size_t bo = ((size_t)iP * V + iV) * K + iK;
                lnR[iP] = a.Rl[bo] * a.G[g(iP, 0)];
                lnR[P + iP] = a.Ru[bo] * a.G[g(iP, R - 1)];
                lnR[2 * P + iP] = dx;
                lnR[3 * P + iP] = a.Rg[g(iP, R - 1)] - a.Rg[g(iP, R - 2)];
            }
        }
        __syncthreads();
        // the L sweep runs in segments when no L line sub-cycles on its own
        const bool seg = seg_shape && __syncthreads_and(tid >= P || nsR[tid] == 1);

        // thread li's line of a sweep: P-line iR = li (stored times G), or
        // R-line iP (in segments: iP = li mod P, segment li / P), stored as
        // v exp(Loss dt)/G + S dt
        auto line_desc = [&](bool pr, bool sg, int li) {
            LineDesc D;
            D.sl = slots + tid;
            D.sls = CS_THREADS;
            if (pr) {
                D.pl = S + li;
                D.st = Rs;
                D.a = 0;
                D.own = P;
                D.n = P;
                D.lt = a.Pl_t;
                D.ut = a.Pu_t;
                D.lbc = lnP[li];
                D.ubc = lnP[(R - 1) + li];
                D.dxl = lnP[2 * (R - 1) + li];
                D.dxu = lnP[3 * (R - 1) + li];
                D.cr = crP + li;
                D.crs = R - 1;
                D.e1 = Gp + li;
                D.e2 = nullptr;
                D.es = R;
            } else {
                const int iP = li < P ? li : li - P;
                const bool hi = sg && li >= P;
                D.pl = S + (size_t)iP * Rs;
                D.st = 1;
                D.a = hi ? m0 : 0;
                D.own = sg ? (hi ? R - m0 : m0) : R;
                D.n = R;
                D.lt = a.Rl_t;
                D.ut = a.Ru_t;
                D.lbc = lnR[iP];
                D.ubc = lnR[P + iP];
                D.dxl = lnR[2 * P + iP];
                D.dxu = lnR[3 * P + iP];
                D.cr = crR + iP;
                D.crs = P;
                D.e1 = hqT + iP;
                D.e2 = spT + iP;
                D.es = P;
            }
            return D;
        };
        for (int it = 0; it < num_steps; it++) {
            // the MLT sweep (ph 0) and the L sweep (ph 1) go through one call
            // of the pass, so the kernel holds one copy of its code
            for (int ph = 0; ph < 2; ph++) {
                const bool pr = ph == 0;
                const bool sg = !pr && seg;
                const int nl = pr ? R - 1 : (sg ? 2 * P : P);
                if (sg) {
                    // each segment saves the cells of the other half it reads
                    // before either half starts writing
                    if (tid < nl) cstream::fill_slots(line_desc(false, true, tid));
                    __syncthreads();
                }
                for (int li = tid; li < nl; li += CS_THREADS) {
                    const LineDesc D = line_desc(pr, sg, li);
                    const int ns = pr ? nsP[li] : (sg ? 1 : nsR[li]);
                    const StepRange rg = pr ? rgP : (sg ? rgRs : rgRw);
                    // the line's own CFL sub-cycles (QUICKEST6.cpp:37-52), the
                    // epilogue on the last one only
                    for (int k = 0; k < ns; k++) {
                        if (!sg) cstream::fill_slots(D);
                        cstream::stream_pass<CS_U>(D, rg, k == ns - 1 ? (pr ? 1 : 2) : 0);
                    }
                }
                if (pr) {
                    // the last L row, which the MLT sweep does not touch (:104)
                    for (int iP = tid - (R - 1); iP < P; iP += CS_THREADS)
                        if (iP >= 0) S[iP * Rs + R - 1] = S[iP * Rs + R - 1] * Gp[(size_t)iP * R + R - 1];
                }
                __syncthreads();
            }
        }
        for (int i = tid; i < PR; i += CS_THREADS) {
            const int iP = i / R, iR = i - iP * R;
            a.psd[g(iP, iR)] = S[iP * Rs + iR];
        }
        __syncthreads();
    }
}

// Launch shape: two steps per unrolled block and the registers capped for
// three resident CTAs per SM (no spills).  Measured at
// 48x101x101x91: one step per block 175.5 ms, two 172.2 ms, three 215 ms,
// four 270 ms per convection step (wider blocks need more live registers
// and larger code); four CTAs per SM spill at 128 registers.
constexpr int CS_U = 2;
constexpr int CS_MINB = 3;

}  // namespace

// The kernel needs both sweeps (P, R >= 11) and a slice that fits the shared
// memory; other shapes take the contracted kernel of convection.cu.
int conv_stream_check(int P, int R)
{
    if (P < 11 || R < 11) return VERB_ERR_SIZE;
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (cs_smem(P, R) > (size_t)maxsm) return VERB_ERR_SIZE;
    return VERB_OK;
}

size_t conv_stream_scratch_doubles(int P, int R) { return cs_scratch(P, R); }

int conv_stream_ctas(int P, int R)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const auto fn = convection_stream_kernel<CS_U, CS_MINB>;
    allow_max_dynamic_smem((const void*)fn);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, CS_THREADS, cs_smem(P, R));
    if (per < 1) per = 1;
    if (per > CS_MINB) per = CS_MINB;
    return sms * per;
}

// the most CTAs a launch runs (scratch is sized for it)
int conv_stream_ctas_max(int P, int R)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    (void)P;
    (void)R;
    return sms * CS_MINB;
}

void launch_convection_stream(const ConvArgs& a, int nctas, cudaStream_t s)
{
    const auto fn = convection_stream_kernel<CS_U, CS_MINB>;
    allow_max_dynamic_smem((const void*)fn);
    fn<<<nctas, CS_THREADS, cs_smem(a.d.P, a.d.R), s>>>(a);
}

}  // namespace verb
