// Radial diffusion in L: batched Thomas solves, one thread per (P,V,K) line.
//
// Compiled with -fmad=false: every operation below is the reference's
// operation in the reference's order, so results are bit-identical to
// Diffusion_1D (src/Diffusion_1D.cpp:43-184, src/MatrixSolver.cpp:353-404,
// 689-720) on the same inputs.
//
// The tridiagonal matrix depends only on L*, D_LL, G_radial, Losses_radial
// and dt, which change at most hourly; its Thomas recurrence (gam_j, bet_j and
// the sub-diagonal a_j) is therefore computed by radial_factor_kernel when
// one of them changes and cached in HBM as [R][lines] (coalesced along lines).
// radial_solve_kernel is the per-step pass: it forms RHS = B f + C, runs the
// forward sweep writing u_j into PSD in place, then the back substitution.
#include "verb_internal.cuh"

namespace verb {

namespace {

struct Row {
    double lo, d, up;
};

// One interior row of getCalculationMatrix1DDiffusion (src/Diffusion_1D.cpp:161-178):
// A_ii = 1/dt - Loss, then SecondDerivativeApproximation_1D twice
// (src/MatrixSolver.cpp:353-404) with multiplicator -0.5.
__device__ __forceinline__ Row radial_interior_row(double xm, double x0, double xp, double Dm,
                                                   double D0, double Dp, double Gm, double G0,
                                                   double Gp, double loss, double dt)
{
    Row w;
    w.lo = 0.0;
    w.up = 0.0;
    w.d = 0.0;
    w.d += 1.0 / dt;
    w.d -= loss;
    // ("x_left", "x_right"): dx1 = -1, dx2 = +1
    {
        double dh1 = x0 - xm, dh21 = x0 - xp, dh22 = xm - x0;
        double cp = -0.5 / G0 / dh1;
        w.d += +cp / dh21 * D0 * G0;
        w.up += -cp / dh21 * D0 * G0;
        w.lo += -cp / dh22 * Dm * Gm;
        w.d += +cp / dh22 * Dm * Gm;
    }
    // ("x_right", "x_left"): dx1 = +1, dx2 = -1
    {
        double dh1 = x0 - xp, dh21 = x0 - xm, dh22 = xp - x0;
        double cp = -0.5 / G0 / dh1;
        w.d += +cp / dh21 * D0 * G0;
        w.lo += -cp / dh21 * D0 * G0;
        w.up += -cp / dh22 * Dp * Gp;
        w.d += +cp / dh22 * Dp * Gp;
    }
    return w;
}

__global__ void radial_factor_kernel(RadialArgs a)
{
    const Dims d = a.d;
    const size_t nlines = (size_t)d.P * d.V * d.K;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nlines) return;
    const size_t vk_n = (size_t)d.V * d.K;
    const size_t p = q / vk_n, vk = q - p * vk_n;
    const size_t base = p * (size_t)d.R * vk_n + vk;
    const int n = d.R;
    const double sc = a.dll_scale;
    auto Dat = [&](int r) {
        double v = a.DLL[base + (size_t)r * vk_n];
        return sc != 1.0 ? v * sc : v;
    };

    // row 0: boundary (src/Diffusion_1D.cpp:115-137)
    double bet, up_prev;
    {
        double x0 = a.L[base], x1 = a.L[base + vk_n];
        double dh = x1 - x0;
        double dd, uu;
        if (a.Ll_t == VERB_BC_CONSTANT_VALUE) {
            dd = 1;
            uu = 0;
        } else if (a.Ll_t == VERB_BC_CONSTANT_DERIVATIVE) {
            dd = 1 / dh;
            uu = -1 / dh;
        } else {
            set_error(a.status, VERB_ERR_BC);
            return;
        }
        bet = dd;
        up_prev = uu;
        a.fa[q] = 0.0;
        a.fbet[q] = bet;
        a.fgam[q] = 0.0;
    }
    double xm = a.L[base], x0 = a.L[base + vk_n];
    double Dm = Dat(0), D0 = Dat(1);
    double Gm = a.G[base], G0 = a.G[base + vk_n];
    for (int r = 1; r < n; r++) {
        Row w;
        if (r == n - 1) {
            // last row: boundary (src/Diffusion_1D.cpp:138-159)
            double dh = x0 - xm;
            w.up = 0.0;
            if (a.Lu_t == VERB_BC_CONSTANT_VALUE) {
                w.d = 1;
                w.lo = 0;
            } else if (a.Lu_t == VERB_BC_CONSTANT_DERIVATIVE) {
                w.d = 1 / dh;
                w.lo = -1 / dh;
            } else {
                set_error(a.status, VERB_ERR_BC);
                return;
            }
        } else {
            size_t ip = base + (size_t)(r + 1) * vk_n;
            double xp = a.L[ip], Dp = Dat(r + 1), Gp = a.G[ip];
            w = radial_interior_row(xm, x0, xp, Dm, D0, Dp, Gm, G0, Gp,
                                    a.loss[base + (size_t)r * vk_n], a.dt);
            xm = x0;
            x0 = xp;
            Dm = D0;
            D0 = Dp;
            Gm = G0;
            G0 = Gp;
        }
        // Thomas recurrence of tridag (src/MatrixSolver.cpp:701-703)
        double gam = up_prev / bet;
        bet = w.d - w.lo * gam;
        const size_t o = (size_t)r * nlines + q;
        a.fa[o] = w.lo;
        a.fbet[o] = bet;
        a.fgam[o] = gam;
        up_prev = w.up;
    }
}

__global__ void radial_solve_kernel(RadialArgs a)
{
    const Dims d = a.d;
    const size_t nlines = (size_t)d.P * d.V * d.K;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nlines) return;
    const size_t vk_n = (size_t)d.V * d.K;
    const size_t p = q / vk_n, vk = q - p * vk_n;
    const size_t base = p * (size_t)d.R * vk_n + vk;
    const int n = d.R;
    const double bint = 0.0 + 1.0 / a.dt;  // matr_B[0][in] += 1.0 / dt
    const double rs = (double)a.radial_sources;
    double* f = a.psd + base;

    // RHS = C + B f (src/Diffusion_1D.cpp:66-76); row 0 is the lower BC row.
    double u;
    {
        double rhs = a.Ll[q];
        rhs += 0.0 * f[0];
        u = rhs / a.fbet[q];
        f[0] = u;
    }
    for (int r = 1; r < n; r++) {
        const size_t o = (size_t)r * vk_n;
        double c, b;
        if (r == n - 1) {
            c = a.Lu[q];
            b = 0.0;
        } else {
            c = 0.0;
            if (a.radial_sources) c += a.S[base + o] * rs;
            b = bint;
        }
        double rhs = c;
        rhs += b * f[o];
        const size_t fo = (size_t)r * nlines + q;
        u = (rhs - a.fa[fo] * u) / a.fbet[fo];
        f[o] = u;
    }
    for (int r = n - 1; r >= 1; r--) {
        const size_t o = (size_t)(r - 1) * vk_n;
        double um = f[o];
        um -= a.fgam[(size_t)r * nlines + q] * u;
        f[o] = um;
        u = um;
    }
}

// tridag (src/MatrixSolver.cpp:689-720) on one system, single thread; gam in
// global scratch after u (u must have 2n entries).
__global__ void tridag_kernel(const double* a, const double* b, const double* c, const double* r,
                              double* u, long n)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double* gam = u + n;
    double bet;
    u[0] = r[0] / (bet = b[0]);
    for (long j = 1; j <= n - 1; j++) {
        gam[j] = c[j - 1] / bet;
        bet = b[j] - a[j] * gam[j];
        u[j] = (r[j] - a[j] * u[j - 1]) / bet;
    }
    for (long j = n - 1; j >= 1; j--) u[j - 1] -= gam[j] * u[j];
}

}  // namespace

void launch_tridag(const double* a, const double* b, const double* c, const double* r, double* u,
                   long n, cudaStream_t s)
{
    tridag_kernel<<<1, 32, 0, s>>>(a, b, c, r, u, n);
}

void launch_radial_factor(const RadialArgs& a, cudaStream_t s)
{
    const size_t nlines = (size_t)a.d.P * a.d.V * a.d.K;
    const int tb = 128;
    radial_factor_kernel<<<(unsigned)((nlines + tb - 1) / tb), tb, 0, s>>>(a);
}

void launch_radial_solve(const RadialArgs& a, cudaStream_t s)
{
    const size_t nlines = (size_t)a.d.P * a.d.V * a.d.K;
    const int tb = 128;
    radial_solve_kernel<<<(unsigned)((nlines + tb - 1) / tb), tb, 0, s>>>(a);
}

}  // namespace verb
