// C ABI: context lifetime, uploads, cache invalidation, phase dispatch, timing,
// and the per-slice entry points.  See include/verb4d_b200.h.
#include "ctx_internal.cuh"

namespace vctx {


size_t bc_elems(const verb_ctx* c, int b)
{
    const Dims& d = c->d;
    switch (b) {
        case VERB_BCF_PL: case VERB_BCF_PU: return (size_t)d.R * d.V * d.K;
        case VERB_BCF_RL: case VERB_BCF_RU: case VERB_BCF_LL: case VERB_BCF_LU:
            return (size_t)d.P * d.V * d.K;
        case VERB_BCF_VL: case VERB_BCF_VU: return (size_t)d.P * d.R * d.K;
        default: return (size_t)d.P * d.R * d.V;
    }
}

int alloc(void** p, size_t bytes)
{
    if (*p) return VERB_OK;
    return cuda_ok(cudaMalloc(p, bytes));
}

int ensure_field(verb_ctx* c, int fid)
{
    if (c->f[fid]) return VERB_OK;
    CK(cudaMalloc(&c->f[fid], npts(c) * sizeof(double)));
    return VERB_OK;
}

// A field the kernels read: defaults (G = 1, sources/losses = 0) when never uploaded.
int need_field(verb_ctx* c, int fid)
{
    if (c->f[fid]) return VERB_OK;
    int s = ensure_field(c, fid);
    if (s) return s;
    if (fid == VERB_F_G_LOCAL || fid == VERB_F_G_RADIAL || fid == VERB_F_G_CONV) {
        std::vector<double> ones(npts(c), 1.0);
        CK(cudaMemcpyAsync(c->f[fid], ones.data(), npts(c) * sizeof(double),
                           cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    } else if (fid == VERB_F_SOURCES || fid == VERB_F_LOSS_LOCAL || fid == VERB_F_LOSS_RADIAL ||
               fid == VERB_F_LOSS_CONV) {
        CK(cudaMemsetAsync(c->f[fid], 0, npts(c) * sizeof(double), c->stream));
    } else {
        return VERB_ERR_ARG;  // grids, coefficients and PSD must be provided
    }
    return VERB_OK;
}

int need_bc(verb_ctx* c, int b)
{
    if (c->bc[b]) return VERB_OK;
    CK(cudaMalloc(&c->bc[b], bc_elems(c, b) * sizeof(double)));
    CK(cudaMemsetAsync(c->bc[b], 0, bc_elems(c, b) * sizeof(double), c->stream));
    return VERB_OK;
}

void mark_dirty(verb_ctx* c, int fid)
{
    switch (fid) {
        case VERB_F_L: case VERB_F_DLL: case VERB_F_G_RADIAL: case VERB_F_LOSS_RADIAL:
            c->radial_dirty = true;
            break;
        case VERB_F_V: case VERB_F_K: case VERB_F_G_LOCAL: case VERB_F_LOSS_LOCAL:
            c->local_dirty = true;
            break;
        case VERB_F_DVV: case VERB_F_DKK: case VERB_F_DVK:
            c->local_dirty = true;
            c->tensor_dirty = true;
            break;
        default: break;
    }
}

EventPair get_pair(verb_ctx* c)
{
    if (!c->pool.empty()) {
        EventPair p = c->pool.back();
        c->pool.pop_back();
        return p;
    }
    EventPair p;
    cudaEventCreate(&p.a);
    cudaEventCreate(&p.b);
    return p;
}



int radial_run(verb_ctx* c, double dt)
{
    const Dims& d = c->d;
    if (d.R < 3) return VERB_OK;
    if (c->bct[VERB_BCF_LL] == VERB_BC_PERIODIC || c->bct[VERB_BCF_LU] == VERB_BC_PERIODIC)
        return VERB_ERR_BC;
    for (int fid : {VERB_F_PSD, VERB_F_L, VERB_F_DLL, VERB_F_G_RADIAL, VERB_F_LOSS_RADIAL}) {
        int s = need_field(c, fid);
        if (s) return s;
    }
    if (c->radial_sources) {
        int s = need_field(c, VERB_F_SOURCES);
        if (s) return s;
    }
    for (int b : {VERB_BCF_LL, VERB_BCF_LU}) {
        int s = need_bc(c, b);
        if (s) return s;
    }
    const size_t nl = (size_t)d.P * d.V * d.K * d.R;
    CK(alloc((void**)&c->rfa, nl * sizeof(double)));
    CK(alloc((void**)&c->rfbet, nl * sizeof(double)));
    CK(alloc((void**)&c->rfgam, nl * sizeof(double)));
    RadialArgs a{};
    a.d = d;
    a.psd = c->f[VERB_F_PSD];
    a.L = c->f[VERB_F_L];
    a.DLL = c->f[VERB_F_DLL];
    a.G = c->f[VERB_F_G_RADIAL];
    a.S = c->f[VERB_F_SOURCES];
    a.loss = c->f[VERB_F_LOSS_RADIAL];
    a.dll_scale = 1.0;  // scales are materialised into the field at upload time
    a.Ll = c->bc[VERB_BCF_LL];
    a.Lu = c->bc[VERB_BCF_LU];
    a.Ll_t = c->bct[VERB_BCF_LL];
    a.Lu_t = c->bct[VERB_BCF_LU];
    a.dt = dt;
    a.radial_sources = c->radial_sources;
    a.fa = c->rfa;
    a.fbet = c->rfbet;
    a.fgam = c->rfgam;
    a.status = c->status;
    if (c->radial_dirty || dt != c->radial_dt) {
        PhaseTimer t(c, PH_RADF);
        launch_radial_factor(a, c->stream);
        c->acc.kernel_launches++;
        c->radial_dirty = false;
        c->radial_dt = dt;
    }
    {
        PhaseTimer t(c, PH_RAD);
        launch_radial_solve(a, c->stream);
        c->acc.kernel_launches++;
    }
    return check_launch();
}

// Local solve shapes chosen by the autotuner, per (P, R, V, K, factor
// precision, ragged) in this process, so later contexts of the same shape
// start with the tuned one.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int, int>, int> g_tuned_solve;

std::tuple<int, int, int, int, int, int> tune_key(const verb_ctx* c)
{
    return {c->d.P, c->d.R, c->d.V, c->d.K, c->local_prec, c->trim_k0 ? 1 : 0};
}

int solve_variant_for(verb_ctx* c)
{
    if (c->solve_variant >= 0) return c->solve_variant;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned_solve.find(tune_key(c));
    return it == g_tuned_solve.end() ? 0 : it->second;
}

int local_prepare(verb_ctx* c, LocalArgs& a, double dts)
{
    const Dims& d = c->d;
    if (d.V > 111) return VERB_ERR_ARG;  // solve windows hold kl+1 <= 128 and kv+1 <= 256
    for (int fid : {VERB_F_PSD, VERB_F_V, VERB_F_K, VERB_F_DVV, VERB_F_DKK, VERB_F_DVK,
                    VERB_F_G_LOCAL, VERB_F_LOSS_LOCAL, VERB_F_SOURCES}) {
        int s = need_field(c, fid);
        if (s) return s;
    }
    for (int b : {VERB_BCF_VL, VERB_BCF_VU, VERB_BCF_KL, VERB_BCF_KU}) {
        int s = need_bc(c, b);
        if (s) return s;
        if (c->bct[b] == VERB_BC_PERIODIC) return VERB_ERR_BC;
    }
    c->kl = d.V + 1;
    c->kv = 2 * c->kl;
    c->klp = (c->kl + 1) & ~1;
    c->kvp = (c->kv + 2) & ~1;
    c->klp32 = (c->kl + 3) & ~3;  // 16-byte columns for cp.async
    c->kvp32 = (c->kv + 4) & ~3;
    const size_t nu = c->trim_k0 ? c->local_unknowns : (size_t)d.P * d.R * d.V * d.K;
    c->local_unknowns = nu;
    if (c->refine_iters > 0) {
        CK(alloc((void**)&c->lrhs, nu * sizeof(double)));
        CK(alloc((void**)&c->lres, nu * sizeof(double)));
        CK(alloc((void**)&c->refine_red, 2 * sizeof(unsigned long long)));
    }
    // the factors themselves are allocated by the first factorisation
    // (local_factor): the Krylov form may never need them
    CK(alloc((void**)&c->lwork, nu * sizeof(double)));
    a.d = d;
    a.psd = c->f[VERB_F_PSD];
    a.Vg = c->f[VERB_F_V];
    a.Kg = c->f[VERB_F_K];
    a.DVV = c->f[VERB_F_DVV];
    a.DKK = c->f[VERB_F_DKK];
    a.DVK = c->f[VERB_F_DVK];
    a.DKV = c->dkv_override ? c->dkv_override : c->f[VERB_F_DVK];
    a.G = c->f[VERB_F_G_LOCAL];
    a.S = c->f[VERB_F_SOURCES];
    a.loss = c->f[VERB_F_LOSS_LOCAL];
    a.Vl = c->bc[VERB_BCF_VL];
    a.Vu = c->bc[VERB_BCF_VU];
    a.Kl = c->bc[VERB_BCF_KL];
    a.Ku = c->bc[VERB_BCF_KU];
    a.Vl_t = c->bct[VERB_BCF_VL];
    a.Vu_t = c->bct[VERB_BCF_VU];
    a.Kl_t = c->bct[VERB_BCF_KL];
    a.Ku_t = c->bct[VERB_BCF_KU];
    a.dt = dts;
    a.local_sources = c->local_sources;
    a.include_boundary = c->include_boundary;
    a.kl = c->kl;
    a.kv = c->kv;
    a.klp = c->klp;
    a.kvp = c->kvp;
    a.Lf = c->Lf;
    a.Uf = c->Uf;
    a.factors32 = c->local_prec == VERB_PREC_MIXED;
    a.klp32 = c->klp32;
    a.kvp32 = c->kvp32;
    a.Lf32 = c->Lf32;
    a.Uf32 = c->Uf32;
    a.ipiv = c->ipiv;
    a.k0 = c->trim_k0;
    a.uoff = c->trim_uoff;
    a.solve_variant = solve_variant_for(c);
    a.work = c->lwork;
    a.status = c->status;
    return VERB_OK;
}

int alloc_factors(verb_ctx* c, LocalArgs& a)
{
    const size_t nu = c->local_unknowns;
    if (c->local_prec == VERB_PREC_MIXED) {
        CK(alloc((void**)&c->Lf32, nu * c->klp32 * sizeof(float)));
        CK(alloc((void**)&c->Uf32, nu * c->kvp32 * sizeof(float)));
    } else {
        CK(alloc((void**)&c->Lf, nu * c->klp * sizeof(double)));
        CK(alloc((void**)&c->Uf, nu * c->kvp * sizeof(double)));
    }
    CK(alloc((void**)&c->ipiv, nu * sizeof(int32_t)));
    a.Lf = c->Lf;
    a.Uf = c->Uf;
    a.Lf32 = c->Lf32;
    a.Uf32 = c->Uf32;
    a.ipiv = c->ipiv;
    return VERB_OK;
}

int local_factor(verb_ctx* c, LocalArgs& a)
{
    CK(alloc_factors(c, a));
    PhaseTimer t(c, PH_LOCF);
    const size_t nu = c->local_unknowns;
    if (a.factors32)
        CK(cudaMemsetAsync(c->Uf32, 0, nu * c->kvp32 * sizeof(float), c->stream));
    else
        CK(cudaMemsetAsync(c->Uf, 0, nu * c->kvp * sizeof(double), c->stream));
    c->acc.kernel_launches += launch_local_factor(a, c->stream);
    c->local_dirty = false;
    c->local_dt = a.dt;
    c->acc.local_factor_launches++;
    return check_launch();
}

int local_run(verb_ctx* c, double dt, double sub_dt)
{
    const Dims& d = c->d;
    if (d.V < 3 || d.K < 3) return VERB_OK;
    int nsub = (int)(dt / sub_dt);
    if (nsub < 1) nsub = 1;
    const double dts = dt / nsub;
    LocalArgs a{};
    int s = local_prepare(c, a, dts);
    if (s) return s;
    PhaseTimer t(c, PH_LOCAL);
    if (c->local_dirty || dts != c->local_dt) {
        s = local_factor(c, a);
        if (s) return s;
    }
    const bool refine = c->refine_iters > 0;
    const size_t nall = c->local_unknowns;
    for (int k = 0; k < nsub; k++) {
        launch_local_rhs(a, k > 0, c->stream);
        c->acc.kernel_launches++;
        if (refine) CK(cudaMemcpyAsync(c->lrhs, c->lwork, nall * sizeof(double),
                                       cudaMemcpyDeviceToDevice, c->stream));
        {
            PhaseTimer ts(c, PH_LOCS);
            launch_local_solve(a, c->stream);
            c->acc.kernel_launches++;
        }
        c->acc.local_solve_launches++;
        if (refine) {
            // iterative refinement in FP64: r = b - A x, A d = r with the
            // cached factors (FP32 in the mixed form), x += d
            LocalArgs ar = a;
            ar.work = c->lres;
            for (int it = 0; it < c->refine_iters; it++) {
                launch_local_residual(a, c->lrhs, c->lwork, c->lres, c->stream);
                {
                    PhaseTimer ts(c, PH_LOCS);
                    launch_local_solve(ar, c->stream);
                }
                if (it == c->refine_iters - 1)
                    CK(cudaMemsetAsync(c->refine_red, 0, 2 * sizeof(unsigned long long), c->stream));
                launch_local_update(a, c->lwork, c->lres, c->refine_red, c->stream);
                c->acc.kernel_launches += 3;
                c->acc.local_solve_launches++;
            }
        }
    }
    launch_local_store(a, c->stream);
    c->acc.kernel_launches++;
    return check_launch();
}

int conv_run(verb_ctx* c, double dt)
{
    const Dims& d = c->d;
    if ((d.P >= 3 && d.P < 11) || (d.R >= 3 && d.R < 11)) return VERB_ERR_GRID;
    const bool pper = c->bct[VERB_BCF_PL] == VERB_BC_PERIODIC;
    if (pper != (c->bct[VERB_BCF_PU] == VERB_BC_PERIODIC)) return VERB_ERR_BC;
    const bool rper = c->bct[VERB_BCF_RL] == VERB_BC_PERIODIC;
    if (rper != (c->bct[VERB_BCF_RU] == VERB_BC_PERIODIC)) return VERB_ERR_BC;
    for (int fid : {VERB_F_PSD, VERB_F_P, VERB_F_R, VERB_F_VP, VERB_F_VR, VERB_F_SOURCES,
                    VERB_F_LOSS_CONV, VERB_F_G_CONV}) {
        int s = need_field(c, fid);
        if (s) return s;
    }
    for (int b : {VERB_BCF_PL, VERB_BCF_PU, VERB_BCF_RL, VERB_BCF_RU}) {
        int s = need_bc(c, b);
        if (s) return s;
    }
    // the streaming kernel needs both sweeps; other shapes run the contracted
    // kernel of convection.cu
    const bool stream = c->conv_arith == VERB_CONV_STREAM && conv_stream_check(d.P, d.R) == VERB_OK;
    if (!stream)
        if (int s = (c->conv_arith == VERB_CONV_EXACT ? conv_check : conv_check_fma)(d.P, d.R)) return s;
    if (!c->conv_nctas) {
        c->conv_nctas = std::max(conv_ctas(d.P, d.R), conv_ctas_fma(d.P, d.R));
        // one allocation serves every arithmetic mode of the context
        size_t b = (size_t)c->conv_nctas * conv_scratch_doubles(d.P, d.R);
        if (conv_stream_check(d.P, d.R) == VERB_OK)
            b = std::max(b, (size_t)conv_stream_ctas_max(d.P, d.R) * conv_stream_scratch_doubles(d.P, d.R));
        c->conv_scratch_bytes = b * sizeof(double);
    }
    CK(alloc((void**)&c->conv_scratch, c->conv_scratch_bytes));
    CK(alloc((void**)&c->conv_substeps, (size_t)d.V * d.K * sizeof(int)));
    CK(alloc((void**)&c->ticket, sizeof(int)));
    ConvArgs a{};
    a.d = d;
    a.psd = c->f[VERB_F_PSD];
    a.Pg = c->f[VERB_F_P];
    a.Rg = c->f[VERB_F_R];
    a.VP = c->f[VERB_F_VP];
    a.VR = c->f[VERB_F_VR];
    a.S = c->f[VERB_F_SOURCES];
    a.loss = c->f[VERB_F_LOSS_CONV];
    a.G = c->f[VERB_F_G_CONV];
    a.Pl = c->bc[VERB_BCF_PL];
    a.Pu = c->bc[VERB_BCF_PU];
    a.Rl = c->bc[VERB_BCF_RL];
    a.Ru = c->bc[VERB_BCF_RU];
    a.Pl_t = c->bct[VERB_BCF_PL];
    a.Pu_t = c->bct[VERB_BCF_PU];
    a.Rl_t = c->bct[VERB_BCF_RL];
    a.Ru_t = c->bct[VERB_BCF_RU];
    a.dt = dt;
    a.scratch = c->conv_scratch;
    a.substeps = c->conv_substeps;
    a.ticket = c->ticket;
    a.status = c->status;
    PhaseTimer t(c, PH_CONV);
    CK(cudaMemsetAsync(c->ticket, 0, sizeof(int), c->stream));
    if (stream)
        launch_convection_stream(a, conv_stream_ctas(d.P, d.R), c->stream);
    else if (c->conv_arith == VERB_CONV_EXACT)
        launch_convection(a, c->conv_nctas, c->stream);
    else
        launch_convection_fma(a, c->conv_nctas, c->stream);
    c->acc.kernel_launches++;
    return check_launch();
}

int tensor_check(verb_ctx* c, double* out)
{
    if (c->tensor_dirty) {
        for (int fid : {VERB_F_DVV, VERB_F_DKK, VERB_F_DVK}) {
            int s = need_field(c, fid);
            if (s) return s;
        }
        CK(alloc((void**)&c->red, 2 * sizeof(unsigned long long)));
        launch_tensor_min(c->f[VERB_F_DVV], c->f[VERB_F_DKK], c->f[VERB_F_DVK], npts(c), c->red + 1,
                          c->stream);
        c->acc.kernel_launches++;
        unsigned long long k = 0;
        CK(cudaMemcpyAsync(&k, c->red + 1, sizeof(k), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->tensor_min = dkey_inv(k);
        c->tensor_dirty = false;
    }
    if (out) *out = c->tensor_min;
    return VERB_OK;
}

int harvest_timing(verb_ctx* c)
{
    CK(cudaStreamSynchronize(c->stream));
    double* dst[PH_N] = {&c->acc.convection_ms, &c->acc.radial_ms, &c->acc.radial_factor_ms,
                         &c->acc.local_ms, &c->acc.local_factor_ms, &c->acc.local_solve_ms,
                         &c->acc.reduce_ms, &c->acc.kf_ms};
    for (int p = 0; p < PH_N; p++) {
        for (EventPair& e : c->ev[p]) {
            float ms = 0;
            cudaEventElapsedTime(&ms, e.a, e.b);
            *dst[p] += ms;
            c->pool.push_back(e);
        }
        c->ev[p].clear();
    }
    return VERB_OK;
}

}  // namespace vctx

// ============================================================================ C ABI

extern "C" {

const char* verb_version(void) { return "verb4d_b200 0.1 (sm_100a)"; }

const char* verb_status_string(int s)
{
    switch (s) {
        case VERB_OK: return "ok";
        case VERB_ERR_PIVOT: return "singular pivot in the banded LU";
        case VERB_ERR_ARG: return "invalid argument";
        case VERB_ERR_CFL: return "Courant number > 1";
        case VERB_ERR_BC: return "unsupported boundary condition type";
        case VERB_ERR_TENSOR: return "DVV*DKK - DVK^2 < 0";
        case VERB_ERR_NAN: return "NaN in the PSD (after a step or the Kalman update)";
        case VERB_ERR_CUDA: return "CUDA error";
        case VERB_ERR_NOMEM: return "out of device memory";
        case VERB_ERR_GRID: return "convection grid shorter than 11 points";
        case VERB_TIMEOUT: return "device wait timed out";
        case VERB_ERR_SIZE: return "size beyond a fixed limit or file dimensions differ";
        case VERB_ERR_IO: return "file could not be opened, read or written";
        default: return "unknown status";
    }
}

int verb_create(verb_ctx** out, int P, int R, int V, int K, void* stream)
{
    if (!out || P < 1 || R < 1 || V < 1 || K < 1) return VERB_ERR_ARG;
    verb_ctx* c = new (std::nothrow) verb_ctx();
    if (!c) return VERB_ERR_NOMEM;
    c->d = Dims{P, R, V, K};
    for (int i = 0; i < VERB_F_COUNT; i++) c->scale[i] = 1.0;
    // reference defaults (src/ReadInitialData.cpp:495-511): periodic MLT, constant value elsewhere
    const int def[VERB_BCF_COUNT] = {0, 0, 1, 1, 1, 1, 1, 1, 1, 1};
    memcpy(c->bct, def, sizeof(def));
    int st = cuda_ok(cudaGetDevice(&c->device));
    if (!st) {
        if (stream) {
            c->stream = (cudaStream_t)stream;
        } else {
            st = cuda_ok(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
            c->own_stream = true;
        }
    }
    if (!st) st = cuda_ok(cudaMalloc(&c->status, sizeof(int)));
    if (!st) st = cuda_ok(cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    if (!st) st = cuda_ok(cudaMalloc(&c->red, 2 * sizeof(unsigned long long)));
    if (st) {
        verb_destroy(c);
        return st;
    }
    *out = c;
    return VERB_OK;
}

int verb_destroy(verb_ctx* c)
{
    if (!c) return VERB_OK;
    if (c->out_thread.joinable()) c->out_thread.join();
    if (c->out_stream) cudaStreamDestroy(c->out_stream);
    if (c->out_ev_snap) cudaEventDestroy(c->out_ev_snap);
    if (c->out_ev_host) cudaEventDestroy(c->out_ev_host);
    cudaFree(c->out_snap);
    cudaFreeHost(c->out_host);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < VERB_F_COUNT; i++) {
        cudaFree(c->f[i]);
        cudaFree(c->fbase[i]);
        if (c->upd[i]) {
            for (UpdComponent& k : c->upd[i]->comps) {
                cudaFree(k.base);
                for (auto& e : k.data_q) cudaFree(e.second);
            }
            delete c->upd[i];
        }
    }
    for (int i = 0; i < VERB_BCF_COUNT; i++) cudaFree(c->bc[i]);
    for (void* p : {(void*)c->Lf32, (void*)c->Uf32, (void*)c->lrhs, (void*)c->lres,
                    (void*)c->refine_red, (void*)c->trim_k0, (void*)c->trim_uoff,
                    (void*)c->maxabs_red})
        cudaFree(p);
    free_krylov(c);
    free_kc(c);
    if (c->step_exec) cudaGraphExecDestroy(c->step_exec);
    for (void* p : {(void*)c->rfa, (void*)c->rfbet, (void*)c->rfgam, (void*)c->Lf, (void*)c->Uf,
                    (void*)c->lwork, (void*)c->ipiv, (void*)c->conv_scratch,
                    (void*)c->conv_substeps, (void*)c->ticket, (void*)c->red, (void*)c->status,
                    (void*)c->Pa, (void*)c->kfwork, (void*)c->obs, (void*)c->kfticket})
        cudaFree(p);
    for (int p = 0; p < PH_N; p++)
        for (EventPair& e : c->ev[p]) c->pool.push_back(e);
    for (EventPair& e : c->pool) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return VERB_OK;
}

int verb_device_bytes(const verb_ctx* c, size_t* bytes)
{
    if (!c || !bytes) return VERB_ERR_ARG;
    size_t b = 0;
    const size_t F = c->d.npts() * sizeof(double);
    for (int i = 0; i < VERB_F_COUNT; i++) b += (c->f[i] ? F : 0) + (c->fbase[i] ? F : 0);
    for (int i = 0; i < VERB_BCF_COUNT; i++)
        if (c->bc[i]) b += bc_elems(c, i) * sizeof(double);
    if (c->rfa) b += 3 * F;
    const size_t ns = c->local_unknowns;
    if (c->Lf) b += ns * (c->klp + c->kvp) * sizeof(double);
    if (c->Lf32) b += ns * (c->klp32 + c->kvp32) * sizeof(float);
    if (c->ipiv) b += ns * sizeof(int32_t);
    if (c->lwork) b += ns * sizeof(double);
    if (c->lrhs) b += 2 * ns * sizeof(double);
    // Krylov form
    const size_t nsys = (size_t)c->d.P * c->d.R;
    if (c->kA9) b += ns * 9 * sizeof(float);
    if (c->kscr) b += ns * 6 * sizeof(float);
    if (c->kfeat) b += ns * 4 * sizeof(float);
    if (c->kout) b += ns * sizeof(float);
    for (const double* p : {c->kb, c->kx, c->kr, c->kd}) if (p) b += ns * sizeof(double);
    if (c->kscale) b += nsys * sizeof(double);
    if (c->conv_scratch) b += c->conv_scratch_bytes;
    if (c->Pa)
        b += (size_t)(c->pa_p_index >= 0 ? 1 : c->d.P) * c->d.V * c->d.K * c->d.R * c->d.R *
             sizeof(double);
    if (c->obs) b += npts(c) * sizeof(double);
    b += c->kfwork_bytes;
    *bytes = b;
    return VERB_OK;
}

static int upload_common(verb_ctx* c, int fid, const void* src, cudaMemcpyKind kind)
{
    if (!c || fid < 0 || fid >= VERB_F_COUNT || !src || c->upd[fid]) return VERB_ERR_ARG;
    graph_invalidate(c);
    const size_t bytes = npts(c) * sizeof(double);
    int s = ensure_field(c, fid);
    if (s) return s;
    if (c->scale[fid] != 1.0) {
        CK(alloc((void**)&c->fbase[fid], bytes));
        CK(cudaMemcpyAsync(c->fbase[fid], src, bytes, kind, c->stream));
        launch_scale_copy(c->f[fid], c->fbase[fid], c->scale[fid], npts(c), c->stream);
        c->acc.kernel_launches++;
    } else {
        CK(cudaMemcpyAsync(c->f[fid], src, bytes, kind, c->stream));
        if (c->fbase[fid]) {
            cudaFree(c->fbase[fid]);
            c->fbase[fid] = nullptr;
        }
    }
    c->uploaded[fid] = true;
    mark_dirty(c, fid);
    return check_launch();
}

int verb_upload_field(verb_ctx* c, int fid, const double* host)
{
    return upload_common(c, fid, host, cudaMemcpyHostToDevice);
}

int verb_upload_field_device(verb_ctx* c, int fid, const double* dev)
{
    return upload_common(c, fid, dev, cudaMemcpyDeviceToDevice);
}

int verb_set_field_scale(verb_ctx* c, int fid, double scale)
{
    if (!c || fid < 0 || fid >= VERB_F_COUNT || c->upd[fid]) return VERB_ERR_ARG;
    graph_invalidate(c);
    if (scale == c->scale[fid]) return VERB_OK;
    const size_t bytes = npts(c) * sizeof(double);
    if (c->f[fid]) {
        if (!c->fbase[fid]) {
            // the current contents are the base (scale 1) field
            CK(cudaMalloc(&c->fbase[fid], bytes));
            CK(cudaMemcpyAsync(c->fbase[fid], c->f[fid], bytes, cudaMemcpyDeviceToDevice, c->stream));
        }
        if (scale != 1.0) {
            launch_scale_copy(c->f[fid], c->fbase[fid], scale, npts(c), c->stream);
            c->acc.kernel_launches++;
        } else {
            CK(cudaMemcpyAsync(c->f[fid], c->fbase[fid], bytes, cudaMemcpyDeviceToDevice, c->stream));
        }
        mark_dirty(c, fid);
    }
    c->scale[fid] = scale;
    return check_launch();
}

int verb_upload_bc(verb_ctx* c, int b, const double* host)
{
    if (!c || b < 0 || b >= VERB_BCF_COUNT || !host) return VERB_ERR_ARG;
    graph_invalidate(c);
    if (!c->bc[b]) CK(cudaMalloc(&c->bc[b], bc_elems(c, b) * sizeof(double)));
    CK(cudaMemcpyAsync(c->bc[b], host, bc_elems(c, b) * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
    return VERB_OK;
}

int verb_set_bc_types(verb_ctx* c, const int* types)
{
    if (!c || !types) return VERB_ERR_ARG;
    graph_invalidate(c);
    for (int i = 0; i < VERB_BCF_COUNT; i++)
        if (types[i] < 0 || types[i] > 2) return VERB_ERR_BC;
    bool rad = types[VERB_BCF_LL] != c->bct[VERB_BCF_LL] || types[VERB_BCF_LU] != c->bct[VERB_BCF_LU];
    bool loc = false;
    for (int b : {VERB_BCF_VL, VERB_BCF_VU, VERB_BCF_KL, VERB_BCF_KU})
        loc = loc || types[b] != c->bct[b];
    memcpy(c->bct, types, sizeof(c->bct));
    if (rad) c->radial_dirty = true;
    if (loc) c->local_dirty = true;
    return VERB_OK;
}

int verb_set_options(verb_ctx* c, int radial_sources, int local_sources, int include_boundary,
                     int positive_psd)
{
    if (!c) return VERB_ERR_ARG;
    graph_invalidate(c);
    c->radial_sources = radial_sources;
    c->local_sources = local_sources;
    if ((include_boundary != 0) != (c->include_boundary != 0)) c->local_dirty = true;
    c->include_boundary = include_boundary;
    c->positive_psd = positive_psd;
    return VERB_OK;
}

int verb_set_local_precision(verb_ctx* c, int mode, int refinements)
{
    if (!c || (mode != VERB_PREC_FP64 && mode != VERB_PREC_MIXED) || refinements < 0 ||
        refinements > 16)
        return VERB_ERR_ARG;
    graph_invalidate(c);
    if (mode != c->local_prec) {
        // release the other form's factors before the next factorisation
        // allocates this one's
        CK(cudaStreamSynchronize(c->stream));
        if (mode == VERB_PREC_MIXED) {
            cudaFree(c->Lf);
            cudaFree(c->Uf);
            c->Lf = c->Uf = nullptr;
        } else {
            cudaFree(c->Lf32);
            cudaFree(c->Uf32);
            c->Lf32 = c->Uf32 = nullptr;
        }
        c->local_prec = mode;
        c->local_dirty = true;
    }
    c->refine_iters = refinements;
    return VERB_OK;
}

int verb_local_refinement(verb_ctx* c, double* rel_correction)
{
    if (!c || !rel_correction) return VERB_ERR_ARG;
    if (!c->refine_red || c->refine_iters == 0) {
        *rel_correction = 0.0;
        return VERB_OK;
    }
    unsigned long long k[2];
    CK(cudaMemcpyAsync(k, c->refine_red, sizeof(k), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const double md = dkey_inv(k[0]), mx = dkey_inv(k[1]);
    *rel_correction = mx > 0 ? md / mx : md;
    return VERB_OK;
}

int verb_invalidate_lu(verb_ctx* c)
{
    if (!c) return VERB_ERR_ARG;
    graph_invalidate(c);
    c->local_dirty = true;
    c->radial_dirty = true;
    return VERB_OK;
}

int verb_download_field(verb_ctx* c, int fid, double* host)
{
    if (!c || fid < 0 || fid >= VERB_F_COUNT || !host || !c->f[fid]) return VERB_ERR_ARG;
    CK(cudaMemcpyAsync(host, c->f[fid], npts(c) * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return VERB_OK;
}

int verb_download_psd(verb_ctx* c, double* host) { return verb_download_field(c, VERB_F_PSD, host); }

int verb_field_device_ptr(verb_ctx* c, int fid, double** dev)
{
    if (!c || fid < 0 || fid >= VERB_F_COUNT || !dev) return VERB_ERR_ARG;
    int s = ensure_field(c, fid);
    if (s) return s;
    *dev = c->f[fid];
    return VERB_OK;
}

int verb_convection(verb_ctx* c, double dt)
{
    if (!c || !(dt > 0)) return VERB_ERR_ARG;
    return conv_run(c, dt);
}

int verb_radial(verb_ctx* c, double dt)
{
    if (!c || !(dt > 0)) return VERB_ERR_ARG;
    return radial_run(c, dt);
}

int verb_local(verb_ctx* c, double dt, double sub_dt)
{
    if (!c || !(dt > 0) || !(sub_dt > 0)) return VERB_ERR_ARG;
    return local_run(c, dt, sub_dt);
}

int verb_local_solve_variants(int* count)
{
    if (!count) return VERB_ERR_ARG;
    *count = local_solve_variants();
    return VERB_OK;
}

int verb_local_solve_variant(int v, int* warps_per_cta, int* l_columns, int* u_columns)
{
    if (v < 0 || v >= local_solve_variants() || !warps_per_cta || !l_columns || !u_columns)
        return VERB_ERR_ARG;
    local_solve_variant_shape(v, warps_per_cta, l_columns, u_columns);
    return VERB_OK;
}

int verb_local_solve_variant_window(int v, int* in_registers)
{
    if (v < 0 || v >= local_solve_variants() || !in_registers) return VERB_ERR_ARG;
    int w = 0, f = 0, b = 0;
    local_solve_variant_shape(v, &w, &f, &b, in_registers);
    return VERB_OK;
}

int verb_set_local_solve_variant(verb_ctx* c, int v)
{
    if (!c || v < -1 || v >= local_solve_variants()) return VERB_ERR_ARG;
    graph_invalidate(c);
    c->solve_variant = v;
    return VERB_OK;
}

int verb_autotune_local_solve(verb_ctx* c, double dt, double sub_dt, double* times_ms, int* chosen)
{
    if (!c || !(dt > 0) || !(sub_dt > 0)) return VERB_ERR_ARG;
    const Dims& d = c->d;
    if (d.V < 3 || d.K < 3) return VERB_ERR_ARG;
    int nsub = (int)(dt / sub_dt);
    if (nsub < 1) nsub = 1;
    LocalArgs a{};
    int s = local_prepare(c, a, dt / nsub);
    if (s) return s;
    if (c->local_dirty || dt / nsub != c->local_dt) {
        s = local_factor(c, a);
        if (s) return s;
    }
    graph_invalidate(c);
    // the first sub-step's right-hand sides, kept aside: every trial solves
    // the same systems in place
    const size_t nu = c->local_unknowns;
    launch_local_rhs(a, false, c->stream);
    double* keep = nullptr;
    CK(cudaMalloc(&keep, nu * sizeof(double)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = cuda_ok(cudaMemcpyAsync(keep, c->lwork, nu * sizeof(double),
                                     cudaMemcpyDeviceToDevice, c->stream));
    const int nv = local_solve_variants();
    int best = 0;
    float best_ms = 0;
    for (int v = 0; v < nv && !st; v++) {
        float vmin = 0;
        for (int rep = 0; rep < 3 && !st; rep++) {
            st = cuda_ok(cudaMemcpyAsync(c->lwork, keep, nu * sizeof(double),
                                         cudaMemcpyDeviceToDevice, c->stream));
            a.solve_variant = v;
            cudaEventRecord(e0, c->stream);
            launch_local_solve(a, c->stream);
            cudaEventRecord(e1, c->stream);
            if (!st) st = cuda_ok(cudaEventSynchronize(e1));
            if (!st) st = check_launch();
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep == 0 || ms < vmin) vmin = ms;
        }
        if (times_ms) times_ms[v] = vmin;
        if (v == 0 || vmin < best_ms) {
            best_ms = vmin;
            best = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(keep);
    if (st) return st;
    c->solve_variant = best;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned_solve[tune_key(c)] = best;
    }
    if (chosen) *chosen = best;
    return VERB_OK;
}

int verb_set_convection_arith(verb_ctx* c, int mode)
{
    if (!c || (mode != VERB_CONV_EXACT && mode != VERB_CONV_FMA && mode != VERB_CONV_STREAM))
        return VERB_ERR_ARG;
    graph_invalidate(c);
    c->conv_arith = mode;
    return VERB_OK;
}

int verb_clamp_positive(verb_ctx* c)
{
    if (!c || !c->f[VERB_F_PSD]) return VERB_ERR_ARG;
    launch_clamp_positive(c->f[VERB_F_PSD], npts(c), c->stream);
    c->acc.kernel_launches++;
    return check_launch();
}

int verb_negative_count(verb_ctx* c, long long* count)
{
    if (!c || !c->f[VERB_F_PSD]) return VERB_ERR_ARG;
    {
        PhaseTimer t(c, PH_RED);
        launch_negative_count(c->f[VERB_F_PSD], npts(c), c->red, c->status, c->stream);
        c->acc.kernel_launches++;
    }
    if (count) {
        unsigned long long k = 0;
        CK(cudaMemcpyAsync(&k, c->red, sizeof(k), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        *count = (long long)k;
    }
    return check_launch();
}

int verb_tensor_check(verb_ctx* c, double* min_value)
{
    if (!c) return VERB_ERR_ARG;
    return tensor_check(c, min_value);
}

int verb_field_maxabs(verb_ctx* c, int n, const int* fields, double* out)
{
    if (!c || n < 1 || n > MAXABS_FIELDS || !fields || !out) return VERB_ERR_ARG;
    MaxabsArgs a{};
    for (int i = 0; i < n; i++) {
        if (fields[i] < 0 || fields[i] >= VERB_F_COUNT || !c->f[fields[i]]) return VERB_ERR_ARG;
        a.x[i] = c->f[fields[i]];
    }
    a.nf = n;
    CK(alloc((void**)&c->maxabs_red, MAXABS_FIELDS * sizeof(unsigned long long)));
    a.out = c->maxabs_red;
    {
        PhaseTimer t(c, PH_RED);
        launch_maxabs(a, npts(c), c->stream);
        c->acc.kernel_launches++;
    }
    unsigned long long k[MAXABS_FIELDS];
    CK(cudaMemcpyAsync(k, c->maxabs_red, sizeof(k), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < n; i++) out[i] = dkey_inv(k[i]);
    return check_launch();
}

// The launches of one step after its host-side checks: phases, clamps and
// the negative-count kernel (its result is read by the caller).
int step_body(verb_ctx* c, double dt, double sub_dt, int run_convection, int run_radial,
              int run_local)
{
    const Dims& d = c->d;
    int s;
    if (c->positive_psd && (s = verb_clamp_positive(c))) return s;
    if (run_convection && (3 < d.P || 3 < d.R)) {
        s = conv_run(c, dt);
        if (s) return s;
    }
    if (c->positive_psd && (s = verb_clamp_positive(c))) return s;
    if (run_radial && d.R >= 3) {
        s = radial_run(c, dt);
        if (s) return s;
    }
    if (c->positive_psd && (s = verb_clamp_positive(c))) return s;
    if (run_local && d.V >= 3 && d.K >= 3) {
        s = local_run(c, dt, sub_dt);
        if (s) return s;
    }
    if (c->positive_psd) return verb_clamp_positive(c);
    return verb_negative_count(c, nullptr);
}

int verb_set_step_graph(verb_ctx* c, int enable)
{
    if (!c) return VERB_ERR_ARG;
    c->use_graph = enable != 0;
    c->graph_valid = false;
    if (!c->use_graph && c->step_exec) {
        CK(cudaStreamSynchronize(c->stream));
        cudaGraphExecDestroy(c->step_exec);
        c->step_exec = nullptr;
    }
    return VERB_OK;
}

int verb_step(verb_ctx* c, double dt, double sub_dt, int run_convection, int run_radial,
              int run_local, long long* negative_count)
{
    if (!c || !(dt > 0)) return VERB_ERR_ARG;
    const Dims& d = c->d;
    int s;
    const bool loc = run_local && d.V >= 3 && d.K >= 3;
    if (loc) {
        double m = 0;
        s = tensor_check(c, &m);
        if (s) return s;
        if (m < 0) return VERB_ERR_TENSOR;
    }
    // a step that factorises, allocates or is timed runs eagerly; the others
    // replay the captured graph of the same step (same dt, sub-step, phases)
    int nsub = (int)(dt / sub_dt);
    if (nsub < 1) nsub = 1;
    const bool eager =
        !c->use_graph || c->timing ||
        (loc && (c->local_dirty || dt / nsub != c->local_dt || !c->lwork)) ||
        (run_radial && d.R >= 3 && (c->radial_dirty || dt != c->radial_dt)) ||
        (run_convection && (3 < d.P || 3 < d.R) && !c->conv_scratch) || !c->red;
    const int flags = (run_convection ? 1 : 0) | (run_radial ? 2 : 0) | (run_local ? 4 : 0);
    if (eager) {
        c->graph_valid = false;
        s = step_body(c, dt, sub_dt, run_convection, run_radial, run_local);
        if (s) return s;
    } else {
        if (!(c->graph_valid && c->g_dt == dt && c->g_sub_dt == sub_dt && c->g_flags == flags)) {
            cudaGraph_t g = nullptr;
            const long long k0 = c->acc.kernel_launches;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            s = step_body(c, dt, sub_dt, run_convection, run_radial, run_local);
            const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (s || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return s ? s : cuda_ok(e);
            }
            c->g_launches = c->acc.kernel_launches - k0;
            c->acc.kernel_launches = k0;
            if (c->step_exec) cudaGraphExecDestroy(c->step_exec);
            c->step_exec = nullptr;
            const cudaError_t ei = cudaGraphInstantiate(&c->step_exec, g, 0);
            cudaGraphDestroy(g);
            CK(ei);
            c->graph_valid = true;
            c->g_dt = dt;
            c->g_sub_dt = sub_dt;
            c->g_flags = flags;
        }
        CK(cudaGraphLaunch(c->step_exec, c->stream));
        c->acc.kernel_launches += c->g_launches;
    }
    c->acc.steps++;
    if (c->positive_psd) {
        if (negative_count) *negative_count = 0;
        return check_launch();
    }
    if (negative_count) {
        unsigned long long k = 0;
        CK(cudaMemcpyAsync(&k, c->red, sizeof(k), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        *negative_count = (long long)k;
    }
    return check_launch();
}

int verb_sync(verb_ctx* c)
{
    if (!c) return VERB_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    int st = 0;
    CK(cudaMemcpy(&st, c->status, sizeof(int), cudaMemcpyDeviceToHost));
    return st;
}

int verb_set_timing(verb_ctx* c, int enable)
{
    if (!c) return VERB_ERR_ARG;
    if (!enable) harvest_timing(c);
    c->timing = enable != 0;
    if (enable) memset(&c->acc, 0, sizeof(c->acc));
    return VERB_OK;
}

int verb_get_timing(verb_ctx* c, verb_timing* out)
{
    if (!c || !out) return VERB_ERR_ARG;
    int s = harvest_timing(c);
    *out = c->acc;
    return s;
}

int verb_convection_substeps(verb_ctx* c, int* host)
{
    if (!c || !host || !c->conv_substeps) return VERB_ERR_ARG;
    CK(cudaMemcpyAsync(host, c->conv_substeps, (size_t)c->d.V * c->d.K * sizeof(int),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return VERB_OK;
}

int verb_local_pivots(verb_ctx* c, int32_t* host)
{
    if (!c || !host || !c->ipiv || c->trim_k0) return VERB_ERR_ARG;
    CK(cudaMemcpyAsync(host, c->ipiv, c->d.npts() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return VERB_OK;
}

int verb_local_factor_lapack(verb_ctx* c, int p, int r, double* ab, long* ipiv1)
{
    if (!c || !c->Lf || c->trim_k0 || p < 0 || r < 0 || p >= c->d.P || r >= c->d.R)
        return VERB_ERR_ARG;
    const int n = c->d.V * c->d.K, kl = c->kl, kv = c->kv, ldab = 2 * kl + kl + 1;
    const size_t sys = (size_t)p * c->d.R + r;
    std::vector<double> L((size_t)n * c->klp), U((size_t)n * c->kvp);
    std::vector<int32_t> ip(n);
    CK(cudaMemcpyAsync(L.data(), c->Lf + sys * n * c->klp, L.size() * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(U.data(), c->Uf + sys * n * c->kvp, U.size() * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(ip.data(), c->ipiv + sys * n, n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (ab) {
        memset(ab, 0, sizeof(double) * (size_t)ldab * n);
        for (int j = 0; j < n; j++) {
            for (int t = 0; t <= kv; t++)  // U rows j-kv+t
                if (j - kv + t >= 0) ab[(size_t)j * ldab + t] = U[(size_t)j * c->kvp + t];
            for (int i = 1; i <= kl && j + i < n; i++)
                ab[(size_t)j * ldab + kv + i] = L[(size_t)j * c->klp + (i - 1)];
        }
    }
    if (ipiv1)
        for (int j = 0; j < n; j++) ipiv1[j] = ip[j] + 1;
    return VERB_OK;
}

}  // extern "C"

// ====================================================== per-slice entry points
namespace {

struct TmpCtx {
    verb_ctx* c = nullptr;
    ~TmpCtx() { verb_destroy(c); }
};

}  // namespace

extern "C" {

int verb_tridag(const double* a, const double* b, const double* c, const double* r, double* u,
                long n)
{
    if (!a || !b || !c || !r || !u || n < 1) return VERB_ERR_ARG;
    double* dv = nullptr;
    CK(cudaMalloc(&dv, sizeof(double) * 6 * n));
    const double* src[4] = {a, b, c, r};
    int s = VERB_OK;
    for (int i = 0; i < 4 && !s; i++)
        s = cuda_ok(cudaMemcpy(dv + i * n, src[i], sizeof(double) * n, cudaMemcpyHostToDevice));
    if (!s) {
        launch_tridag(dv, dv + n, dv + 2 * n, dv + 3 * n, dv + 4 * n, n, 0);
        s = cuda_ok(cudaMemcpy(u, dv + 4 * n, sizeof(double) * n, cudaMemcpyDeviceToHost));
    }
    cudaFree(dv);
    return s;
}

int verb_diffusion_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                      int ubc_t, const double* D, const double* G, const double* S,
                      const double* loss, double dt)
{
    if (!psd || !x || !D || !G || !S || !loss || n < 3) return VERB_ERR_ARG;
    TmpCtx t;
    int s = verb_create(&t.c, 1, n, 1, 1, nullptr);
    if (s) return s;
    int types[VERB_BCF_COUNT] = {0, 0, 1, 1, lbc_t, ubc_t, 1, 1, 1, 1};
    if ((s = verb_set_bc_types(t.c, types))) return s;
    if ((s = verb_set_options(t.c, 1, 0, 1, 0))) return s;
    const int fids[6] = {VERB_F_PSD, VERB_F_L, VERB_F_DLL, VERB_F_G_RADIAL, VERB_F_SOURCES,
                         VERB_F_LOSS_RADIAL};
    const double* srcs[6] = {psd, x, D, G, S, loss};
    for (int i = 0; i < 6; i++)
        if ((s = verb_upload_field(t.c, fids[i], srcs[i]))) return s;
    if ((s = verb_upload_bc(t.c, VERB_BCF_LL, &lbc))) return s;
    if ((s = verb_upload_bc(t.c, VERB_BCF_LU, &ubc))) return s;
    if ((s = verb_radial(t.c, dt))) return s;
    if ((s = verb_sync(t.c))) return s;
    return verb_download_psd(t.c, psd);
}

int verb_diffusion_2d(double* psd, const double* x, const double* y, int nx, int ny,
                      const double* xl, const double* xu, const double* yl, const double* yu,
                      int xl_t, int xu_t, int yl_t, int yu_t, const double* Dxx, const double* Dyy,
                      const double* Dxy, const double* Dyx, const double* G, const double* S,
                      const double* loss, double dt, double sub_dt, double* lu_cache,
                      long* index_cache, int recompute_lu)
{
    if (!psd || !x || !y || nx < 3 || ny < 3) return VERB_ERR_ARG;
    TmpCtx t;
    int s = verb_create(&t.c, 1, 1, nx, ny, nullptr);
    if (s) return s;
    int types[VERB_BCF_COUNT] = {0, 0, 1, 1, 1, 1, xl_t, xu_t, yl_t, yu_t};
    if ((s = verb_set_bc_types(t.c, types))) return s;
    if ((s = verb_set_options(t.c, 0, 1, 1, 0))) return s;
    const int fids[9] = {VERB_F_PSD, VERB_F_V, VERB_F_K, VERB_F_DVV, VERB_F_DKK, VERB_F_DVK,
                         VERB_F_G_LOCAL, VERB_F_SOURCES, VERB_F_LOSS_LOCAL};
    const double* srcs[9] = {psd, x, y, Dxx, Dyy, Dxy, G, S, loss};
    for (int i = 0; i < 9; i++)
        if ((s = verb_upload_field(t.c, fids[i], srcs[i]))) return s;
    const size_t n = (size_t)nx * ny;
    double* dkv = nullptr;
    CK(cudaMalloc(&dkv, n * sizeof(double)));
    s = cuda_ok(cudaMemcpy(dkv, Dyx, n * sizeof(double), cudaMemcpyHostToDevice));
    t.c->dkv_override = dkv;
    if (!s) s = verb_upload_bc(t.c, VERB_BCF_VL, xl);
    if (!s) s = verb_upload_bc(t.c, VERB_BCF_VU, xu);
    if (!s) s = verb_upload_bc(t.c, VERB_BCF_KL, yl);
    if (!s) s = verb_upload_bc(t.c, VERB_BCF_KU, yu);
    if (!s && lu_cache && !recompute_lu) {
        // reuse the caller's LAPACK-layout factors: convert into the device layout
        LocalArgs a{};
        int nsub = (int)(dt / sub_dt);
        if (nsub < 1) nsub = 1;
        s = local_prepare(t.c, a, dt / nsub);
        if (!s) s = alloc_factors(t.c, a);
        if (!s) {
            const int kl = t.c->kl, kv = t.c->kv, klp = t.c->klp, kvp = t.c->kvp;
            const int ldab = 3 * kl + 1;
            std::vector<double> L(n * klp, 0.0), U(n * kvp, 0.0);
            std::vector<int32_t> ip(n);
            for (size_t j = 0; j < n; j++) {
                for (int q = 0; q <= kv; q++) U[j * kvp + q] = lu_cache[j * ldab + q];
                for (int i = 1; i <= kl && j + i < n; i++)
                    L[j * klp + (i - 1)] = lu_cache[j * ldab + kv + i];
                ip[j] = (int32_t)(index_cache[j] - 1);
            }
            s = cuda_ok(cudaMemcpy(t.c->Lf, L.data(), L.size() * 8, cudaMemcpyHostToDevice));
            if (!s) s = cuda_ok(cudaMemcpy(t.c->Uf, U.data(), U.size() * 8, cudaMemcpyHostToDevice));
            if (!s) s = cuda_ok(cudaMemcpy(t.c->ipiv, ip.data(), n * 4, cudaMemcpyHostToDevice));
            t.c->local_dirty = false;
            t.c->local_dt = dt / nsub;
        }
    }
    if (!s) s = verb_local(t.c, dt, sub_dt);
    if (!s) s = verb_sync(t.c);
    if (!s) s = verb_download_psd(t.c, psd);
    if (!s && lu_cache && recompute_lu) s = verb_local_factor_lapack(t.c, 0, 0, lu_cache, index_cache);
    cudaFree(dkv);
    return s;
}

int verb_convection_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                       int ubc_t, const double* ux, double dt)
{
    if (!psd || !x || !ux || n < 11) return n < 11 ? VERB_ERR_GRID : VERB_ERR_ARG;
    if ((lbc_t == VERB_BC_PERIODIC) != (ubc_t == VERB_BC_PERIODIC)) return VERB_ERR_BC;
    double* dv = nullptr;
    int* st = nullptr;
    CK(cudaMalloc(&dv, sizeof(double) * 3 * n));
    int s = cuda_ok(cudaMalloc(&st, sizeof(int)));
    if (!s) s = cuda_ok(cudaMemset(st, 0, sizeof(int)));
    if (!s) s = cuda_ok(cudaMemcpy(dv, psd, 8 * n, cudaMemcpyHostToDevice));
    if (!s) s = cuda_ok(cudaMemcpy(dv + n, x, 8 * n, cudaMemcpyHostToDevice));
    if (!s) s = cuda_ok(cudaMemcpy(dv + 2 * n, ux, 8 * n, cudaMemcpyHostToDevice));
    if (!s) {
        launch_convection_line(dv, dv + n, n, lbc, ubc, lbc_t, ubc_t, dv + 2 * n, dt, st, 0);
        s = check_launch();
    }
    int dst = 0;
    if (!s) s = cuda_ok(cudaMemcpy(psd, dv, 8 * n, cudaMemcpyDeviceToHost));
    if (!s) s = cuda_ok(cudaMemcpy(&dst, st, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(dv);
    cudaFree(st);
    return s ? s : dst;
}

int verb_convection_2d(double* psd, const double* P, const double* R, int nP, int nR,
                       const double* pl, const double* pu, const double* rl, const double* ru,
                       int pl_t, int pu_t, int rl_t, int ru_t, const double* VP, const double* VR,
                       const double* S, const double* loss, const double* G, double dt)
{
    if (!psd || !P || !R) return VERB_ERR_ARG;
    TmpCtx t;
    int s = verb_create(&t.c, nP, nR, 1, 1, nullptr);
    if (s) return s;
    int types[VERB_BCF_COUNT] = {pl_t, pu_t, rl_t, ru_t, 1, 1, 1, 1, 1, 1};
    if ((s = verb_set_bc_types(t.c, types))) return s;
    const int fids[8] = {VERB_F_PSD, VERB_F_P, VERB_F_R, VERB_F_VP, VERB_F_VR, VERB_F_SOURCES,
                         VERB_F_LOSS_CONV, VERB_F_G_CONV};
    const double* srcs[8] = {psd, P, R, VP, VR, S, loss, G};
    for (int i = 0; i < 8; i++)
        if ((s = verb_upload_field(t.c, fids[i], srcs[i]))) return s;
    if ((s = verb_upload_bc(t.c, VERB_BCF_PL, pl))) return s;
    if ((s = verb_upload_bc(t.c, VERB_BCF_PU, pu))) return s;
    if ((s = verb_upload_bc(t.c, VERB_BCF_RL, rl))) return s;
    if ((s = verb_upload_bc(t.c, VERB_BCF_RU, ru))) return s;
    if ((s = verb_convection(t.c, dt))) return s;
    if ((s = verb_sync(t.c))) return s;
    return verb_download_psd(t.c, psd);
}

int verb_assimilate_radial(verb_ctx* c, const double* obs_host, double dt, double model_error,
                           double obs_error, int p_index)
{
    if (!c || !obs_host || !(dt > 0)) return VERB_ERR_ARG;
    const Dims& d = c->d;
    if (d.R < 3 || d.R > 128) return VERB_ERR_ARG;
    for (int fid : {VERB_F_PSD, VERB_F_R, VERB_F_DLL, VERB_F_G_RADIAL}) {
        int s = need_field(c, fid);
        if (s) return s;
    }
    for (int b : {VERB_BCF_LL, VERB_BCF_LU}) {
        int s = need_bc(c, b);
        if (s) return s;
    }
    // covariances of the columns in use: one MLT (the reference's P index,
    // src/DataAssimilationDiffusion.cpp:116,139) or all of them
    if (p_index < -1 || p_index >= d.P) return VERB_ERR_ARG;
    if (c->Pa && p_index != c->pa_p_index) return VERB_ERR_ARG;
    const size_t cols = (size_t)(p_index >= 0 ? 1 : d.P) * d.V * d.K, RR = (size_t)d.R * d.R;
    if (!c->Pa) {
        CK(cudaMalloc(&c->Pa, cols * RR * sizeof(double)));
        CK(cudaMemsetAsync(c->Pa, 0, cols * RR * sizeof(double), c->stream));
        c->pa_p_index = p_index;
    }
    CK(alloc((void**)&c->obs, npts(c) * sizeof(double)));
    CK(cudaMemcpyAsync(c->obs, obs_host, npts(c) * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
    KFArgs a{};
    a.d = d;
    a.psd = c->f[VERB_F_PSD];
    a.Rg = c->f[VERB_F_R];
    a.DLL = c->f[VERB_F_DLL];
    a.G = c->f[VERB_F_G_RADIAL];
    a.Ll = c->bc[VERB_BCF_LL];
    a.Lu = c->bc[VERB_BCF_LU];
    a.dll_scale = 1.0;
    a.Ll_t = c->bct[VERB_BCF_LL];
    a.Lu_t = c->bct[VERB_BCF_LU];
    a.obs = c->obs;
    a.Pa = c->Pa;
    a.dt = dt;
    a.model_error = model_error;
    a.obs_error = obs_error;
    a.p_index = p_index;
    a.status = c->status;
    const int nctas = kf_ctas(d, p_index);
    const size_t wb = (size_t)nctas * 5 * RR * sizeof(double);
    if (wb > c->kfwork_bytes) {
        cudaFree(c->kfwork);
        c->kfwork = nullptr;
        CK(cudaMalloc(&c->kfwork, wb));
        c->kfwork_bytes = wb;
    }
    CK(alloc((void**)&c->kfticket, sizeof(int)));
    a.work = c->kfwork;
    a.ticket = c->kfticket;
    PhaseTimer t(c, PH_KF);
    launch_kf(a, nctas, c->stream);
    c->acc.kernel_launches++;
    return check_launch();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Updatable fields (src/UpdatableMatrix.cpp:602-846, 913-961).

namespace {

bool updatable_field(int fid)
{
    return fid >= VERB_F_DLL && fid < VERB_F_COUNT;  // coefficients, velocities, G, sources, losses
}

int component_of(verb_ctx* c, int fid, int comp, UpdComponent** out)
{
    if (!c || fid < 0 || fid >= VERB_F_COUNT || !c->upd[fid] || comp < 0 ||
        comp >= (int)c->upd[fid]->comps.size())
        return VERB_ERR_ARG;
    *out = &c->upd[fid]->comps[comp];
    return VERB_OK;
}

// one UpdatableMatrix::update on the host side: pop every queue entry due at
// current_time and report whether anything changed
bool pop_component(UpdComponent& k, double t, double** new_base)
{
    bool updated = false;
    // data: the last due entry, loaded only if newer than the last load (:636-661)
    double* data = nullptr;
    double data_time = 0;
    while (!k.data_q.empty() && t >= k.data_q.front().first) {
        if (data) cudaFree(data);  // superseded before it was used
        data = k.data_q.front().second;
        data_time = k.data_q.front().first;
        k.data_q.pop_front();
    }
    if (data) {
        if (t >= data_time && k.last_update_time < data_time) {
            *new_base = data;
            k.last_update_time = t;
            updated = true;
        } else {
            cudaFree(data);
        }
    }
    // scale (:676-695) and limits (:724-788): the latest due value, updated
    // whenever an entry is popped
    while (!k.scale_q.empty() && t >= k.scale_q.front().first) {
        k.scale = k.scale_q.front().second;
        k.scale_q.pop_front();
        updated = true;
    }
    for (int a = 0; a < 4; a++)
        for (int w = 0; w < 2; w++)
            while (!k.limit_q[a][w].empty() && t >= k.limit_q[a][w].front().first) {
                k.lim[a][w] = k.limit_q[a][w].front().second;
                k.limit_q[a][w].pop_front();
                updated = true;
            }
    return updated;
}

}  // namespace

int verb_field_add_component(verb_ctx* c, int fid, const double* host_base, int* comp)
{
    if (!c || !host_base || !updatable_field(fid)) return VERB_ERR_ARG;
    graph_invalidate(c);
    if (!c->upd[fid]) c->upd[fid] = new (std::nothrow) UpdField();
    if (!c->upd[fid]) return VERB_ERR_NOMEM;
    UpdField& u = *c->upd[fid];
    if ((int)u.comps.size() >= MAX_COMPONENTS) return VERB_ERR_SIZE;
    UpdComponent k;
    CK(cudaMalloc(&k.base, npts(c) * sizeof(double)));
    CK(cudaMemcpyAsync(k.base, host_base, npts(c) * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
    u.comps.push_back(k);
    u.built = false;
    if (comp) *comp = (int)u.comps.size() - 1;
    return VERB_OK;
}

int verb_field_set_merge(verb_ctx* c, int fid, int merge)
{
    if (!c || fid < 0 || fid >= VERB_F_COUNT || !c->upd[fid] ||
        (merge != VERB_MERGE_SUM && merge != VERB_MERGE_MEAN))
        return VERB_ERR_ARG;
    graph_invalidate(c);
    c->upd[fid]->merge = merge;
    c->upd[fid]->built = false;
    return VERB_OK;
}

int verb_component_queue_data(verb_ctx* c, int fid, int comp, double time, const double* host)
{
    UpdComponent* k = nullptr;
    if (int s = component_of(c, fid, comp, &k)) return s;
    if (!host || (!k->data_q.empty() && time < k->data_q.back().first)) return VERB_ERR_ARG;
    double* d = nullptr;
    CK(cudaMalloc(&d, npts(c) * sizeof(double)));
    CK(cudaMemcpyAsync(d, host, npts(c) * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k->data_q.emplace_back(time, d);
    return VERB_OK;
}

int verb_component_queue_scale(verb_ctx* c, int fid, int comp, double time, double scale)
{
    UpdComponent* k = nullptr;
    if (int s = component_of(c, fid, comp, &k)) return s;
    if (!k->scale_q.empty() && time < k->scale_q.back().first) return VERB_ERR_ARG;
    k->scale_q.emplace_back(time, scale);
    return VERB_OK;
}

int verb_component_queue_limit(verb_ctx* c, int fid, int comp, int axis, int which, double time,
                               double value)
{
    UpdComponent* k = nullptr;
    if (int s = component_of(c, fid, comp, &k)) return s;
    if (axis < 0 || axis > 3 || (which != 0 && which != 1)) return VERB_ERR_ARG;
    auto& q = k->limit_q[axis][which];
    if (!q.empty() && time < q.back().first) return VERB_ERR_ARG;
    q.emplace_back(time, value);
    return VERB_OK;
}

int verb_update_fields(verb_ctx* c, double current_time, unsigned int* updated_mask)
{
    if (!c) return VERB_ERR_ARG;
    graph_invalidate(c);
    unsigned int mask = 0;
    for (int fid = 0; fid < VERB_F_COUNT; fid++) {
        UpdField* u = c->upd[fid];
        if (!u || u->comps.empty()) continue;
        bool changed = !u->built;
        for (UpdComponent& k : u->comps) {
            double* nb = nullptr;
            if (pop_component(k, current_time, &nb)) changed = true;
            if (nb) {
                // the replacement becomes the base once the stream has used the old one
                double* old = k.base;
                k.base = nb;
                CK(cudaStreamSynchronize(c->stream));
                cudaFree(old);
            }
        }
        if (!changed) continue;
        // grid axes of the field (src/VERB4D_Solver.cpp:635-682; D_LL uses L*)
        const int ax[4] = {VERB_F_P, fid == VERB_F_DLL ? VERB_F_L : VERB_F_R, VERB_F_V, VERB_F_K};
        MergeArgs m{};
        for (int a = 0; a < 4; a++) {
            if (int s = need_field(c, ax[a])) return s;
            m.axis[a] = c->f[ax[a]];
        }
        m.ncomp = (int)u->comps.size();
        m.mean = u->merge == VERB_MERGE_MEAN;
        for (int i = 0; i < m.ncomp; i++) {
            const UpdComponent& k = u->comps[i];
            m.comp[i].base = k.base;
            m.comp[i].scale = k.scale;
            for (int a = 0; a < 4; a++) {
                m.comp[i].from[a] = k.lim[a][0];
                m.comp[i].to[a] = k.lim[a][1];
            }
        }
        if (int s = ensure_field(c, fid)) return s;
        launch_merge_components(c->f[fid], m, npts(c), c->stream);
        c->acc.kernel_launches++;
        c->uploaded[fid] = true;
        u->built = true;
        mark_dirty(c, fid);
        mask |= 1u << fid;
    }
    if (updated_mask) *updated_mask = mask;
    return check_launch();
}

// ---------------------------------------------------------------------------
// PSD output and restart files (.pltb: Matrix4D::writeToBinaryFile /
// readFromBinaryFile, src/Matrix.cpp:5700-5720, 5780-5808: four int32 sizes,
// then the values in [P][R][V][K] order), written asynchronously as the
// reference's output_writer does (src/VERB4D_Solver.cpp:1255-1267).

namespace {

int write_pltb(const char* path, const Dims& d, const double* host)
{
    FILE* f = fopen(path, "wb");
    if (!f) return VERB_ERR_IO;
    const int32_t sz[4] = {d.P, d.R, d.V, d.K};
    bool ok = fwrite(sz, sizeof(int32_t), 4, f) == 4;
    ok = ok && fwrite(host, sizeof(double), d.npts(), f) == d.npts();
    ok = (fclose(f) == 0) && ok;
    return ok ? VERB_OK : VERB_ERR_IO;
}

}  // namespace

int verb_output_wait(verb_ctx* c)
{
    if (!c) return VERB_ERR_ARG;
    if (c->out_thread.joinable()) c->out_thread.join();
    const int s = c->out_status;
    c->out_status = VERB_OK;
    return s;
}

int verb_write_field_pltb(verb_ctx* c, int fid, const char* path, int async_write)
{
    if (!c || !path || fid < 0 || fid >= VERB_F_COUNT || !c->f[fid]) return VERB_ERR_ARG;
    // one output in flight, as the reference waits for its previous writer
    if (int s = verb_output_wait(c)) return s;
    const size_t bytes = npts(c) * sizeof(double);
    if (!c->out_snap) {
        CK(cudaMalloc(&c->out_snap, bytes));
        CK(cudaMallocHost(&c->out_host, bytes));
        CK(cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->out_ev_snap, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->out_ev_host, cudaEventDisableTiming));
    }
    // snapshot on the compute stream (the next step may overwrite the field),
    // then the device-to-host copy on the output stream, overlapping compute
    CK(cudaMemcpyAsync(c->out_snap, c->f[fid], bytes, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaEventRecord(c->out_ev_snap, c->stream));
    CK(cudaStreamWaitEvent(c->out_stream, c->out_ev_snap, 0));
    CK(cudaMemcpyAsync(c->out_host, c->out_snap, bytes, cudaMemcpyDeviceToHost, c->out_stream));
    CK(cudaEventRecord(c->out_ev_host, c->out_stream));
    std::string p(path);
    c->out_thread = std::thread([c, p]() {
        int s = cuda_ok(cudaEventSynchronize(c->out_ev_host));
        if (!s) s = write_pltb(p.c_str(), c->d, c->out_host);
        c->out_status = s;
    });
    return async_write ? VERB_OK : verb_output_wait(c);
}

int verb_read_field_pltb(verb_ctx* c, int fid, const char* path)
{
    if (!c || !path || fid < 0 || fid >= VERB_F_COUNT) return VERB_ERR_ARG;
    graph_invalidate(c);
    FILE* f = fopen(path, "rb");
    if (!f) return VERB_ERR_IO;
    int32_t sz[4];
    std::vector<double> buf;
    int s = VERB_OK;
    if (fread(sz, sizeof(int32_t), 4, f) != 4) s = VERB_ERR_IO;
    else if (sz[0] != c->d.P || sz[1] != c->d.R || sz[2] != c->d.V || sz[3] != c->d.K) s = VERB_ERR_SIZE;
    if (!s) {
        buf.resize(npts(c));
        if (fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) s = VERB_ERR_IO;
    }
    fclose(f);
    if (s) return s;
    s = verb_upload_field(c, fid, buf.data());
    if (!s) s = cuda_ok(cudaStreamSynchronize(c->stream));
    return s;
}

int verb_append_lst(const char* lst_path, double time, const char* filename)
{
    // Matrix4D::writeToLstFile (src/Matrix.cpp:5760-5778) with the time as
    // write_PSD_output formats it (fixed, 5 decimals; VERB4D_Solver.cpp:180-184)
    if (!lst_path || !filename) return VERB_ERR_ARG;
    FILE* f = fopen(lst_path, "a");
    if (!f) return VERB_ERR_IO;
    const bool ok = fprintf(f, "%.5f\t%s\n", time, filename) > 0;
    return (fclose(f) == 0 && ok) ? VERB_OK : VERB_ERR_IO;
}

// ---------------------------------------------------------------------------
// L* remapping (src/VERB4D_Solver.cpp:557-619).

int verb_remap_L(verb_ctx* c, const double* new_L_host)
{
    if (!c || !new_L_host) return VERB_ERR_ARG;
    graph_invalidate(c);
    for (int fid : {VERB_F_PSD, VERB_F_L}) {
        int s = need_field(c, fid);
        if (s) return s;
    }
    if (c->upd[VERB_F_L]) return VERB_ERR_ARG;
    const size_t bytes = npts(c) * sizeof(double);
    double *newL = nullptr, *scratch = nullptr;
    CK(cudaMalloc(&newL, bytes));
    int s = cuda_ok(cudaMalloc(&scratch, 2 * bytes));
    if (!s) s = cuda_ok(cudaMemcpyAsync(newL, new_L_host, bytes, cudaMemcpyHostToDevice, c->stream));
    if (!s) {
        launch_remap(c->f[VERB_F_PSD], c->f[VERB_F_L], newL, scratch, scratch + npts(c), c->d,
                     c->status, c->stream);
        c->acc.kernel_launches++;
        s = check_launch();
    }
    if (!s) s = cuda_ok(cudaMemcpyAsync(c->f[VERB_F_L], newL, bytes, cudaMemcpyDeviceToDevice, c->stream));
    if (!s) s = cuda_ok(cudaStreamSynchronize(c->stream));
    cudaFree(newL);
    cudaFree(scratch);
    if (s) return s;
    mark_dirty(c, VERB_F_L);
    return verb_sync(c);
}

// ---------------------------------------------------------------------------
// Device memory a context of the given size will hold (no allocation): the
// fields and boundary arrays, the cached radial and local factors in the
// chosen precision, the convection scratch and, with kf_columns > 0, the
// Kalman-filter covariances of that many columns.  Used to admit ensemble
// members within an HBM budget.
int verb_estimate_device_bytes(int P, int R, int V, int K, int precision, int refinements,
                               long long kf_columns, size_t* bytes)
{
    if (!bytes || P < 1 || R < 1 || V < 1 || K < 1) return VERB_ERR_ARG;
    const size_t np = (size_t)P * R * V * K;
    size_t b = (VERB_F_COUNT + 1) * np * sizeof(double);                  // fields + D_LL base
    b += (2 * (size_t)R * V * K + 4 * (size_t)P * V * K + 2 * (size_t)P * R * K +
          2 * (size_t)P * R * V) * sizeof(double);                          // boundary arrays
    b += 3 * np * sizeof(double);                                           // radial factors
    if (V >= 3 && K >= 3) {
        const int kl = V + 1, kv = 2 * kl;
        if (precision == VERB_PREC_MIXED)
            b += np * ((size_t)((kl + 3) & ~3) + ((kv + 4) & ~3)) * sizeof(float);
        else
            b += np * ((size_t)((kl + 1) & ~1) + ((kv + 2) & ~1)) * sizeof(double);
        b += np * (sizeof(double) + sizeof(int32_t));                       // work, pivots
        if (refinements > 0) b += 2 * np * sizeof(double);
    }
    if (P >= 3 || R >= 3) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        size_t cb = (size_t)2 * sms * conv_scratch_doubles(P, R);
        if (conv_stream_check(P, R) == VERB_OK)
            cb = std::max(cb, (size_t)conv_stream_ctas_max(P, R) * conv_stream_scratch_doubles(P, R));
        b += cb * sizeof(double);
    }
    if (kf_columns > 0)
        b += ((size_t)kf_columns * R * R + np) * sizeof(double) +
             (size_t)2 * 148 * 5 * R * R * sizeof(double);
    *bytes = b;
    return VERB_OK;
}

// ---------------------------------------------------------------------------
// Ragged local systems: each (P,R) system keeps pitch-angle indices
// k0[sys]..K-1 (the trapped range outside the loss cone), with a
// ConstantValue 0 boundary at its new lower edge.  Systems with fewer than 3
// pitch angles left are not solved.  Passing nullptr restores full systems.
int verb_set_local_trim(verb_ctx* c, const int* k0_host)
{
    if (!c) return VERB_ERR_ARG;
    graph_invalidate(c);
    const Dims& d = c->d;
    const size_t nsys = (size_t)d.P * d.R;
    CK(cudaStreamSynchronize(c->stream));
    // the factor arrays change size: release them (refactored at the next solve)
    for (void** p : {(void**)&c->Lf, (void**)&c->Uf, (void**)&c->Lf32, (void**)&c->Uf32,
                     (void**)&c->ipiv, (void**)&c->lwork, (void**)&c->lrhs, (void**)&c->lres}) {
        cudaFree(*p);
        *p = nullptr;
    }
    free_krylov(c);
    cudaFree(c->trim_k0);
    cudaFree(c->trim_uoff);
    c->trim_k0 = nullptr;
    c->trim_uoff = nullptr;
    c->local_dirty = true;
    if (!k0_host) {
        c->local_unknowns = nsys * d.V * d.K;
        return VERB_OK;
    }
    std::vector<long long> off(nsys);
    long long tot = 0;
    for (size_t s = 0; s < nsys; s++) {
        if (k0_host[s] < 0 || k0_host[s] > d.K) return VERB_ERR_ARG;
        off[s] = tot;
        tot += (long long)d.V * (d.K - k0_host[s]);
    }
    CK(cudaMalloc(&c->trim_k0, nsys * sizeof(int)));
    CK(cudaMalloc(&c->trim_uoff, nsys * sizeof(long long)));
    CK(cudaMemcpy(c->trim_k0, k0_host, nsys * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->trim_uoff, off.data(), nsys * sizeof(long long), cudaMemcpyHostToDevice));
    c->local_unknowns = (size_t)tot;
    return VERB_OK;
}
