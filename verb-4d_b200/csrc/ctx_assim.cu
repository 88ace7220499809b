// Context side of the convection data assimilation
// (verb_assimilate_convection): per-slice model-matrix cache and analysis
// covariances, chunking of the (V,K) slices, binary exponentiation with
// per-slice exponents, and the sequence of batched kernels in kfconv.cu.
#include "ctx_internal.cuh"

namespace vctx {

void free_kc(verb_ctx* c)
{
    for (void** p : {(void**)&c->kc_M, (void**)&c->kc_Pa, (void**)&c->kc_W, (void**)&c->kc_vec,
                     (void**)&c->kc_int})
    {
        cudaFree(*p);
        *p = nullptr;
    }
    c->kc_valid = false;
    c->kc_chunk = 0;
}

// out[b] = base[b]^e[b] for the slices of a chunk (binary exponentiation;
// products of powers of one matrix commute, so the order of the factors
// only changes rounding).  cur and sq hold the running square, tmp the
// product; idx_dev is scratch for the per-bit slice lists.
int kc_pow(verb_ctx* c, int nb, const double* base, size_t sbase, const std::vector<int>& e,
           double* out, size_t sout, double* cur, double* sq, double* tmp, size_t sW, int* idx_dev)
{
    const int N = c->d.P * c->d.R;
    const size_t NN = (size_t)N * N;
    launch_kc_copy(base, sbase, cur, sW, NN, nb, nullptr, c->stream);
    int emax = 0;
    for (int v : e) emax = std::max(emax, v);
    std::vector<char> started(nb, 0);
    std::vector<int> sel;
    auto gemm = [&](const double* A, size_t sA, const double* B, size_t sB, double* C, size_t sC,
                    int batch, const int* idx) {
        BGemm g{};
        g.A = A; g.sA = sA; g.lda = N;
        g.B = B; g.sB = sB; g.ldb = N;
        g.C = C; g.sC = sC; g.ldc = N;
        g.M = N; g.N = N; g.K = N;
        g.sgn = 1.0;
        g.idx = idx;
        launch_bgemm(g, false, batch, c->stream);
        c->acc.kernel_launches++;
    };
    for (int bit = 0; (1 << bit) <= emax; bit++) {
        std::vector<int> first, mult;
        for (int b = 0; b < nb; b++)
            if (e[b] >> bit & 1) (started[b] ? mult : first).push_back(b);
        if (!first.empty()) {
            CK(cudaMemcpyAsync(idx_dev, first.data(), first.size() * sizeof(int),
                               cudaMemcpyHostToDevice, c->stream));
            launch_kc_copy(cur, sW, out, sout, NN, (int)first.size(), idx_dev, c->stream);
            for (int b : first) started[b] = 1;
        }
        if (!mult.empty()) {
            int* id2 = idx_dev + nb;
            CK(cudaMemcpyAsync(id2, mult.data(), mult.size() * sizeof(int), cudaMemcpyHostToDevice,
                               c->stream));
            gemm(out, sout, cur, sW, tmp, sW, (int)mult.size(), id2);
            launch_kc_copy(tmp, sW, out, sout, NN, (int)mult.size(), id2, c->stream);
        }
        if ((2 << bit) <= emax) {
            gemm(cur, sW, cur, sW, sq, sW, nb, nullptr);
            std::swap(cur, sq);
        }
        // the host lists are reused by the next bit: let the copies finish
        CK(cudaStreamSynchronize(c->stream));
    }
    return VERB_OK;
}

int kc_run(verb_ctx* c, const double* obs_host, double dt, double model_error, double obs_error,
           int use_log, double corr_time, int growing_q, int has_vx_updated, int chunk)
{
    const Dims& d = c->d;
    for (int fid : {VERB_F_PSD, VERB_F_P, VERB_F_R, VERB_F_VP, VERB_F_VR}) {
        int s = need_field(c, fid);
        if (s) return s;
    }
    if (d.P < 3 || d.R < 3) return VERB_ERR_GRID;
    const int N = d.P * d.R;
    const size_t NN = (size_t)N * N;
    const int nsl = d.V * d.K;
    // persistent: the model matrix cache and Pa of every slice
    if (!c->kc_M) {
        CK(alloc((void**)&c->kc_M, (size_t)nsl * NN * sizeof(double)));
        CK(alloc((void**)&c->kc_Pa, (size_t)nsl * NN * sizeof(double)));
        CK(cudaMemsetAsync(c->kc_Pa, 0, (size_t)nsl * NN * sizeof(double), c->stream));
        c->kc_valid = false;
    }
    int B = chunk > 0 ? chunk : (int)std::max<size_t>(1, ((size_t)4 << 30) / (4 * NN * sizeof(double)));
    B = std::min(B, nsl);
    if (c->kc_chunk != B) {
        for (void** p : {(void**)&c->kc_W, (void**)&c->kc_vec, (void**)&c->kc_int}) {
            cudaFree(*p);
            *p = nullptr;
        }
        c->kc_chunk = B;
    }
    CK(alloc((void**)&c->kc_W, (size_t)B * 4 * NN * sizeof(double)));
    CK(alloc((void**)&c->kc_vec, (size_t)B * 3 * N * sizeof(double)));   // t, x, y
    CK(alloc((void**)&c->kc_int, ((size_t)B * (N + 4)) * sizeof(int)));  // oidx, m, nt, 2 lists
    CK(alloc((void**)&c->obs, npts(c) * sizeof(double)));
    CK(cudaMemcpyAsync(c->obs, obs_host, npts(c) * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
    double* W0 = c->kc_W;
    double* W1 = W0 + (size_t)B * NN;
    double* W2 = W1 + (size_t)B * NN;
    double* W3 = W2 + (size_t)B * NN;
    double* tv = c->kc_vec;
    double* xv = tv + (size_t)B * N;
    double* yv = xv + (size_t)B * N;
    int* oidx = c->kc_int;
    int* mdev = oidx + (size_t)B * N;
    int* ntdev = mdev + B;
    int* lists = ntdev + B;  // 2 * B
    const bool rebuild = has_vx_updated || !c->kc_valid;
    const int e1d = (int)std::ceil(3. / 24 / dt);
    KCArgs a{};
    a.d = d;
    a.dt = dt;
    a.model_error = model_error;
    a.obs_error = obs_error;
    a.corr_time = corr_time;
    a.use_log = use_log;
    a.growing_q = growing_q;
    a.Pg = c->f[VERB_F_P];
    a.Rg = c->f[VERB_F_R];
    a.VP = c->f[VERB_F_VP];
    a.VR = c->f[VERB_F_VR];
    a.S = c->f[VERB_F_SOURCES];
    a.psd = c->f[VERB_F_PSD];
    a.obs = c->obs;
    a.status = c->status;
    for (int s0 = 0; s0 < nsl; s0 += B) {
        const int nb = std::min(B, nsl - s0);
        a.s0 = s0;
        double* Mc = c->kc_M + (size_t)s0 * NN;
        double* Pa = c->kc_Pa + (size_t)s0 * NN;
        if (rebuild) {
            std::vector<int> nt(nb);
            launch_kc_split(a, nb, ntdev, c->stream);
            CK(cudaMemcpyAsync(nt.data(), ntdev, nb * sizeof(int), cudaMemcpyDeviceToHost,
                               c->stream));
            launch_kc_model(a, nb, ntdev, W0, NN, c->stream);
            CK(cudaStreamSynchronize(c->stream));
            c->acc.kernel_launches += 2;
            CK(kc_pow(c, nb, W0, NN, nt, Mc, NN, W1, W2, W3, NN, lists));
        }
        // M1d = M^ceil(3/24/dt) into W1 (W0 and W2 as scratch; W3 the product)
        {
            std::vector<int> e(nb, e1d);
            CK(kc_pow(c, nb, Mc, NN, e, W3, NN, W0, W2, W1, NN, lists));
        }
        // Q = M1d diag(t) M1d^T (+ diagonal terms) into W2
        launch_kc_tdiag(a, nb, tv, N, c->stream);
        {
            BGemm g{};
            g.A = W3; g.sA = NN; g.lda = N;
            g.B = W3; g.sB = NN; g.ldb = N;
            g.C = W2; g.sC = NN; g.ldc = N;
            g.dk = tv; g.sdk = N;
            g.M = N; g.N = N; g.K = N;
            g.sgn = 1.0;
            launch_bgemm(g, true, nb, c->stream);
        }
        launch_kc_qdiag(a, nb, W2, NN, c->stream);
        launch_kc_pa_init(a, nb, c->kc_Pa, NN, c->stream);
        // Pf = (M Pa) M^T + Q into W3 (W0 = M Pa)
        {
            BGemm g{};
            g.A = Mc; g.sA = NN; g.lda = N;
            g.B = Pa; g.sB = NN; g.ldb = N;
            g.C = W0; g.sC = NN; g.ldc = N;
            g.M = N; g.N = N; g.K = N;
            g.sgn = 1.0;
            launch_bgemm(g, false, nb, c->stream);
            BGemm h{};
            h.A = W0; h.sA = NN; h.lda = N;
            h.B = Mc; h.sB = NN; h.ldb = N;
            h.C = W3; h.sC = NN; h.ldc = N;
            h.Cin = W2; h.sCin = NN; h.ldcin = N;
            h.M = N; h.N = N; h.K = N;
            h.sgn = 1.0;
            launch_bgemm(h, true, nb, c->stream);
        }
        // observation space, gain, update
        launch_kc_obs(a, nb, mdev, oidx, yv, xv, N, c->stream);
        std::vector<int> m(nb);
        CK(cudaMemcpyAsync(m.data(), mdev, nb * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        int mm = 0;
        for (int v : m) mm = std::max(mm, v);
        c->acc.kernel_launches += 8;
        if (mm == 0) {
            // no observation in the chunk: x unchanged, Pa = Pf
            launch_kc_copy(W3, NN, Pa, NN, NN, nb, nullptr, c->stream);
            continue;
        }
        launch_kc_gain(a, nb, W3, NN, W0, W1, NN, mdev, oidx, yv, xv, N, mm, c->stream);
        launch_kc_update(a, nb, W0, NN, mdev, oidx, yv, xv, N, mm, W3, NN, W2, c->stream);
        {
            BGemm g{};
            g.A = W0; g.sA = NN; g.lda = mm;
            g.B = W2; g.sB = NN; g.ldb = N;
            g.C = Pa; g.sC = NN; g.ldc = N;
            g.Cin = W3; g.sCin = NN; g.ldcin = N;
            g.M = N; g.N = N; g.K = mm;
            g.sgn = -1.0;
            launch_bgemm(g, false, nb, c->stream);
        }
        c->acc.kernel_launches += 4;
    }
    c->kc_valid = true;
    CK(check_launch());
    int st = VERB_OK;
    CK(cudaMemcpyAsync(&st, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return st;
}

}  // namespace vctx

extern "C" {

int verb_assimilate_convection(verb_ctx* c, const double* obs_host, double dt, double model_error,
                               double obs_error, int use_log, double correlation_time,
                               int growing_q, int has_vx_updated, int slice_chunk)
{
    if (!c || !obs_host || !(dt > 0) || !(dt <= 0.125) || !(model_error > 0) ||
        !(obs_error > 0) || !(correlation_time > 0) || slice_chunk < 0)
        return VERB_ERR_ARG;
    return kc_run(c, obs_host, dt, model_error, obs_error, use_log, correlation_time, growing_q,
                  has_vx_updated, slice_chunk);
}

int verb_convection_da_state(verb_ctx* c, int v, int k, double* Pa_host, double* model_host)
{
    if (!c || v < 0 || v >= c->d.V || k < 0 || k >= c->d.K || !c->kc_Pa) return VERB_ERR_ARG;
    const size_t NN = (size_t)c->d.P * c->d.R * c->d.P * c->d.R;
    const size_t sl = (size_t)v * c->d.K + k;
    if (Pa_host)
        CK(cudaMemcpyAsync(Pa_host, c->kc_Pa + sl * NN, NN * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
    if (model_host)
        CK(cudaMemcpyAsync(model_host, c->kc_M + sl * NN, NN * sizeof(double),
                           cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return VERB_OK;
}

}  // extern "C"
