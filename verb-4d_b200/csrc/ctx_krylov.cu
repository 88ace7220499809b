// Context side of the Krylov form of the local solve (verb_local_krylov) and
// of the training triples (verb_local_triples): buffers, the outer FP64
// refinement around the FP32 BiCGSTAB kernels, the per-system residual check
// and the LU fallback.  The kernels are in local.cu and cnn.cu.
#include "ctx_internal.cuh"

namespace vctx {

void free_krylov(verb_ctx* c)
{
    for (void** p : {(void**)&c->kA9, (void**)&c->kscr, (void**)&c->kfeat, (void**)&c->kout,
                     (void**)&c->kb, (void**)&c->kx, (void**)&c->kr, (void**)&c->kd,
                     (void**)&c->kscale, (void**)&c->kiters, (void**)&c->kpend,
                     (void**)&c->kcount, (void**)&c->kmax, (void**)&c->kprev,
                     (void**)&c->kpfeat, (void**)&c->kpc}) {
        cudaFree(*p);
        *p = nullptr;
    }
}

int krylov_buffers(verb_ctx* c, bool features)
{
    const size_t nu = c->local_unknowns;
    const size_t ns = (size_t)c->d.P * c->d.R;
    CK(alloc((void**)&c->kb, nu * sizeof(double)));
    CK(alloc((void**)&c->kscale, ns * sizeof(double)));
    if (!c->kpend) {
        // systems the residual check skips keep pend = 0
        CK(alloc((void**)&c->kpend, ns));
        CK(cudaMemsetAsync(c->kpend, 0, ns, c->stream));
    }
    CK(alloc((void**)&c->kcount, 2 * sizeof(unsigned int)));
    CK(alloc((void**)&c->kmax, 4 * sizeof(unsigned long long)));
    if (features) {
        if (!c->kfeat) {
            // skipped systems keep zero features: the network reads them too
            CK(alloc((void**)&c->kfeat, nu * 4 * sizeof(float)));
            CK(cudaMemsetAsync(c->kfeat, 0, nu * 4 * sizeof(float), c->stream));
        }
        CK(alloc((void**)&c->kout, nu * sizeof(float)));
    }
    return VERB_OK;
}

// The local step with the Krylov solve (see verb_local_krylov).
int krylov_run(verb_ctx* c, double dt, double sub_dt, int guess, verb_cnn* cnn, int smooth,
               double omega, int max_outer, int inner_maxit, double inner_tol, double resid_tol,
               verb_krylov_stats* stats)
{
    const Dims& d = c->d;
    if (stats) *stats = verb_krylov_stats{};
    if (d.V < 3 || d.K < 3) return VERB_OK;
    const int nsys = d.P * d.R;
    if (cnn) {
        int ci, co, H, W, mb;
        CK(cnn_shape(cnn, &ci, &co, &H, &W, &mb));
        if (ci != 4 || co != 1 || H != d.K || W != d.V || mb < nsys || c->trim_k0)
            return VERB_ERR_ARG;
    }
    int nsub = (int)(dt / sub_dt);
    if (nsub < 1) nsub = 1;
    const double dts = dt / nsub;
    LocalArgs a{};
    int s = local_prepare(c, a, dts);
    if (s) return s;
    PhaseTimer t(c, PH_LOCAL);
    const size_t nu = c->local_unknowns;
    CK(krylov_buffers(c, cnn != nullptr));
    for (double** p : {&c->kx, &c->kr, &c->kd}) CK(alloc((void**)p, nu * sizeof(double)));
    CK(alloc((void**)&c->kA9, nu * 9 * sizeof(float)));
    CK(alloc((void**)&c->kscr, nu * 6 * sizeof(float)));
    CK(alloc((void**)&c->kiters, nsys * sizeof(int)));
    CK(alloc((void**)&c->kprev, nsys * sizeof(double)));
    // the FP32 matrices depend on the coefficients and the sub-step only;
    // they are rebuilt every call (one pass over the coefficient fields)
    launch_local_assemble32(a, c->kA9, c->stream);
    c->acc.kernel_launches++;
    if (c->kpc_net) {
        // the learned preconditioner's coefficients from the matrix
        if (c->trim_k0) return VERB_ERR_ARG;
        CK(alloc((void**)&c->kpfeat, nu * 9 * sizeof(float)));
        CK(alloc((void**)&c->kpc, nu * 25 * sizeof(float)));
        launch_precond_features(a, c->kA9, c->kpfeat, c->stream);
        CK(cnn_forward_on(c->kpc_net, c->kpfeat, c->kpc, nsys, c->stream));
        c->acc.kernel_launches += 1 + 4;
    }
    verb_krylov_stats st{};
    double guess_max = 0, res_max = 0;
    for (int k = 0; k < nsub; k++) {
        // the state the sub-step starts from, in the unknown order: the PSD
        // on the first sub-step, the previous sub-step's solution (kx) after
        double* fstate = c->kx;
        if (k == 0 && guess != VERB_GUESS_ZERO) {
            fstate = c->kd;
            launch_gather_state(a, fstate, c->stream);
            c->acc.kernel_launches++;
        }
        launch_local_rhs(a, k > 0, c->stream);
        CK(cudaMemcpyAsync(c->kb, c->lwork, nu * sizeof(double), cudaMemcpyDeviceToDevice,
                           c->stream));
        c->acc.kernel_launches++;
        if (guess == VERB_GUESS_ZERO) {
            CK(cudaMemsetAsync(c->kx, 0, nu * sizeof(double), c->stream));
        } else if (guess == VERB_GUESS_PREV) {
            launch_warm_start(a, fstate, nullptr, c->kscale, c->kx, c->stream);
            c->acc.kernel_launches++;
        } else {
            launch_local_features(a, fstate, c->kfeat, c->kscale, c->stream);
            CK(cnn_forward_on(cnn, c->kfeat, c->kout, nsys, c->stream));
            launch_warm_start(a, fstate, c->kout, c->kscale, c->kx, c->stream);
            c->acc.kernel_launches += 2 + 4;  // features, warm start, 4 conv layers
        }
        // smoothing sweeps damp the guess's high-frequency error, which the
        // stiff rows amplify in the residual
        for (int sw = 0; sw < smooth; sw++) {
            launch_local_residual(a, c->kb, c->kx, c->kr, c->stream);
            launch_jacobi_update(a, c->kA9, c->kr, c->kx, omega, c->stream);
            c->acc.kernel_launches += 2;
        }
        // outer passes: check, then correct the pending systems; a pass
        // that leaves a system's FP64 residual above a tenth of its previous
        // value sends the system to the LU
        unsigned int cnt[2] = {0, 0};
        int pass = 0;
        CK(cudaMemsetAsync(c->kprev, 0, nsys * sizeof(double), c->stream));
        CK(cudaMemsetAsync(c->kiters, 0, nsys * sizeof(int), c->stream));
        for (;; pass++) {
            CK(cudaMemsetAsync(c->kcount, 0, 2 * sizeof(unsigned int), c->stream));
            CK(cudaMemsetAsync(c->kmax, 0, sizeof(unsigned long long), c->stream));
            launch_residual_check(a, c->kb, c->kx, resid_tol, 0.1, c->kprev, c->kpend, c->kcount,
                                  c->kmax, c->stream);
            c->acc.kernel_launches++;
            unsigned long long key;
            CK(cudaMemcpyAsync(cnt, c->kcount, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaMemcpyAsync(&key, c->kmax, sizeof(key), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            const double rel = dkey_inv(key);
            if (pass == 0) guess_max = fmax(guess_max, rel);
            if (cnt[0] == 0 || pass == max_outer) {
                res_max = fmax(res_max, rel);
                break;
            }
            LocalArgs ap = a;
            ap.sel = c->kpend;
            ap.sel_mask = 1;
            launch_local_residual(ap, c->kb, c->kx, c->kr, c->stream);
            // the FP64 check decides convergence: no inner flag is kept
            launch_bicgstab(ap, c->kA9, c->kpc_net ? c->kpc : nullptr, c->kr, c->kd, c->kscr,
                            inner_maxit, (float)inner_tol,
                            c->kiters, nullptr, c->stream);
            launch_local_update(ap, c->kx, c->kd, c->kmax + 2, c->stream);
            c->acc.kernel_launches += 3;
        }
        st.outer_passes += pass;
        st.systems += nsys;
        const unsigned int nfall = cnt[0] + cnt[1];
        if (stats) {
            std::vector<int> it(nsys);
            std::vector<unsigned char> pe(nsys);
            CK(cudaMemcpyAsync(it.data(), c->kiters, nsys * sizeof(int), cudaMemcpyDeviceToHost,
                               c->stream));
            CK(cudaMemcpyAsync(pe.data(), c->kpend, nsys, cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            for (int q = 0; q < nsys; q++) {
                st.inner_iterations += it[q];
                if (!pe[q]) st.solved_iterations += it[q];
            }
        }
        if (nfall) {
            // LU for the systems still above the tolerance: the rhs is in
            // lwork; factor (those systems only) and solve in place, then
            // take their solutions into x
            LocalArgs ap = a;
            ap.sel = c->kpend;
            ap.sel_mask = 3;
            s = alloc_factors(c, ap);
            if (s) return s;
            const size_t nuf = c->local_unknowns;
            if (ap.factors32)
                CK(cudaMemsetAsync(c->Uf32, 0, nuf * c->kvp32 * sizeof(float), c->stream));
            else
                CK(cudaMemsetAsync(c->Uf, 0, nuf * c->kvp * sizeof(double), c->stream));
            c->acc.kernel_launches += launch_local_factor(ap, c->stream);
            launch_local_solve(ap, c->stream);
            c->acc.kernel_launches++;
            // the mixed form's FP64 refinement (FP32 factors), as in the LU step
            for (int it = 0; it < c->refine_iters; it++) {
                launch_local_residual(ap, c->kb, c->lwork, c->lres, c->stream);
                LocalArgs ar = ap;
                ar.work = c->lres;
                launch_local_solve(ar, c->stream);
                // the statistic reports the last correction of this call
                if (it == c->refine_iters - 1)
                    CK(cudaMemsetAsync(c->refine_red, 0, 2 * sizeof(unsigned long long),
                                       c->stream));
                launch_local_update(ap, c->lwork, c->lres, c->refine_red, c->stream);
                c->acc.kernel_launches += 3;
            }
            launch_masked_copy(ap, c->kx, c->lwork, c->stream);
            c->acc.kernel_launches++;
            c->local_dirty = true;  // the factors of the other systems are stale
            st.fallbacks += nfall;
        }
        CK(cudaMemcpyAsync(c->lwork, c->kx, nu * sizeof(double), cudaMemcpyDeviceToDevice,
                           c->stream));
    }
    launch_local_store(a, c->stream);
    c->acc.kernel_launches++;
    s = check_launch();
    if (s) return s;
    if (stats) {
        st.max_rel_residual = res_max;
        st.guess_rel_residual = guess_max;
        *stats = st;
    }
    return VERB_OK;
}

// A local LU step that also emits the CNN's training triples (see
// verb_local_triples).
int triples_run(verb_ctx* c, double dt, double sub_dt, float* feat, float* target)
{
    const Dims& d = c->d;
    if (d.V < 3 || d.K < 3 || c->trim_k0) return VERB_ERR_ARG;
    int nsub = (int)(dt / sub_dt);
    if (nsub < 1) nsub = 1;
    const double dts = dt / nsub;
    LocalArgs a{};
    int s = local_prepare(c, a, dts);
    if (s) return s;
    if (c->local_dirty || dts != c->local_dt) {
        s = local_factor(c, a);
        if (s) return s;
    }
    const size_t nu = c->local_unknowns;
    CK(krylov_buffers(c, false));
    for (int k = 0; k < nsub; k++) {
        const bool last = k == nsub - 1;
        if (last) {
            // the state this sub-step starts from (kb, unknown order)
            if (k == 0)
                launch_gather_state(a, c->kb, c->stream);
            else
                CK(cudaMemcpyAsync(c->kb, c->lwork, nu * sizeof(double),
                                   cudaMemcpyDeviceToDevice, c->stream));
            launch_local_features(a, c->kb, feat, c->kscale, c->stream);
        }
        launch_local_rhs(a, k > 0, c->stream);
        if (c->refine_iters > 0)
            CK(cudaMemcpyAsync(c->lrhs, c->lwork, nu * sizeof(double), cudaMemcpyDeviceToDevice,
                               c->stream));
        launch_local_solve(a, c->stream);
        // the solution the LU step itself would take: with refinement
        // configured, its FP64 refinement steps too
        for (int it = 0; it < c->refine_iters; it++) {
            launch_local_residual(a, c->lrhs, c->lwork, c->lres, c->stream);
            LocalArgs ar = a;
            ar.work = c->lres;
            launch_local_solve(ar, c->stream);
            if (last && it == c->refine_iters - 1)
                CK(cudaMemsetAsync(c->refine_red, 0, 2 * sizeof(unsigned long long), c->stream));
            launch_local_update(a, c->lwork, c->lres, c->refine_red, c->stream);
            c->acc.kernel_launches += 3;
        }
        if (last) launch_local_targets(a, c->kb, c->lwork, c->kscale, target, c->stream);
        c->acc.kernel_launches += last ? 5 : 2;
    }
    launch_local_store(a, c->stream);
    c->acc.kernel_launches++;
    return check_launch();
}

}  // namespace vctx

extern "C" {

int verb_local_krylov(verb_ctx* c, double dt, double sub_dt, int guess, verb_cnn* cnn,
                      int smooth, double omega, int max_outer, int inner_maxit, double inner_tol,
                      double resid_tol, verb_krylov_stats* stats)
{
    if (!c || !(dt > 0) || !(sub_dt > 0) || guess < VERB_GUESS_ZERO || guess > VERB_GUESS_CNN ||
        (guess == VERB_GUESS_CNN) != (cnn != nullptr) || smooth < 0 || !(omega > 0) ||
        !(omega < 2) || max_outer < 0 || inner_maxit < 1 || !(inner_tol > 0) || !(resid_tol > 0))
        return VERB_ERR_ARG;
    return krylov_run(c, dt, sub_dt, guess, cnn, smooth, omega, max_outer, inner_maxit, inner_tol,
                      resid_tol, stats);
}

int verb_local_triples(verb_ctx* c, double dt, double sub_dt, float* feat_dev, float* target_dev)
{
    if (!c || !(dt > 0) || !(sub_dt > 0) || !feat_dev || !target_dev) return VERB_ERR_ARG;
    return triples_run(c, dt, sub_dt, feat_dev, target_dev);
}

}  // extern "C"

extern "C" {

int verb_set_krylov_preconditioner(verb_ctx* c, verb_cnn* net)
{
    if (!c) return VERB_ERR_ARG;
    if (net) {
        int ci, co, H, W, mb;
        CK(cnn_shape(net, &ci, &co, &H, &W, &mb));
        if (ci != 9 || co != 25 || H != c->d.K || W != c->d.V || mb < c->d.P * c->d.R)
            return VERB_ERR_ARG;
    }
    c->kpc_net = net;
    return VERB_OK;
}

int verb_local_precond_inputs(verb_ctx* c, double dt, double sub_dt, float* feat_dev, float* A9_dev)
{
    if (!c || !feat_dev || !A9_dev || !(dt > 0) || !(sub_dt > 0)) return VERB_ERR_ARG;
    const Dims& d = c->d;
    if (d.V < 3 || d.K < 3 || c->trim_k0) return VERB_ERR_ARG;
    int nsub = (int)(dt / sub_dt);
    if (nsub < 1) nsub = 1;
    LocalArgs a{};
    int s = local_prepare(c, a, dt / nsub);
    if (s) return s;
    launch_local_assemble32(a, A9_dev, c->stream);
    launch_precond_features(a, A9_dev, feat_dev, c->stream);
    c->acc.kernel_launches += 2;
    CK(cudaStreamSynchronize(c->stream));
    return check_launch();
}

int verb_precond_loss_grad(const float* A9, const float* C, const float* Z, int nsys, int V, int K,
                           int nprobe, float* gC, float* loss_host, void* stream)
{
    if (!A9 || !C || !Z || !gC || nsys < 1 || V < 1 || K < 1 || nprobe < 1) return VERB_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float* loss = nullptr;
    CK(cudaMallocAsync((void**)&loss, sizeof(float), s));
    int st = cuda_ok(cudaMemsetAsync(loss, 0, sizeof(float), s));
    if (!st) st = launch_precond_grad(A9, C, Z, gC, loss, nsys, V, K, nprobe, s);
    float h = 0.f;
    if (!st) st = cuda_ok(cudaMemcpyAsync(&h, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    cudaFreeAsync(loss, s);
    if (!st) st = cuda_ok(cudaStreamSynchronize(s));
    if (!st) st = check_launch();
    if (loss_host) *loss_host = h;
    return st;
}

}  // extern "C"
