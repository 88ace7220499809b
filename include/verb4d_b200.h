/*
 * verb4d_b200 -- B200 (sm_100a) implementation of the VERB-4D operator-split
 * Fokker-Planck step behind a plain C ABI.
 *
 * Two layers:
 *
 *  1. A device-resident, batched context (verb_ctx).  It replaces the four
 *     per-slice OpenMP loops of the reference driver
 *       convection  src/VERB4D_Solver.cpp:851-978  -> verb_convection()
 *       radial      src/VERB4D_Solver.cpp:990-1070 -> verb_radial()
 *       local       src/VERB4D_Solver.cpp:1081-1216 -> verb_local()
 *       negatives   src/VERB4D_Solver.cpp:1218-1242 -> verb_negative_count()
 *       radial KF   src/VERB4D_Solver.cpp:1244-1253 -> verb_assimilate_radial()
 *     Fields are uploaded when the reference's UpdatableMatrix::update()
 *     reports a change (src/UpdatableMatrix.cpp:602); the LU factors of the
 *     local systems live in HBM (the LU_CACHING cache of
 *     src/VERB4D_Solver.cpp:340-365) and are refactored when DVV, DKK, DVK,
 *     G_local, Losses_local, the grids, the BC types or dt change.
 *
 *  2. Per-slice entry points with the argument meaning of the reference's
 *     routines (host pointers, one slice per call) for drop-in linking and
 *     parity tests.
 *
 * Array layouts are the reference's: 4-D fields are [P][R][V][K] doubles with
 * K fastest (src/Matrix.cpp:4211-4220); boundary arrays are 3-D as in
 * src/ReadInitialData.cpp:541-563: Pl/Pu [R][V][K], Rl/Ru and Ll/Lu
 * [P][V][K], Vl/Vu [P][R][K], Kl/Ku [P][R][V].  Boundary-condition type codes
 * are those of src/BoundaryConditionType.hpp:53-88 (0 Periodic,
 * 1 ConstantValue, 2 ConstantDerivative).
 *
 * Errors: every call returns a verb_status.  Where the reference calls
 * exit(EXIT_FAILURE) (LAPACK info, Courant check, unknown BC, diffusion
 * tensor check) this library returns the matching code instead; kernels
 * record the first device-side error in a status word that verb_sync()
 * returns.  No kernel traps.
 */
#ifndef VERB4D_B200_H
#define VERB4D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    VERB_OK = 0,
    VERB_ERR_PIVOT = 1,   /* exactly singular pivot (LAPACK info != 0, src/MatrixSolver.cpp:273-276) */
    VERB_ERR_ARG = 2,     /* bad argument / unsupported size */
    VERB_ERR_CFL = 3,     /* Courant number > 1 (src/Convection_1D_ULTIMATE_QUICKEST6.cpp:48-52) */
    VERB_ERR_BC = 4,      /* unsupported boundary-condition type for this operator */
    VERB_ERR_TENSOR = 5,  /* min(DVV*DKK - DVK^2) < 0 (src/VERB4D_Solver.cpp:747-753) */
    VERB_ERR_NAN = 6,     /* NaN after the Kalman update (src/DataAssimilation.cpp:62-67),
                             or a NaN in the PSD after a step (no counterpart) */
    VERB_ERR_CUDA = 7,    /* CUDA runtime error */
    VERB_ERR_NOMEM = 8,   /* device allocation failed / would not fit */
    VERB_ERR_GRID = 9,    /* convection line shorter than 11 points (QUICKEST6.cpp:56-59) */
    VERB_TIMEOUT = 10,    /* a bounded device wait gave up */
    VERB_ERR_SIZE = 11,   /* size beyond a fixed limit (the no-allocation scratch, line
                             length, component count) or a file of other dimensions */
    VERB_ERR_IO = 12      /* a file could not be opened, read or written */
} verb_status;

enum { VERB_BC_PERIODIC = 0, VERB_BC_CONSTANT_VALUE = 1, VERB_BC_CONSTANT_DERIVATIVE = 2 };

/* 4-D fields of the context (names of src/VERB4D_Solver.cpp:210-245). */
typedef enum {
    VERB_F_PSD = 0,
    VERB_F_P, VERB_F_R, VERB_F_V, VERB_F_K, VERB_F_L,
    VERB_F_DLL, VERB_F_DVV, VERB_F_DKK, VERB_F_DVK,
    VERB_F_VP, VERB_F_VR,
    VERB_F_G_LOCAL, VERB_F_G_RADIAL, VERB_F_G_CONV,
    VERB_F_SOURCES, VERB_F_LOSS_LOCAL, VERB_F_LOSS_RADIAL, VERB_F_LOSS_CONV,
    VERB_F_COUNT
} verb_field;

/* 3-D boundary arrays. */
typedef enum {
    VERB_BCF_PL = 0, VERB_BCF_PU, VERB_BCF_RL, VERB_BCF_RU, VERB_BCF_LL, VERB_BCF_LU,
    VERB_BCF_VL, VERB_BCF_VU, VERB_BCF_KL, VERB_BCF_KU, VERB_BCF_COUNT
} verb_bc_field;

typedef struct verb_ctx verb_ctx;

/* Phase timings (milliseconds, CUDA events on the context stream), filled when
 * timing is enabled with verb_set_timing(ctx, 1). */
typedef struct {
    double convection_ms, radial_ms, radial_factor_ms, local_ms, local_factor_ms,
        local_solve_ms, reduce_ms, kf_ms;
    long long steps, local_solve_launches, local_factor_launches;
    long long kernel_launches;  /* every kernel this context launched since timing was enabled */
} verb_timing;

/* ---- context lifetime ---------------------------------------------------- */
/* stream: a cudaStream_t (NULL = the context creates its own). */
int verb_create(verb_ctx** out, int P, int R, int V, int K, void* stream);
int verb_destroy(verb_ctx* ctx);
int verb_device_bytes(const verb_ctx* ctx, size_t* bytes);

/* ---- inputs (UpdatableMatrix::update() == true  ->  upload) --------------- */
int verb_upload_field(verb_ctx* ctx, int field, const double* host);      /* host [P][R][V][K] */
int verb_upload_field_device(verb_ctx* ctx, int field, const double* dev);/* device pointer */
/* Scale factor applied on the device as field = base * scale, the reference's
 * UpdatableMatrix scale queue (src/UpdatableMatrix.cpp:698-708).  Default 1. */
int verb_set_field_scale(verb_ctx* ctx, int field, double scale);
int verb_upload_bc(verb_ctx* ctx, int bc_field, const double* host);
/* types[10] in verb_bc_field order (Pl,Pu,Rl,Ru,Ll,Lu,Vl,Vu,Kl,Ku). */
int verb_set_bc_types(verb_ctx* ctx, const int* types);
/* Source/loss routing of src/VERB4D_Solver.cpp:404-426 and the include_boundary
 * / positive_PSD switches of src/ReadInitialData.cpp:214-230. */
int verb_set_options(verb_ctx* ctx, int radial_sources, int local_sources, int include_boundary,
                     int positive_psd);
/* Force the local LU factors to be recomputed at the next verb_local(). */
int verb_invalidate_lu(verb_ctx* ctx);
/* Precision of the local (V,K) solve.  VERB_PREC_FP64 (default): the LU
 * factors are kept in FP64, as LAPACK's dgbtrf leaves them
 * (src/MatrixSolver.cpp:223-340, cached as in src/VERB4D_Solver.cpp:340-365).
 * VERB_PREC_MIXED: the same factorisation (FP64 arithmetic, the same pivots)
 * is stored in FP32, which halves the factor cache and the bytes every solve
 * streams.  With refinements > 0 (either form) each solve is followed by that
 * many steps of FP64 iterative refinement: r = b - A x with A assembled in
 * FP64, A d = r with the cached factors, x += d.  FP64 with 0 refinements is
 * the reference's arithmetic; every other setting has no counterpart in the
 * reference.  Changing the form frees the other form's factors and refactors
 * at the next verb_local(). */
#define VERB_PREC_FP64 0
#define VERB_PREC_MIXED 1
int verb_set_local_precision(verb_ctx* ctx, int mode, int refinements);
/* Ragged local systems (the batched form of the loss-cone trimmed local
 * diffusion; no counterpart in the reference): system (p, r), index p*R + r,
 * keeps pitch-angle indices k0[p*R + r] .. K-1 and is the Diffusion_2D system
 * of that sub-grid (src/Diffusion_2D.cpp:19-153) with a ConstantValue 0
 * boundary at its lower pitch-angle edge; PSD below the edge is left as it
 * is, and systems with fewer than 3 pitch angles are not solved.  Factor
 * storage shrinks with the trimmed unknowns.  nullptr restores full systems.
 * Local pivots / LAPACK-layout factors are not available while trimmed. */
int verb_set_local_trim(verb_ctx* ctx, const int* k0_host);
/* max |d| / max |x| of the last refinement step of the last verb_local()
 * (0 without refinement). */
int verb_local_refinement(verb_ctx* ctx, double* rel_correction);
int verb_download_psd(verb_ctx* ctx, double* host);
int verb_download_field(verb_ctx* ctx, int field, double* host);
/* Device pointer of a field (for zero-copy use from the caller's CUDA code). */
int verb_field_device_ptr(verb_ctx* ctx, int field, double** dev);

/* ---- updatable input fields -------------------------------------------------
 * The reference's UpdatableMatrix / UpdatableListMatrix time-update system
 * (src/UpdatableMatrix.cpp:602-846, 913-961) on the device.  A field (D_LL
 * .. the loss rates) becomes a list of components; each has a base array and
 * time-ordered queues of replacement arrays (the .lst data files), scale
 * factors and from/to limits per grid axis (0 MLT, 1 R, or L* for D_LL, 2 V,
 * 3 K; `which` 0 = from, 1 = to).  verb_update_fields(t) pops every entry due
 * at t as update() does, rebuilds the changed fields on the device (component
 * = base * scale, zeroed outside the limits; field = sum, or mean over finite
 * component values) and marks the cached LU / Thomas factors for
 * recomputation as the driver does (src/VERB4D_Solver.cpp:1091-1096).
 * Replacement arrays are copied to the device when queued.  A field with
 * components cannot also be uploaded or scaled directly. */
#define VERB_MERGE_SUM 0
#define VERB_MERGE_MEAN 1
int verb_field_add_component(verb_ctx* ctx, int field, const double* host_base, int* component);
int verb_field_set_merge(verb_ctx* ctx, int field, int merge);
int verb_component_queue_data(verb_ctx* ctx, int field, int component, double time,
                              const double* host);
int verb_component_queue_scale(verb_ctx* ctx, int field, int component, double time, double scale);
int verb_component_queue_limit(verb_ctx* ctx, int field, int component, int axis, int which,
                               double time, double value);
/* updated_mask: bit f set when field f was rebuilt. */
int verb_update_fields(verb_ctx* ctx, double current_time, unsigned int* updated_mask);

/* L* remapping (src/VERB4D_Solver.cpp:557-619): interpolate every (P,V,K)
 * line of the PSD from the current L* field to new_L_host ([P][R][V][K],
 * strictly increasing along R) with the reference's monotone cubic
 * interpolator (Opm::MonotCubicInterpolator), then make new_L the L* field.
 * The reference's Cubic1D wrapper (src/Interpolation.cpp:26-51) builds its
 * point vectors after reserving them (n zero points precede the grid) and
 * returns an empty matrix that the caller assigns over the result, so its
 * output is undefined; this entry point interpolates the line as the
 * wrapper's documentation describes.  Jacobians that depend on L* are
 * updated by the caller, as the reference's driver does (:563-565). */
int verb_remap_L(verb_ctx* ctx, const double* new_L_host);

/* Device bytes a context of this size will need once it has run a step
 * (fields, boundary arrays, cached radial and local factors in the given
 * precision, convection scratch, and Kalman-filter covariances of kf_columns
 * columns).  Allocates nothing; used to admit ensemble members within an HBM
 * budget.  No counterpart in the reference. */
int verb_estimate_device_bytes(int P, int R, int V, int K, int precision, int refinements,
                               long long kf_columns, size_t* bytes);

/* ---- learned warm start -----------------------------------------------------
 * A small CNN of 3x3 convolutions (zero padding, ReLU between layers, FP16
 * weights, FP32 accumulation) with hand-written forward, backward and Adam
 * kernels.  It is trained on (coefficient fields, right-hand side, solution)
 * triples of the local (V,K) systems and gives the warm start of their
 * Krylov solve (verb_local_krylov).  No counterpart in the reference.
 * channels[0..layers] are the channel counts (input first); images are
 * H x W; tensors are device NCHW FP32.  Parameters are ordered layer by
 * layer: weights [Cout][Cin][3][3], then bias [Cout]. */
typedef struct verb_cnn verb_cnn;
int verb_cnn_create(verb_cnn** out, int layers, const int* channels, int H, int W, int max_batch,
                    void* stream);
int verb_cnn_destroy(verb_cnn* cnn);
int verb_cnn_param_count(const verb_cnn* cnn, long long* count);
int verb_cnn_set_params(verb_cnn* cnn, const float* host);
/* grad_host (may be NULL) receives the gradients of the last training step */
int verb_cnn_get_params(verb_cnn* cnn, float* host, float* grad_host);
int verb_cnn_forward(verb_cnn* cnn, const float* in_dev, float* out_dev, int batch);
/* MSE loss against target_dev, backward pass, Adam step (lr <= 0: gradients only) */
int verb_cnn_train_step(verb_cnn* cnn, const float* in_dev, const float* target_dev, int batch,
                        float lr, float* loss_host);
/* Backward pass and Adam step (lr <= 0: gradients only) for an output
 * gradient the caller computed (grad_out_dev, the network output's shape),
 * through the activations of the last verb_cnn_forward, which must have run
 * on in_dev with the same batch. */
int verb_cnn_backward_step(verb_cnn* cnn, const float* in_dev, const float* grad_out_dev, int batch,
                           float lr);

/* ---- convection data assimilation ------------------------------------------
 * runKalmanFilterConvection2D (src/DataAssimilationConvection.cpp:124-253)
 * on every (V,K) slice, as DataAssimilationManagerConvection::assimilate
 * (:45-121) calls it from the driver (src/VERB4D_Solver.cpp:1246): the state
 * is the slice's N = P*R PSD values, the model matrix is the upwind transport
 * operator of the step raised to its Courant split count (cached per slice
 * until has_vx_updated), the loss rate is the Sources field over the PSD (the
 * driver's argument), no saturation map.  obs_host is a [P][R][V][K] field
 * with NaN where there is no observation.  Pa and the model matrices
 * (2 N^2 doubles per slice) persist in the context; slice_chunk bounds the
 * slices processed together (0: chunks of about 4 GB of work space).
 * Deviation: a slice without observations keeps its PSD and takes Pa = Pf;
 * the reference's dummy observation row (H = 0, y = 0) makes the linear
 * form's innovation matrix singular (trans_solve exits) and the log form's
 * innovation log(0) (the NaN check throws). */
int verb_assimilate_convection(verb_ctx* ctx, const double* obs_host, double dt, double model_error,
                               double obs_error, int use_log, double correlation_time,
                               int growing_q, int has_vx_updated, int slice_chunk);
/* Pa (N x N) and the cached model matrix of slice (v, k); either may be NULL. */
int verb_convection_da_state(verb_ctx* ctx, int v, int k, double* Pa_host, double* model_host);

/* ---- autotuner ---------------------------------------------------------------
 * The local solve comes in verb_local_solve_variants() shapes: systems (warps)
 * per CTA and L / U factor columns in flight per warp.  Deeper factor rings
 * hide more memory latency per system but leave shared memory for fewer
 * resident systems, so the best shape depends on the grid and the factor
 * precision.  verb_autotune_local_solve factorises if needed, forms the first
 * sub-step's right-hand sides and times every shape on them (best of three,
 * CUDA events on the context's stream; the PSD is not changed), then uses the
 * fastest for this context and for later contexts of the same (P, R, V, K,
 * precision, ragged) in the process.  times_ms (may be NULL) receives one
 * entry per shape.  All shapes give identical results.  No counterpart in the
 * reference. */
int verb_local_solve_variants(int* count);
int verb_local_solve_variant(int v, int* warps_per_cta, int* l_columns, int* u_columns);
/* 1 when shape v keeps the right-hand-side window of the substitutions in
 * registers (the factor columns still stream through shared memory), 0 when
 * the window lives in shared memory.  Bands wider than the register window
 * holds (V > 126) fall back to the shared-memory window. */
int verb_local_solve_variant_window(int v, int* in_registers);
/* v = -1: the shape tuned for this context's shape in this process (else 0) */
int verb_set_local_solve_variant(verb_ctx* ctx, int v);
int verb_autotune_local_solve(verb_ctx* ctx, double dt, double sub_dt, double* times_ms,
                              int* chosen);

/* Convection arithmetic.  VERB_CONV_EXACT (the default) restates the
 * reference's operations one by one without contraction, so results are
 * bit-identical to it (exp() of loss rates aside).  VERB_CONV_FMA runs the
 * same kernel compiled with multiply-add contraction (and nine warps per
 * block): about 18 % faster, and within a few units in the last place of the
 * exact form per step.  VERB_CONV_STREAM runs one thread per line through all
 * four stages of a pass at once (register windows, nothing staged between
 * stages), contracted, with the G product and the loss/source epilogue
 * applied as the sweeps store; it needs both sweeps (P and R >= 11) and
 * otherwise runs the VERB_CONV_FMA kernel; within a few units in the last
 * place of the reference per step.  Convection_2D
 * (src/Convection_2D.cpp:36-169) has one arithmetic; the switch has no
 * counterpart in the reference. */
#define VERB_CONV_EXACT 0
#define VERB_CONV_FMA 1
#define VERB_CONV_STREAM 2
int verb_set_convection_arith(verb_ctx* ctx, int mode);

/* ---- Krylov form of the local (V,K) solve ----------------------------------
 * verb_local_krylov takes the same local step as verb_local but solves each
 * (P,R) system by iterative refinement in FP64 around an FP32 BiCGSTAB with
 * a Jacobi (diagonal) preconditioner, one CTA per system, starting from
 * x0 = 0 (VERB_GUESS_ZERO), x0 = f (VERB_GUESS_PREV: the state the step
 * starts from) or the CNN's prediction x0 = f + max|f| * cnn(features)
 * (VERB_GUESS_CNN), followed by `smooth` weighted-Jacobi sweeps
 * x += omega (b - A x) / diag(A) in FP64.  Each outer pass forms r = b - A x in FP64, solves
 * A d = r to inner_tol in FP32 (at most inner_maxit iterations) and adds d.
 * A system is done when max|b - A x| / max|b| <= resid_tol; systems still
 * above it after max_outer passes, or whose residual a pass did not reduce
 * at least tenfold, are solved by the banded LU (in the mixed form: FP32
 * factors and the form's FP64 refinement steps) (factorised
 * for those systems only; the factors are allocated on first use) so the
 * step is always accurate to the residual tolerance or exact.  The features
 * are [sys][4][K][V] FP32: (log10 D_VV - m)/2, (log10 D_KK - m)/2 with
 * m = log10(0.864), D_VK / sqrt(D_VV D_KK) and f / max|f|; the network's
 * output is the step's relative increment (x - f) / max|f| on the same grid.
 * (The system's right-hand side is not a guess: its interior rows are
 * scaled by 1/dt.)  The CNN form needs untrimmed systems.  No counterpart in
 * the reference (its local step is the LU). */
#define VERB_GUESS_ZERO 0
#define VERB_GUESS_PREV 1
#define VERB_GUESS_CNN 2
typedef struct {
    long long systems;           /* systems solved (per sub-step, summed) */
    long long fallbacks;         /* systems finished by the LU */
    long long inner_iterations;  /* BiCGSTAB iterations over all systems */
    long long solved_iterations; /* ... over the systems the Krylov solve finished */
    long long outer_passes;      /* refinement passes taken (max over sub-steps, summed) */
    double max_rel_residual;     /* largest max|b-Ax|/max|b| before the fallback */
    double guess_rel_residual;   /* largest relative residual of the initial guess */
} verb_krylov_stats;
int verb_local_krylov(verb_ctx* ctx, double dt, double sub_dt, int guess, verb_cnn* cnn,
                      int smooth, double omega, int max_outer, int inner_maxit, double inner_tol,
                      double resid_tol, verb_krylov_stats* stats);
/* Learned preconditioner of the Krylov form (no counterpart in the reference):
 * a CNN with 9 input channels and 25 output channels on the K x V grid of a
 * local system predicts, for every unknown i, the 25 coefficients C[o](i) of
 * a sparse approximate inverse on its 5 x 5 neighbourhood o,
 *   M v (i) = sum_o (delta(o = 0) + C[o](i)) v(i + o) / diag(i + o),
 * which replaces the Jacobi preconditioner of the BiCGSTAB in
 * verb_local_krylov (C = 0 is Jacobi).  Its inputs are the system's matrix:
 * log10(|diag| dt) and the eight off-diagonal entries of each row over the
 * diagonal, [sys][9][K][V] (verb_local_precond_inputs, which also returns the
 * FP32 diagonals [sys][9][V*K]).  verb_precond_loss_grad gives its training
 * signal: for nprobe probe vectors z per system ([sys][nprobe][V*K]) the loss
 * mean |D^-1 A M D z - z|^2 on the Jacobi-scaled system (D = diag(A), so
 * every row counts alike) and its gradient with respect to C
 * ([sys][25][V*K]), to pass to verb_cnn_backward_step.  net = NULL restores Jacobi.  The context
 * keeps the pointer: the network must outlive its use. */
int verb_set_krylov_preconditioner(verb_ctx* ctx, verb_cnn* net);
int verb_local_precond_inputs(verb_ctx* ctx, double dt, double sub_dt, float* feat_dev,
                              float* A9_dev);
int verb_precond_loss_grad(const float* A9_dev, const float* C_dev, const float* Z_dev, int nsys,
                           int V, int K, int nprobe, float* gC_dev, float* loss_host, void* stream);
/* One local step by the LU (as verb_local, with its refinement steps) that also
 * writes, for the last sub-step, the CNN features of every system
 * (feat_dev, [P*R][4][K][V] floats) and the training target
 * (target_dev, [P*R][K][V] floats, (x - f) / max|f|).  Untrimmed systems only;
 * skipped (boundary) systems are left unwritten. */
int verb_local_triples(verb_ctx* ctx, double dt, double sub_dt, float* feat_dev, float* target_dev);

/* ---- output and restart files ----------------------------------------------
 * .pltb files as the reference writes and reads them (Matrix4D::
 * writeToBinaryFile / readFromBinaryFile, src/Matrix.cpp:5700-5720,
 * 5780-5808): four int32 sizes (P, R, V, K), then the values.  A write takes a
 * device snapshot of the field on the context stream and returns; the copy to
 * pinned host memory runs on an output stream and a host thread writes the
 * file, as the reference's asynchronous output_writer does
 * (src/VERB4D_Solver.cpp:1255-1267).  One write is in flight at a time (the
 * next write waits for it); verb_output_wait joins it and returns its status.
 * Restart: read the PSD file back into VERB_F_PSD and continue from its time
 * (the reference's initial_PSD / time_first / it_first,
 * src/ReadInitialData.cpp:207-208). */
int verb_write_field_pltb(verb_ctx* ctx, int field, const char* path, int async_write);
int verb_output_wait(verb_ctx* ctx);
int verb_read_field_pltb(verb_ctx* ctx, int field, const char* path);
/* Append "time<TAB>filename" to a PSD.lst list (Matrix4D::writeToLstFile,
 * src/Matrix.cpp:5760-5778; time printed with 5 decimals). */
int verb_append_lst(const char* lst_path, double time, const char* filename);

/* ---- the step ------------------------------------------------------------ */
/* Convection_2D over every (V,K) slice (src/Convection_2D.cpp:36-169). */
int verb_convection(verb_ctx* ctx, double dt);
/* Diffusion_1D over every (P,V,K) line (src/Diffusion_1D.cpp:43-88). */
int verb_radial(verb_ctx* ctx, double dt);
/* Diffusion_2D + Lapack over every (P,R) system with cached factors
 * (src/Diffusion_2D.cpp:19-153, src/MatrixSolver.cpp:223-340). */
int verb_local(verb_ctx* ctx, double dt, double sub_dt);
/* max(PSD, 1e-21) (src/VERB4D_Solver.cpp:621). */
int verb_clamp_positive(verb_ctx* ctx);
/* Whole step in the reference order: tensor check, convection, radial, local,
 * negative count (src/VERB4D_Solver.cpp:747-1242).  run_* select the phases. */
int verb_step(verb_ctx* ctx, double dt, double sub_dt, int run_convection, int run_radial,
              int run_local, long long* negative_count);
/* Replay steps from a CUDA graph: the launches of a steady-state step (no
 * factorisation, allocation or phase timing) are captured on first use and
 * replayed while dt, sub_dt, the phase flags and every launch argument stay
 * the same; uploads of fields other than the PSD, scales, boundary types,
 * options and forms drop the graph, and the next such step captures it again.
 * Results are identical to eager steps.  Off by default.  No counterpart in
 * the reference (its time loop, src/VERB4D_Solver.cpp:747-1282, runs on the
 * host). */
int verb_set_step_graph(verb_ctx* ctx, int enable);
/* Number of PSD points < 0 (src/VERB4D_Solver.cpp:1226-1240). */
int verb_negative_count(verb_ctx* ctx, long long* count);
/* min(DVV*DKK - DVK*DVK) over the grid (src/VERB4D_Solver.cpp:747-753). */
int verb_tensor_check(verb_ctx* ctx, double* min_value);
/* max |field| of n <= 8 fields (verb_field codes) in one pass over the grid:
 * the per-step log of src/VERB4D_Solver.cpp:636-675 (VP, VR, DLL, DVV, DVK,
 * DKK after their update; DLL with its scale factor applied), with
 * Matrix4D::maxabs's semantics (src/Matrix.cpp:5908-5915: NaN values are
 * skipped, -inf for an empty grid).  Every listed field must have been
 * uploaded. */
int verb_field_maxabs(verb_ctx* ctx, int n, const int* fields, double* out);
/* Wait for the context stream; returns the first device-side error. */
int verb_sync(verb_ctx* ctx);
int verb_set_timing(verb_ctx* ctx, int enable);
int verb_get_timing(verb_ctx* ctx, verb_timing* out);
/* Slice-level convection sub-step counts of the last verb_convection()
 * ([V][K] ints, src/Convection_2D.cpp:57-86). */
int verb_convection_substeps(verb_ctx* ctx, int* host_vk);
/* Local LU pivots (0-based, [P][R][V*K] int32) and one system's factors in
 * LAPACK band layout (ldab = 3*(V+1)+1 rows, column-major, as dgbtrf leaves
 * them) for parity checks and LU-cache hand-off. */
int verb_local_pivots(verb_ctx* ctx, int32_t* host);
int verb_local_factor_lapack(verb_ctx* ctx, int p, int r, double* ab_host, long* ipiv1_host);
/* (FP64 form only: VERB_ERR_ARG when the factors are held in FP32.) */

/* ---- radial Kalman filter ------------------------------------------------ */
/* One assimilation update of every (P,V,K) radial column (the reference
 * applies it at P index 0 only: src/DataAssimilationDiffusion.cpp:116,139;
 * p_index >= 0 restricts it the same way, -1 runs all P).  obs is a host
 * [P][R][V][K] array with NaN where there is no observation.  The analysis
 * covariances live on the device, initialised to 5*model_error*I on first use
 * (src/DataAssimilationDiffusion.cpp:212-218).
 * The covariances are held for the columns in use (one MLT for p_index >= 0,
 * all for -1); later calls must pass the first call's p_index. */
int verb_assimilate_radial(verb_ctx* ctx, const double* obs_host, double dt, double model_error,
                           double obs_error, int p_index);

/* ---- per-slice entry points (host pointers, one slice per call) ----------- */
/* tridag, src/MatrixSolver.cpp:689-720 (a,b,c,r,u of length n). */
int verb_tridag(const double* a, const double* b, const double* c, const double* r, double* u,
                long n);
/* Diffusion_1D, src/Diffusion_1D.cpp:43-88 (psd updated in place). */
int verb_diffusion_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                      int ubc_t, const double* D, const double* G, const double* S,
                      const double* loss, double dt);
/* Diffusion_2D (LU_CACHING form), src/Diffusion_2D.cpp:20-153: psd,x,y,D*,G,S,loss
 * are [nx][ny]; xl/xu have ny entries, yl/yu nx.  lu_cache (ldab*nx*ny doubles,
 * LAPACK band layout) and index_cache (nx*ny longs, 1-based) are the caller's
 * cache slot: written when recompute_lu != 0, read otherwise.  Both may be
 * NULL, which factors every call (the plain build). */
int verb_diffusion_2d(double* psd, const double* x, const double* y, int nx, int ny,
                      const double* xl, const double* xu, const double* yl, const double* yu,
                      int xl_t, int xu_t, int yl_t, int yu_t, const double* Dxx, const double* Dyy,
                      const double* Dxy, const double* Dyx, const double* G, const double* S,
                      const double* loss, double dt, double sub_dt, double* lu_cache,
                      long* index_cache, int recompute_lu);
/* Convection_1D_ULTIMATE_QUICKEST6, src/Convection_1D_ULTIMATE_QUICKEST6.cpp:22. */
int verb_convection_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                       int ubc_t, const double* ux, double dt);
/* Convection_2D, src/Convection_2D.cpp:36 on one [P][R] slice. */
int verb_convection_2d(double* psd, const double* P, const double* R, int nP, int nR,
                       const double* pl, const double* pu, const double* rl, const double* ru,
                       int pl_t, int pu_t, int rl_t, int ru_t, const double* VP, const double* VR,
                       const double* S, const double* loss, const double* G, double dt);

/* ---- no-allocation entry point ---------------------------------------------- */
/* No counterpart in the reference.  Convection_2D on one [P][R] slice whose
 * arrays (same meaning and layout as verb_convection_2d) already live in the
 * caller's DEVICE memory, for callers that cannot allocate device memory (a
 * host application or plugin that owns every allocation, or a path where an
 * allocation is not allowed).  It calls no allocator: the kernel's scratch is
 * a fixed array in the library's device code of 5 doubles per point of
 * VERB_NOALLOC_MAX_POINTS points (320 KiB) plus a few status words, held on
 * every device that loads that code until exit.  CUDA loads device code
 * lazily, so the first call on a device loads it (the array and the kernel
 * take their device memory then, and the device may synchronise) and looks
 * up the array's address: make that first call outside any region where
 * allocation is not allowed, and before any stream capture.
 * nP*nR > VERB_NOALLOC_MAX_POINTS returns VERB_ERR_SIZE.  All calls share that
 * array, so calls that overlap on the GPU race: serialise them.  `stream` is
 * a cudaStream_t (NULL = default stream); the call returns after the slice is
 * done, with the device-side status (e.g. VERB_ERR_CFL, the slice then left
 * unchanged) or VERB_ERR_CUDA for a failure of its own launch; an error left
 * pending by the caller's earlier CUDA work is not reported or cleared. */
#define VERB_NOALLOC_MAX_POINTS 8192
int verb_convection_2d_noalloc(double* psd, const double* P, const double* R, int nP, int nR,
                               const double* pl, const double* pu, const double* rl,
                               const double* ru, int pl_t, int pu_t, int rl_t, int ru_t,
                               const double* VP, const double* VR, const double* S,
                               const double* loss, const double* G, double dt, void* stream);

/* ---- library information --------------------------------------------------- */
const char* verb_version(void);
const char* verb_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif /* VERB4D_B200_H */
