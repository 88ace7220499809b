// The device-resident context (struct verb_ctx) and the helpers shared by
// its source files (ctx.cu: lifetime, uploads, phases, step; ctx_krylov.cu:
// the Krylov form of the local solve; ctx_assim.cu: the convection
// assimilation).  Private to the library.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <tuple>
#include <new>
#include <string>
#include <thread>
#include <algorithm>
#include <utility>
#include <vector>

#include "verb_internal.cuh"

using namespace verb;

namespace vctx {

enum Phase { PH_CONV = 0, PH_RAD, PH_RADF, PH_LOCAL, PH_LOCF, PH_LOCS, PH_RED, PH_KF, PH_N };

struct EventPair {
    cudaEvent_t a, b;
};

}  // namespace vctx
using vctx::EventPair;
using vctx::PH_N;

// One component of an updatable field (src/UpdatableMatrix.h:60-90): base
// array, queued replacement arrays, scale and limit queues.
struct UpdComponent {
    double* base = nullptr;
    std::deque<std::pair<double, double*>> data_q;           // (time, device array)
    std::deque<std::pair<double, double>> scale_q;
    std::deque<std::pair<double, double>> limit_q[4][2];     // [axis][from, to]
    double scale = 1.0;                                       // latest_scale_coefficient
    double lim[4][2] = {{-1e99, 1e99}, {-1e99, 1e99}, {-1e99, 1e99}, {-1e99, 1e99}};
    double last_update_time = -1;
};
struct UpdField {
    std::vector<UpdComponent> comps;
    int merge = VERB_MERGE_SUM;
    bool built = false;
};

struct verb_ctx {
    Dims d{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double* f[VERB_F_COUNT] = {};
    double* fbase[VERB_F_COUNT] = {};   // unscaled copy when a scale != 1 is set
    double scale[VERB_F_COUNT];
    bool uploaded[VERB_F_COUNT] = {};
    double* bc[VERB_BCF_COUNT] = {};
    int bct[VERB_BCF_COUNT];
    int radial_sources = 0, local_sources = 1, include_boundary = 1, positive_psd = 0;
    // radial Thomas factors
    double *rfa = nullptr, *rfbet = nullptr, *rfgam = nullptr;
    bool radial_dirty = true;
    double radial_dt = -1;
    // local LU factors
    double *Lf = nullptr, *Uf = nullptr, *lwork = nullptr;
    int32_t* ipiv = nullptr;
    int kl = 0, kv = 0, klp = 0, kvp = 0;
    // mixed-precision form: FP32 factors, FP64 refinement (rhs copy, residual)
    int local_prec = VERB_PREC_FP64, refine_iters = 0;
    float *Lf32 = nullptr, *Uf32 = nullptr;
    int klp32 = 0, kvp32 = 0;
    double *lrhs = nullptr, *lres = nullptr;
    unsigned long long* refine_red = nullptr;  // max |last correction|, max |x|
    // ragged (trimmed) local systems: first pitch-angle index per (P,R)
    // system and the first unknown of each system
    int* trim_k0 = nullptr;
    long long* trim_uoff = nullptr;
    size_t local_unknowns = 0;  // unknowns of all systems (trimmed or full)
    // convection data assimilation: per (V,K) slice the model matrix cache
    // and Pa (N x N, N = P*R); chunk work space (4 N x N per slice), vectors
    // (t, x, y) and integer lists
    double *kc_M = nullptr, *kc_Pa = nullptr, *kc_W = nullptr, *kc_vec = nullptr;
    int* kc_int = nullptr;
    bool kc_valid = false;
    int kc_chunk = 0;
    // Krylov form: FP32 diagonals and BiCGSTAB vectors, FP64 b / x / r / d,
    // CNN features and output, per-system scale, iterations, pending flags
    float *kA9 = nullptr, *kscr = nullptr, *kfeat = nullptr, *kout = nullptr;
    double *kb = nullptr, *kx = nullptr, *kr = nullptr, *kd = nullptr, *kscale = nullptr;
    double* kprev = nullptr;              // previous relative residual per system
    int* kiters = nullptr;
    unsigned char* kpend = nullptr;
    unsigned int* kcount = nullptr;       // [0] pending systems, [1] given up
    unsigned long long* kmax = nullptr;   // [0] max relative residual key, [2..3] update maxima
    // learned preconditioner of the Krylov form: the network, its features
    // [sys][9][n] and coefficients [sys][25][n]
    verb_cnn* kpc_net = nullptr;
    float *kpfeat = nullptr, *kpc = nullptr;
    bool local_dirty = true;
    double local_dt = -1;
    int solve_variant = -1;  // local solve shape; -1: the process-wide tuned one, else 0
    const double* dkv_override = nullptr;  // Dyx for the per-slice entry point
    // convection
    double* conv_scratch = nullptr;
    int* conv_substeps = nullptr;
    int* ticket = nullptr;
    int conv_nctas = 0;
    size_t conv_scratch_bytes = 0;  // for every arithmetic mode's kernel
    int conv_arith = VERB_CONV_EXACT;
    // reductions / status
    unsigned long long* red = nullptr;  // [0] negatives, [1] tensor min key
    unsigned long long* maxabs_red = nullptr;  // [MAXABS_FIELDS] max |field| keys
    int* status = nullptr;
    bool tensor_dirty = true;
    double tensor_min = 0;
    // Kalman filter
    double *Pa = nullptr, *kfwork = nullptr, *obs = nullptr;
    size_t kfwork_bytes = 0;
    int* kfticket = nullptr;
    int pa_p_index = -2;  // the p_index Pa was sized for (-2: not yet)
    // updatable fields (nullptr: plain uploaded field)
    UpdField* upd[VERB_F_COUNT] = {};
    // asynchronous output: device snapshot -> pinned host copy on a copy
    // stream -> file written by a host thread
    double* out_snap = nullptr;
    double* out_host = nullptr;
    cudaStream_t out_stream = nullptr;
    cudaEvent_t out_ev_snap = nullptr, out_ev_host = nullptr;
    std::thread out_thread;
    int out_status = VERB_OK;
    // CUDA graph of the steady-state step (captured on first use, replayed
    // while nothing the step's launches depend on changes)
    bool use_graph = false;
    bool graph_valid = false;
    cudaGraphExec_t step_exec = nullptr;
    double g_dt = 0, g_sub_dt = 0;
    int g_flags = 0;
    long long g_launches = 0;
    // timing
    bool timing = false;
    std::vector<EventPair> ev[PH_N];
    std::vector<EventPair> pool;
    verb_timing acc{};
};


namespace vctx {

// anything that changes a launch argument of the step (a field other than the
// PSD, scales, boundary types, options, forms) drops the captured step graph
inline void graph_invalidate(verb_ctx* c) { c->graph_valid = false; }

inline int cuda_ok(cudaError_t e)
{
    if (e == cudaSuccess) return VERB_OK;
    if (e == cudaErrorMemoryAllocation) return VERB_ERR_NOMEM;
    return VERB_ERR_CUDA;
}

inline int cuda_ok(int s) { return s; }

#define CK(x)                                 \
    do {                                      \
        int _s = cuda_ok(x);                  \
        if (_s != VERB_OK) return _s;         \
    } while (0)

inline size_t npts(const verb_ctx* c) { return c->d.npts(); }
inline int check_launch() { return cuda_ok(cudaGetLastError()); }

int alloc(void** p, size_t bytes);  // cudaMalloc unless *p is set already
int need_field(verb_ctx* c, int fid);
EventPair get_pair(verb_ctx* c);

// CUDA events around one phase, recorded while timing is on
struct PhaseTimer {
    verb_ctx* c;
    int ph;
    EventPair p{};
    PhaseTimer(verb_ctx* c_, int ph_) : c(c_), ph(ph_)
    {
        if (c->timing) {
            p = get_pair(c);
            cudaEventRecord(p.a, c->stream);
        }
    }
    ~PhaseTimer()
    {
        if (c->timing) {
            cudaEventRecord(p.b, c->stream);
            c->ev[ph].push_back(p);
        }
    }
};

int local_prepare(verb_ctx* c, LocalArgs& a, double dts);
int alloc_factors(verb_ctx* c, LocalArgs& a);
int local_factor(verb_ctx* c, LocalArgs& a);
void free_krylov(verb_ctx* c);  // ctx_krylov.cu
void free_kc(verb_ctx* c);      // ctx_assim.cu

}  // namespace vctx
using namespace vctx;
