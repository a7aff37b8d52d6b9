// gpt_api.cu -- the C ABI (include/gpt.h): handle, preallocated workspace,
// the reference's kernels as single-instance entry points, and the SQP loop
// (toplevel.cuh:24-503) driven from the host with every decision on the device.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gpt.h"
#include "gpt_common.cuh"
#include "gpt_internal.h"

using namespace gpt;

namespace {

thread_local std::string g_last_error;

gpt_status set_err(gpt_status st, const std::string &msg)
{
    g_last_error = msg;
    return st;
}
gpt_status cuda_err(cudaError_t e, const char *where)
{
    return set_err(GPT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define GPT_CUDA(call)                                        \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_err(e_, #call);    \
    } while (0)

// Makes a handle's device current for the duration of one entry point and restores the
// caller's current device on return, so a handle may be used from a thread whose current
// device is another GPU.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        int cur = -1;
        if (cudaGetDevice(&cur) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        if (cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard &) = delete;
    DeviceGuard &operator=(const DeviceGuard &) = delete;
};

}  // namespace

namespace gpt {
cudaError_t ensure_func_attrs(const void *func, size_t smem_bytes, bool cluster16)
{
    static std::mutex mu;
    struct Entry {
        const void *func;
        int device;
        size_t smem;
        bool cluster16;
    };
    static std::vector<Entry> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    Entry *hit = nullptr;
    for (Entry &t : done)
        if (t.func == func && t.device == dev) hit = &t;
    if (hit && hit->smem >= smem_bytes && (hit->cluster16 || !cluster16)) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    if (e != cudaSuccess) return e;
    if (cluster16) {
        e = cudaFuncSetAttribute(func, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    if (hit) {
        hit->smem = smem_bytes;
        hit->cluster16 = hit->cluster16 || cluster16;
    } else {
        done.push_back({func, dev, smem_bytes, cluster16});
    }
    return cudaSuccess;
}
}  // namespace gpt

constexpr int MAX_BRANCHES = 8;  // most concurrent part-batch branches of a graph iteration (sqp_graph)

struct GraphKey {
    int B, total, maxN, minN;
    int split[3 * MAX_BRANCHES];  // sqp_graph >= 2: per branch its first knot, longest and shortest horizon
    ProblemParams P;
    SolverParams SP;
};
struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec;
};

struct gpt_handle {
    gpt_problem_config pc;
    gpt_solver_config sc;
    int device = 0;
    int num_sms = 148;
    size_t cap_knots = 0;  // max_batch * max_knot_points
    // workspace
    float *G = nullptr, *C = nullptr, *g = nullptr, *c = nullptr, *S = nullptr,
          *gamma = nullptr, *Ginv = nullptr, *dz = nullptr, *xs = nullptr, *knot_merit = nullptr,
          *merits = nullptr;
    InstState *st = nullptr;
    int *knot_off = nullptr, *knot_inst = nullptr;
    uint32_t *pcg_log = nullptr, *pcg_out = nullptr, *d_active = nullptr;
    double *lam64 = nullptr;   // FP64 multipliers from the PCG, consumed by dz
    double *Ginv64 = nullptr;  // FP64 inverses (Q + rho I)^-1, (R + rho I)^-1 from Schur, consumed by dz
    double *Ginv64c = nullptr; // the same in compact form (GC64 doubles per knot) from the FP64 Schur kernel
    double *crw = nullptr;     // FP64 cyclic-reduction couplings of the PCG preconditioner, 196 per knot
    // adjoint workspace: right-hand side, its zero constraint part, gamma, multipliers, mu_z, partials
    float *adj_h = nullptr, *adj_zero = nullptr, *adj_gamma = nullptr, *adj_lam = nullptr, *adj_mu = nullptr,
          *adj_part = nullptr;
    double *adj_lam64 = nullptr;
    // FP64 Schur rows (PK64 doubles per knot) and right-hand sides for the cyclic-reduction PCG
    double *S64 = nullptr, *gamma64 = nullptr, *adj_gamma64 = nullptr;
    // the stair preconditioner (pcg_precond 2): S and Pinv in the reference's 3-block layout (allocated when
    // that preconditioner is first configured)
    float *Sref = nullptr, *Pref = nullptr;
    // the SQP loop as a CUDA graph: copies of the caller's buffers, the iteration count of the
    // device-side while loop, capture streams and the instantiated graphs per batch shape
    float *gxu = nullptr, *glam = nullptr, *ggoal = nullptr;
    uint32_t *d_iter = nullptr;
    // tracking loop: the previous solution (plant controls), trajectory row offsets, the shared
    // update clock, per-instance totals (the working xu, lambda and goal are gxu, glam, ggoal)
    float *trk_xu_old = nullptr;
    int *trk_rows = nullptr;
    TrackClock *trk_clk = nullptr;
    TrackInst *trk_inst = nullptr;
    InstState *trk_stbak = nullptr;  // per-solve state saved around an update's adjoint
    float *trk_ggrad = nullptr;      // the adjoint's per-knot goal gradients (6 per knot)
    float *trk_kloss = nullptr;      // the update's per-knot loss terms
    int *h_trk_rows = nullptr;
    TrackInst *h_trk_inst = nullptr;
    cudaStream_t cap_stream = nullptr, body_stream = nullptr;
    // the part-batch branches of a graph iteration (sqp_graph >= 2): streams 1.. and their events
    cudaStream_t branch_stream[MAX_BRANCHES] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[MAX_BRANCHES] = {};
    std::vector<GraphEntry> graphs;
    // autotuned PCG cluster size per batch shape (gpt_autotune); used when pcg_cluster_size is 0
    struct Tuned {
        int B, total, maxN, minN;
        uint32_t cluster;
        uint8_t cta[4];    // CTAs per SM of the KKT, FP64 Schur, merit and dz launches
        uint8_t branches;  // part-batch branches per graph iteration (sqp_graph 1 only; 0 = not tuned)
    };
    // a schedule under trial inside gpt_autotune (overrides the tuned entry)
    bool trial = false;
    uint8_t trial_cta[4] = {0, 0, 0, 0};
    std::vector<Tuned> tuned;
    uint32_t cap_sqp_iter = 0;  // pcg_log rows allocated at creation
    // pinned host staging
    uint32_t *h_active = nullptr;
    InstState *h_st = nullptr;
    uint32_t *h_pcg_out = nullptr;
    uint32_t *h_pcg_log = nullptr;
    int *h_knot_off = nullptr, *h_knot_inst = nullptr;  // staging of the batch layout's upload
    // cached batch layout
    std::vector<int> off_cache;
    cudaEvent_t ev = nullptr;
    // optional per-phase CUDA-event timing of the SQP loop's launches
    int profile = 0;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_phase;
    size_t ev_used = 0;
    double phase_ms[GPT_NUM_PHASES] = {0};
    uint64_t phase_launches[GPT_NUM_PHASES] = {0};
};

namespace {

ProblemParams to_params(const gpt_problem_config &pc)
{
    ProblemParams P;
    P.dt = pc.timestep;
    P.integrator = (int)pc.integrator;
    P.q_ee = pc.q_ee;
    P.qd_cost = pc.qd_cost;
    P.r_cost = pc.r_cost;
    P.mu = pc.mu;
    P.ref_terminal = (int)pc.ref_terminal;
    return P;
}
SolverParams to_solver(const gpt_solver_config &sc)
{
    SolverParams S{};
    S.sqp_max_iter = sc.sqp_max_iter;
    S.pcg_max_iter = sc.pcg_max_iter;
    S.pcg_tol = sc.pcg_exit_tol;
    S.pcg_exit_mode = sc.pcg_exit_mode;
    S.rho_factor = sc.rho_factor;
    S.rho_max = sc.rho_max;
    S.rho_min = sc.rho_min;
    S.pcg_cluster_size = sc.pcg_cluster_size;
    S.pcg_precond = sc.pcg_precond;
    S.schur_fp64 = sc.schur_fp64;
    S.sqp_graph = sc.sqp_graph;
    return S;
}
BatchView single_view(uint32_t N)
{
    BatchView bv;
    bv.B = 1;
    bv.total_knots = (int)N;
    bv.knot_off = nullptr;
    bv.knot_inst = nullptr;
    bv.st = nullptr;
    return bv;
}
bool check_n(const gpt_handle *h, uint32_t N) { return N >= 2 && N <= h->pc.max_knot_points; }

template <typename T>
cudaError_t dalloc(T **p, size_t n)
{
    return cudaMalloc((void **)p, sizeof(T) * (n ? n : 1));
}

}  // namespace

namespace gpt {
gpt_status record_error(gpt_status st, const char *msg) { return set_err(st, msg); }
ProblemParams problem_params(const gpt_problem_config &pc) { return to_params(pc); }
}  // namespace gpt

extern "C" {

void gpt_default_problem_config(gpt_problem_config *o)
{
    if (!o) return;
    o->state_size = 14;
    o->control_size = 7;
    o->max_knot_points = 128;
    o->max_batch = 1;
    o->timestep = 1.0f / 64.0f;
    o->integrator = 0;
    o->q_ee = 1.0f;
    o->qd_cost = 1e-4f;
    o->r_cost = 1e-4f;
    o->mu = 10.0f;
    o->ref_terminal = 1;
}

void gpt_default_solver_config(gpt_solver_config *o)
{
    if (!o) return;
    o->sqp_max_iter = 40;
    o->pcg_max_iter = 167;
    o->pcg_exit_tol = 1e-5f;
    o->pcg_exit_mode = 0;
    o->rho_factor = 1.2f;
    o->rho_max = 10.0f;
    o->rho_min = 1e-3f;
    o->pcg_cluster_size = 0;
    o->pcg_precond = 1;
    o->schur_fp64 = 1;
    o->sqp_graph = 1;
}

const char *gpt_last_error(void) { return g_last_error.c_str(); }
const char *gpt_version(void) { return "gpt-b200 0.1 (sm_100a)"; }

gpt_status gpt_set_solver_config(gpt_handle *h, const gpt_solver_config *sc)
{
    if (!h || !sc) return set_err(GPT_ERR_BAD_ARG, "null argument");
    if (sc->sqp_max_iter == 0 || sc->sqp_max_iter > 4096) return set_err(GPT_ERR_BAD_ARG, "sqp_max_iter out of range");
    if (!(sc->rho_factor > 1.0f) || !(sc->rho_min > 0.0f)) return set_err(GPT_ERR_BAD_ARG, "rho schedule out of range");
    if (sc->pcg_cluster_size == GPT_PCG_WARP_PAIR || sc->pcg_cluster_size == GPT_PCG_WARP_QUAD) {
        if (sc->pcg_precond != 1)
            return set_err(GPT_ERR_BAD_ARG, "pcg_cluster_size GPT_PCG_WARP_PAIR / GPT_PCG_WARP_QUAD needs pcg_precond 1");
    } else if (sc->pcg_cluster_size & (sc->pcg_cluster_size - 1) || sc->pcg_cluster_size > 16) {
        return set_err(GPT_ERR_BAD_ARG,
                       "pcg_cluster_size must be 0, 1, 2, 4, 8, 16, GPT_PCG_WARP_PAIR or GPT_PCG_WARP_QUAD");
    }
    if (sc->pcg_precond > 2) return set_err(GPT_ERR_BAD_ARG, "pcg_precond must be 0, 1 or 2");
    if (sc->pcg_precond == 2 && !h->Sref) {
        // the stair preconditioner's SQP loop forms S and Pinv in the reference's 3-block layout: its
        // buffers are allocated here, outside any solve
        const size_t T = h->cap_knots;
        if (cudaMalloc((void **)&h->Sref, sizeof(float) * S_STRIDE * T) != cudaSuccess ||
            cudaMalloc((void **)&h->Pref, sizeof(float) * S_STRIDE * T) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(h->Sref);
            h->Sref = nullptr;
            return set_err(GPT_ERR_CUDA, "cannot allocate the stair preconditioner's Schur buffers");
        }
        cudaMemset(h->Sref, 0, sizeof(float) * S_STRIDE * T);
        cudaMemset(h->Pref, 0, sizeof(float) * S_STRIDE * T);
    }
    if (sc->schur_fp64 > 1) return set_err(GPT_ERR_BAD_ARG, "schur_fp64 must be 0 or 1");
    if (sc->sqp_graph > (uint32_t)MAX_BRANCHES) return set_err(GPT_ERR_BAD_ARG, "sqp_graph must be 0 .. 8");
    if (sc->sqp_max_iter > h->cap_sqp_iter) {
        // pcg log is sized at creation
        return set_err(GPT_ERR_CAPACITY, "sqp_max_iter larger than at creation");
    }
    h->sc = *sc;
    return GPT_OK;
}

gpt_status gpt_set_cost_weights(gpt_handle *h, float q_ee, float qd_cost, float r_cost)
{
    if (!h) return set_err(GPT_ERR_BAD_ARG, "null argument");
    if (!(q_ee >= 0.0f) || !(qd_cost >= 0.0f) || !(r_cost >= 0.0f))
        return set_err(GPT_ERR_BAD_ARG, "cost weights must be finite and non-negative");
    h->pc.q_ee = q_ee;
    h->pc.qd_cost = qd_cost;
    h->pc.r_cost = r_cost;
    return GPT_OK;
}

gpt_status gpt_create(const gpt_problem_config *pc, const gpt_solver_config *sc, gpt_handle **out)
{
    if (!pc || !sc || !out) return set_err(GPT_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    if (pc->state_size != 14 || pc->control_size != 7)
        return set_err(GPT_ERR_BAD_ARG, "state_size must be 14 and control_size 7 (iiwa14)");
    if (pc->max_knot_points < 2 || pc->max_knot_points > (uint32_t)MAX_PCG_KNOTS)
        return set_err(GPT_ERR_BAD_ARG, "max_knot_points must be in [2, 512]");
    if (pc->max_batch < 1 || pc->max_batch > 65536) return set_err(GPT_ERR_BAD_ARG, "max_batch out of range");
    if (!(pc->timestep > 0.f) || pc->integrator > 1) return set_err(GPT_ERR_BAD_ARG, "bad timestep/integrator");
    if (sc->sqp_max_iter == 0 || sc->sqp_max_iter > 4096) return set_err(GPT_ERR_BAD_ARG, "sqp_max_iter out of range");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_err(GPT_ERR_NO_DEVICE, "no CUDA device");
    }
    gpt_handle *h = new gpt_handle();
    h->pc = *pc;
    h->sc = *sc;
    cudaGetDevice(&h->device);
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    const size_t T = (size_t)pc->max_batch * pc->max_knot_points;
    const size_t B = pc->max_batch;
    h->cap_knots = T;
    h->cap_sqp_iter = sc->sqp_max_iter;
    cudaError_t e = cudaSuccess;
#define ALLOC(p, n) \
    if (e == cudaSuccess) e = dalloc(&h->p, (n))
    ALLOC(G, G_STRIDE * T);
    ALLOC(C, C_STRIDE * T);
    ALLOC(g, NX * T);
    ALLOC(c, NS * T);
    ALLOC(S, PK * T);
    ALLOC(gamma, NS * T);
    ALLOC(Ginv, G_STRIDE * T);
    ALLOC(dz, NX * T);
    ALLOC(xs, NS * B);
    ALLOC(knot_merit, NUM_ALPHAS * T);
    ALLOC(merits, NUM_ALPHAS * B);
    ALLOC(st, B);
    ALLOC(knot_off, B + 1);
    ALLOC(knot_inst, T);
    ALLOC(pcg_log, B * sc->sqp_max_iter);
    ALLOC(pcg_out, 2 * B);
    ALLOC(d_active, 1);
    ALLOC(lam64, NS * T);
    ALLOC(Ginv64, G_STRIDE * T);
    ALLOC(Ginv64c, GC64 * T);
    ALLOC(crw, 2 * SS * T);
    ALLOC(adj_h, NX * T);
    ALLOC(adj_zero, NS * T);
    ALLOC(adj_gamma, NS * T);
    ALLOC(adj_lam, NS * T);
    ALLOC(adj_mu, NX * T);
    ALLOC(adj_part, adjoint_part_floats() * T);
    ALLOC(adj_lam64, NS * T);
    ALLOC(S64, PK64 * T);
    ALLOC(gamma64, NS * T);
    ALLOC(adj_gamma64, NS * T);
    ALLOC(gxu, NX * T);
    ALLOC(glam, NS * T);
    ALLOC(ggoal, 6 * T);
    ALLOC(d_iter, 1);
    ALLOC(trk_xu_old, NX * T);
    ALLOC(trk_rows, B + 1);
    ALLOC(trk_clk, 1);
    ALLOC(trk_inst, B);
    ALLOC(trk_stbak, B);
    ALLOC(trk_ggrad, 6 * T);
    ALLOC(trk_kloss, T);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->body_stream, cudaStreamNonBlocking);
    for (int i = 1; i < MAX_BRANCHES; ++i) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->branch_stream[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
#undef ALLOC
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_active, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_st, sizeof(InstState) * B);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_pcg_out, sizeof(uint32_t) * 2 * B);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_pcg_log, sizeof(uint32_t) * B * sc->sqp_max_iter);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_knot_off, sizeof(int) * (B + 1));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_knot_inst, sizeof(int) * T);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_trk_rows, sizeof(int) * (B + 1));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_trk_inst, sizeof(TrackInst) * B);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMemset(h->S, 0, sizeof(float) * PK * T);
    if (e == cudaSuccess) e = cudaMemset(h->dz, 0, sizeof(float) * NX * T);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        gpt_destroy(h);
        return cuda_err(e, "gpt_create workspace");
    }
    if (sc->pcg_precond == 2) {
        const gpt_status st2 = gpt_set_solver_config(h, sc);
        if (st2 != GPT_OK) {
            gpt_destroy(h);
            return st2;
        }
    }
    *out = h;
    return GPT_OK;
}

gpt_status gpt_set_profiling(gpt_handle *h, int enable)
{
    if (!h) return set_err(GPT_ERR_BAD_ARG, "null handle");
    h->profile = enable ? 1 : 0;
    return GPT_OK;
}

gpt_status gpt_get_phase_stats(gpt_handle *h, double *h_ms, uint64_t *h_launches, int reset)
{
    if (!h) return set_err(GPT_ERR_BAD_ARG, "null handle");
    for (int i = 0; i < GPT_NUM_PHASES; ++i) {
        if (h_ms) h_ms[i] = h->phase_ms[i];
        if (h_launches) h_launches[i] = h->phase_launches[i];
        if (reset) {
            h->phase_ms[i] = 0.0;
            h->phase_launches[i] = 0;
        }
    }
    return GPT_OK;
}

gpt_status gpt_destroy(gpt_handle *h)
{
    if (!h) return GPT_OK;
    DeviceGuard dg(h->device);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    cudaFree(h->G); cudaFree(h->C); cudaFree(h->g); cudaFree(h->c); cudaFree(h->S);
    cudaFree(h->gamma); cudaFree(h->Ginv); cudaFree(h->dz); cudaFree(h->xs); cudaFree(h->knot_merit);
    cudaFree(h->merits); cudaFree(h->st); cudaFree(h->knot_off); cudaFree(h->knot_inst); cudaFree(h->pcg_log);
    cudaFree(h->pcg_out); cudaFree(h->d_active); cudaFree(h->lam64); cudaFree(h->Ginv64); cudaFree(h->Ginv64c);
    cudaFree(h->crw);
    cudaFree(h->adj_h); cudaFree(h->adj_zero); cudaFree(h->adj_gamma); cudaFree(h->adj_lam); cudaFree(h->adj_mu);
    cudaFree(h->adj_part); cudaFree(h->adj_lam64);
    cudaFree(h->S64); cudaFree(h->gamma64); cudaFree(h->adj_gamma64);
    cudaFree(h->Sref); cudaFree(h->Pref);
    for (auto &ge : h->graphs) cudaGraphExecDestroy(ge.exec);
    cudaFree(h->gxu); cudaFree(h->glam); cudaFree(h->ggoal); cudaFree(h->d_iter);
    cudaFree(h->trk_xu_old); cudaFree(h->trk_rows); cudaFree(h->trk_clk); cudaFree(h->trk_inst);
    cudaFree(h->trk_stbak); cudaFree(h->trk_ggrad); cudaFree(h->trk_kloss);
    cudaFreeHost(h->h_trk_rows); cudaFreeHost(h->h_trk_inst);
    cudaFreeHost(h->h_knot_off); cudaFreeHost(h->h_knot_inst);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->body_stream) cudaStreamDestroy(h->body_stream);
    for (int i = 1; i < MAX_BRANCHES; ++i) {
        if (h->branch_stream[i]) cudaStreamDestroy(h->branch_stream[i]);
        if (h->ev_join[i]) cudaEventDestroy(h->ev_join[i]);
    }
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    cudaFreeHost(h->h_active); cudaFreeHost(h->h_st); cudaFreeHost(h->h_pcg_out); cudaFreeHost(h->h_pcg_log);
    if (h->ev) cudaEventDestroy(h->ev);
    delete h;
    return GPT_OK;
}

// ---------------------------------------------------------------------------
// single-instance kernels
// ---------------------------------------------------------------------------

gpt_status gpt_form_kkt(gpt_handle *h, uint32_t N, const float *d_xu, const float *d_goal, const float *d_xs,
                        float *d_G, float *d_C, float *d_g, float *d_c, gpt_stream_t stream)
{
    if (!h || !d_xu || !d_goal || !d_xs || !d_G || !d_C || !d_g || !d_c) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N)) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
    GPT_CUDA(launch_kkt(single_view(N), to_params(h->pc), d_xu, d_goal, d_xs, d_G, d_C, d_g, d_c, h->num_sms,
                        (cudaStream_t)stream));
    return GPT_OK;
}

gpt_status gpt_form_schur(gpt_handle *h, uint32_t N, float rho, const float *d_G, const float *d_C, const float *d_g,
                          const float *d_c, float *d_S, float *d_Pinv, float *d_gamma, float *d_Ginv,
                          double *d_Ginv64, gpt_stream_t stream)
{
    if (!h || !d_G || !d_C || !d_g || !d_c || !d_S || !d_Pinv || !d_gamma || !d_Ginv)
        return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N)) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
    GPT_CUDA(launch_schur(0, single_view(N), rho, d_G, d_C, d_g, d_c, d_S, d_Pinv, d_gamma, d_Ginv, d_Ginv64, nullptr,
                          1, h->num_sms, (cudaStream_t)stream));
    return GPT_OK;
}

gpt_status gpt_form_schur_csc(gpt_handle *h, uint32_t N, float rho, const float *d_G, const float *d_C,
                              const float *d_g, const float *d_c, float *d_val, float *d_gamma, float *d_Ginv,
                              gpt_stream_t stream)
{
    if (!h || !d_G || !d_C || !d_g || !d_c || !d_val || !d_gamma || !d_Ginv)
        return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N)) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
    GPT_CUDA(launch_schur(2, single_view(N), rho, d_G, d_C, d_g, d_c, nullptr, nullptr, d_gamma, d_Ginv, nullptr, d_val,
                          0, h->num_sms, (cudaStream_t)stream));
    return GPT_OK;
}

gpt_status gpt_form_ss(gpt_handle *h, uint32_t N, const float *d_S, float *d_Pinv, gpt_stream_t stream)
{
    if (!h || !d_S || !d_Pinv) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N)) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
    GPT_CUDA(launch_form_ss(single_view(N), d_S, d_Pinv, h->num_sms, (cudaStream_t)stream));
    return GPT_OK;
}

gpt_status gpt_prep_csr(uint32_t N, int32_t *cp, int32_t *ri)
{
    if (!cp || !ri || N < 1) return set_err(GPT_ERR_BAD_ARG, "bad argument");
    const int tri = (NS + 1) * NS / 2, brow = SS + tri;
    cp[0] = 0;
    for (uint32_t b = 0; b < N; ++b)
        for (int r = 0; r < NS; ++r) {
            const int bb = (int)b;
            const int off = (bb > 0) * tri + (bb > 0) * (bb - 1) * brow + (bb > 0) * r * NS + (r + 1) * r / 2;
            const int len = (bb > 0) * NS + r + 1;
            cp[bb * NS + r + 1] = off + len;
            for (int k = 0; k < len; ++k) ri[off + k] = (bb > 0) * (bb - 1) * NS + k;
        }
    return GPT_OK;
}

gpt_status gpt_pcg(gpt_handle *h, uint32_t N, const float *d_S, const float *d_Pinv, const float *d_gamma,
                   float *d_lambda, double *d_lambda64, uint32_t max_iter, float tol, uint32_t exit_mode,
                   uint32_t *h_iters, uint8_t *h_maxit, gpt_stream_t stream)
{
    if (!h || !d_S || !d_Pinv || !d_gamma || !d_lambda) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N) || exit_mode > 1) return set_err(GPT_ERR_BAD_ARG, "knot_points/exit_mode out of range");
    if (((uintptr_t)d_S & 15u) != 0) return set_err(GPT_ERR_BAD_ARG, "d_S must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    if (h->sc.pcg_cluster_size == GPT_PCG_WARP_PAIR || h->sc.pcg_cluster_size == GPT_PCG_WARP_QUAD) {
        // the one-CTA kernels read packed FP64 rows: the caller's S and gamma, converted exactly
        GPT_CUDA(launch_pack_rows64((int)N, d_S, d_gamma, h->S64, h->gamma64, h->num_sms, s));
        GPT_CUDA(launch_pcg(single_view(N), (int)N, (int)N, 2, 1, reinterpret_cast<const float *>(h->S64), d_Pinv,
                            d_gamma, h->gamma64, d_lambda, d_lambda64, h->crw, (int)max_iter, tol, (int)exit_mode,
                            h->pcg_out, nullptr, 0, (int)h->sc.pcg_cluster_size, h->num_sms, s));
    } else {
        GPT_CUDA(launch_pcg(single_view(N), (int)N, (int)N, 0, (int)h->sc.pcg_precond, d_S, d_Pinv, d_gamma, nullptr,
                            d_lambda, d_lambda64, h->crw, (int)max_iter, tol, (int)exit_mode, h->pcg_out, nullptr, 0,
                            (int)h->sc.pcg_cluster_size, h->num_sms, s));
    }
    GPT_CUDA(cudaMemcpyAsync(h->h_pcg_out, h->pcg_out, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GPT_CUDA(cudaStreamSynchronize(s));
    if (h_iters) *h_iters = h->h_pcg_out[0];
    if (h_maxit) *h_maxit = (uint8_t)(h->h_pcg_out[1] & 1u);
    if (h->h_pcg_out[1] & 2u) return set_err(GPT_ERR_NONFINITE, "non-finite value in PCG");
    return GPT_OK;
}

gpt_status gpt_compute_dz(gpt_handle *h, uint32_t N, const float *d_Ginv, const double *d_Ginv64, const float *d_C,
                          const float *d_g, const float *d_lambda, const double *d_lambda64, float *d_dz,
                          gpt_stream_t stream)
{
    if (!h || (!d_Ginv && !d_Ginv64) || !d_C || !d_g || (!d_lambda && !d_lambda64) || !d_dz)
        return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N)) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
    GPT_CUDA(launch_dz(single_view(N), d_Ginv, d_Ginv64, nullptr, d_C, d_g, d_lambda, d_lambda64, d_dz, h->num_sms,
                       (cudaStream_t)stream));
    return GPT_OK;
}

gpt_status gpt_compute_merit(gpt_handle *h, uint32_t N, const float *d_xu, const float *d_goal, float *d_merit,
                             gpt_stream_t stream)
{
    if (!h || !d_xu || !d_goal || !d_merit) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N)) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
    cudaStream_t s = (cudaStream_t)stream;
    BatchView bv = single_view(N);
    GPT_CUDA(launch_merit(bv, to_params(h->pc), 1, d_xu, nullptr, d_goal, nullptr, h->knot_merit, h->num_sms, s));
    GPT_CUDA(launch_accept(bv, 0, to_solver(h->sc), h->knot_merit, nullptr, nullptr, h->merits, nullptr, h->num_sms, s));
    GPT_CUDA(cudaMemcpyAsync(d_merit, h->merits, sizeof(float), cudaMemcpyDeviceToDevice, s));
    return GPT_OK;
}

gpt_status gpt_ls_compute_merit(gpt_handle *h, uint32_t N, const float *d_xs, const float *d_xu, const float *d_goal,
                                const float *d_dz, float *d_merits, gpt_stream_t stream)
{
    if (!h || !d_xs || !d_xu || !d_goal || !d_dz || !d_merits) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N)) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
    cudaStream_t s = (cudaStream_t)stream;
    BatchView bv = single_view(N);
    GPT_CUDA(launch_merit(bv, to_params(h->pc), NUM_ALPHAS, d_xu, d_dz, d_goal, d_xs, h->knot_merit, h->num_sms, s));
    GPT_CUDA(launch_accept(bv, 2, to_solver(h->sc), h->knot_merit, nullptr, nullptr, h->merits, nullptr, h->num_sms, s));
    GPT_CUDA(cudaMemcpyAsync(d_merits, h->merits, NUM_ALPHAS * sizeof(float), cudaMemcpyDeviceToDevice, s));
    return GPT_OK;
}

// ---------------------------------------------------------------------------
// SQP loop
// ---------------------------------------------------------------------------

// Brackets one phase launch with a pair of events when profiling is on.
struct PhaseTimer {
    gpt_handle *h;
    cudaStream_t s;
    int phase;
    size_t slot = (size_t)-1;
    PhaseTimer(gpt_handle *h_, cudaStream_t s_, int phase_) : h(h_), s(s_), phase(phase_)
    {
        if (!h->profile) return;
        if (h->ev_used + 2 > h->ev_pool.size()) {
            for (int i = 0; i < 64; ++i) {
                cudaEvent_t e;
                if (cudaEventCreate(&e) != cudaSuccess) return;
                h->ev_pool.push_back(e);
                h->ev_phase.push_back(0);
            }
        }
        slot = h->ev_used;
        h->ev_used += 2;
        h->ev_phase[slot] = phase;
        cudaEventRecord(h->ev_pool[slot], s);
    }
    ~PhaseTimer()
    {
        if (slot != (size_t)-1) cudaEventRecord(h->ev_pool[slot + 1], s);
    }
};

// After the stream synchronised: fold the recorded event pairs into the per-phase totals.
static void collect_phase_times(gpt_handle *h)
{
    for (size_t i = 0; i + 1 < h->ev_used; i += 2) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, h->ev_pool[i], h->ev_pool[i + 1]) == cudaSuccess) {
            h->phase_ms[h->ev_phase[i]] += ms;
            h->phase_launches[h->ev_phase[i]] += 1;
        }
    }
    h->ev_used = 0;
}

// Batch layout (knot offsets and owner table, cached), per-instance state (rho
// from h_rho, active) and the view the kernels take.
static gpt_status setup_batch(gpt_handle *h, uint32_t B, const uint32_t *Ns, const float *h_rho, float rho_reset,
                              BatchView &bv, int &maxN_out, int &minN_out, cudaStream_t s)
{
    if (B == 0 || B > h->pc.max_batch) return set_err(GPT_ERR_CAPACITY, "batch exceeds handle capacity");
    // batch layout
    std::vector<int> off(B + 1, 0);
    for (uint32_t b = 0; b < B; ++b) {
        if (!check_n(h, Ns[b])) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
        off[b + 1] = off[b] + (int)Ns[b];
    }
    const int total = off[B];
    if ((size_t)total > h->cap_knots) return set_err(GPT_ERR_CAPACITY, "total knots exceed workspace");
    int maxN = 0, minN = 1 << 30;
    for (uint32_t b = 0; b < B; ++b) {
        maxN = Ns[b] > (uint32_t)maxN ? (int)Ns[b] : maxN;
        minN = Ns[b] < (uint32_t)minN ? (int)Ns[b] : minN;
    }
    if (off != h->off_cache) {
        // stream-ordered upload from pinned staging: every entry point that reaches here synchronises
        // its stream before returning, so the staging is free again at the next call
        for (uint32_t b = 0; b <= B; ++b) h->h_knot_off[b] = off[b];
        for (uint32_t b = 0; b < B; ++b)
            for (int k = off[b]; k < off[b + 1]; ++k) h->h_knot_inst[k] = (int)b;
        GPT_CUDA(cudaMemcpyAsync(h->knot_off, h->h_knot_off, sizeof(int) * (B + 1), cudaMemcpyHostToDevice, s));
        GPT_CUDA(cudaMemcpyAsync(h->knot_inst, h->h_knot_inst, sizeof(int) * total, cudaMemcpyHostToDevice, s));
        h->off_cache = off;
    }
    for (uint32_t b = 0; b < B; ++b) {
        InstState &st = h->h_st[b];
        std::memset(&st, 0, sizeof(st));
        st.rho = h_rho ? h_rho[b] : 1e-3f;
        st.drho = 1.0f;
        st.rho_reset = rho_reset;
        st.active = 1;
    }
    GPT_CUDA(cudaMemcpyAsync(h->st, h->h_st, sizeof(InstState) * B, cudaMemcpyHostToDevice, s));
    bv.B = (int)B;
    bv.total_knots = total;
    bv.knot_off = h->knot_off;
    bv.knot_inst = h->knot_inst;
    bv.st = h->st;
    maxN_out = maxN;
    minN_out = minN;
    return GPT_OK;
}


// What one batched solve needs beyond the handle: the batch view and the parameters.
struct SqpPlan {
    BatchView bv;
    ProblemParams P;
    SolverParams SP;
    int maxN, minN, ns;
};

// x_s and the merit of the initial iterate (toplevel.cuh:110,235-244)
static gpt_status enqueue_prologue(gpt_handle *h, const SqpPlan &pl, const float *d_goal, float *d_xu, cudaStream_t s)
{
    PhaseTimer t(h, s, GPT_PHASE_INIT);
    GPT_CUDA(launch_init(pl.bv, d_xu, h->xs, pl.ns, s));
    GPT_CUDA(launch_kkt_gconst(pl.bv, pl.P, h->G, pl.ns, s));  // G's weight-only entries, once per solve
    GPT_CUDA(launch_merit(pl.bv, pl.P, 1, d_xu, nullptr, d_goal, h->xs, h->knot_merit, pl.ns, s,
                          ctas_or_default(pl.SP.cta_merit)));
    GPT_CUDA(launch_accept(pl.bv, 0, pl.SP, h->knot_merit, nullptr, nullptr, nullptr, nullptr, pl.ns, s));
    return GPT_OK;
}

// One SQP iteration for every active instance (toplevel.cuh:254-446); leaves the number of
// instances still active in h->d_active (cleared first unless reset_active is false).
static gpt_status enqueue_iteration(gpt_handle *h, const SqpPlan &pl, const float *d_goal, float *d_lambda,
                                    float *d_xu, cudaStream_t s, bool reset_active = true,
                                    float *merits_out = nullptr)
{
    const BatchView &bv = pl.bv;
    const SolverParams &SP = pl.SP;
    const int ns = pl.ns;
    const bool f64 = SP.pcg_precond == 1 && SP.schur_fp64;
    const bool stair = SP.pcg_precond == 2;
    const float *S_rows = f64 ? reinterpret_cast<const float *>(h->S64) : (stair ? h->Sref : h->S);
    {
        PhaseTimer t(h, s, GPT_PHASE_KKT);
        GPT_CUDA(launch_kkt(bv, pl.P, d_xu, d_goal, h->xs, h->G, h->C, h->g, h->c, ns, s, ctas_or_default(SP.cta_kkt),
                            false));
    }
    {
        PhaseTimer t(h, s, GPT_PHASE_SCHUR);
        if (f64) {
            GPT_CUDA(launch_schur64(bv, h->G, h->C, h->g, h->c, h->S64, h->gamma64, nullptr, h->Ginv64, h->Ginv64c,
                                    ns, s, ctas_or_default(SP.cta_schur)));
        } else if (stair) {
            // the reference's rows and block-Jacobi Pinv (gato_form_schur_jacobi), then the stair blocks
            if (!h->Sref) return set_err(GPT_ERR_BAD_ARG, "pcg_precond 2 was not configured on this handle");
            GPT_CUDA(launch_schur(0, bv, 0.f, h->G, h->C, h->g, h->c, h->Sref, h->Pref, h->gamma, h->Ginv, h->Ginv64,
                                  nullptr, 1, ns, s));
            GPT_CUDA(launch_form_ss(bv, h->Sref, h->Pref, ns, s));
        } else {
            GPT_CUDA(launch_schur(1, bv, 0.f, h->G, h->C, h->g, h->c, h->S, nullptr, h->gamma, h->Ginv, h->Ginv64,
                                  nullptr, SP.pcg_precond == 0 ? 1 : 0, ns, s));
        }
    }
    {
        PhaseTimer t(h, s, GPT_PHASE_PCG);
        GPT_CUDA(launch_pcg(bv, pl.maxN, pl.minN, f64 ? 2 : (stair ? 0 : 1), (int)SP.pcg_precond, S_rows,
                            stair ? h->Pref : nullptr, h->gamma,
                            h->gamma64, d_lambda, h->lam64, h->crw, (int)SP.pcg_max_iter, SP.pcg_tol,
                            (int)SP.pcg_exit_mode, nullptr, h->pcg_log, (int)SP.sqp_max_iter,
                            (int)SP.pcg_cluster_size, ns, s));
    }
    {
        PhaseTimer t(h, s, GPT_PHASE_DZ);
        GPT_CUDA(launch_dz(bv, h->Ginv, h->Ginv64, f64 ? h->Ginv64c : nullptr, h->C, h->g, d_lambda, h->lam64, h->dz,
                           ns, s, ctas_or_default(SP.cta_dz)));
    }
    {
        PhaseTimer t(h, s, GPT_PHASE_MERIT);
        GPT_CUDA(launch_merit(bv, pl.P, NUM_ALPHAS, d_xu, h->dz, d_goal, h->xs, h->knot_merit, ns, s,
                              ctas_or_default(SP.cta_merit)));
    }
    if (reset_active) GPT_CUDA(cudaMemsetAsync(h->d_active, 0, sizeof(uint32_t), s));
    {
        PhaseTimer t(h, s, GPT_PHASE_ACCEPT);
        GPT_CUDA(launch_accept(bv, 1, SP, h->knot_merit, h->dz, d_xu, merits_out, h->d_active, ns, s));
    }
    return GPT_OK;
}

// sqp_graph K >= 2: the batch as K parts (contiguous instance ranges of near-equal size) whose
// iterations run on K branches of the graph, so that one part's latency-bound PCG overlaps the
// others' throughput-bound KKT, Schur and merit kernels.  The parts share no workspace (every
// buffer is indexed by the batch's knot or instance); the active count is cleared once before all.
static int branch_count(const gpt_handle *h, const SqpPlan &pl)
{
    if (pl.SP.sqp_graph < 2 || pl.bv.knot_off == nullptr || h->off_cache.size() != (size_t)pl.bv.B + 1) return 1;
    int k = (int)pl.SP.sqp_graph;
    k = k < MAX_BRANCHES ? k : MAX_BRANCHES;
    return k < pl.bv.B ? k : pl.bv.B;
}

static void split_plan(const gpt_handle *h, const SqpPlan &pl, int K, SqpPlan *part)
{
    const std::vector<int> &off = h->off_cache;
    const int B = pl.bv.B;
    for (int i = 0; i < K; ++i) {
        const int b0 = (int)((int64_t)B * i / K), b1 = (int)((int64_t)B * (i + 1) / K);
        part[i] = pl;
        BatchView &v = part[i].bv;
        v.b0 = b0;
        v.B = b1 - b0;
        v.j0 = off[b0];
        v.total_knots = off[b1] - off[b0];
        int mx = 0, mn = 1 << 30;
        for (int b = b0; b < b1; ++b) {
            const int n = off[b + 1] - off[b];
            mx = n > mx ? n : mx;
            mn = n < mn ? n : mn;
        }
        part[i].maxN = mx;
        part[i].minN = mn;
    }
}

static gpt_status enqueue_iteration_split(gpt_handle *h, const SqpPlan &pl, int K, cudaStream_t s)
{
    SqpPlan part[MAX_BRANCHES];
    split_plan(h, pl, K, part);
    GPT_CUDA(cudaMemsetAsync(h->d_active, 0, sizeof(uint32_t), s));
    GPT_CUDA(cudaEventRecord(h->ev_fork, s));
    for (int i = 1; i < K; ++i) GPT_CUDA(cudaStreamWaitEvent(h->branch_stream[i], h->ev_fork, 0));
    for (int i = 0; i < K; ++i) {
        const gpt_status st =
            enqueue_iteration(h, part[i], h->ggoal, h->glam, h->gxu, i == 0 ? s : h->branch_stream[i], false);
        if (st != GPT_OK) return st;
    }
    for (int i = 1; i < K; ++i) {
        GPT_CUDA(cudaEventRecord(h->ev_join[i], h->branch_stream[i]));
        GPT_CUDA(cudaStreamWaitEvent(s, h->ev_join[i], 0));
    }
    return GPT_OK;
}

// Loop control of the graph's while node: counts the iterations and continues while an
// instance is active and fewer than sqp_max_iter iterations ran (the count bounds the loop
// even if the activity flags were never cleared).
__global__ void sqp_continue_kernel(cudaGraphConditionalHandle cond, const uint32_t *__restrict__ active,
                                    uint32_t *__restrict__ iter, uint32_t max_iter)
{
    const uint32_t it = *iter + 1u;
    *iter = it;
    cudaGraphSetConditional(cond, (*active > 0u && it < max_iter) ? 1u : 0u);
}

// The whole solve as one CUDA graph: prologue, then a while node whose body is one SQP
// iteration followed by sqp_continue_kernel.  Built by stream capture on the handle's
// private streams for each (batch shape, parameters) and cached.
static gpt_status sqp_graph_for(gpt_handle *h, const SqpPlan &pl, cudaGraphExec_t *out)
{
    GraphKey key;
    std::memset(&key, 0, sizeof(key));
    key.B = pl.bv.B;
    key.total = pl.bv.total_knots;
    key.maxN = pl.maxN;
    key.minN = pl.minN;
    const int K = branch_count(h, pl);
    if (K > 1) {
        SqpPlan part[MAX_BRANCHES];
        split_plan(h, pl, K, part);
        for (int i = 0; i < K; ++i) {
            key.split[3 * i] = part[i].bv.j0;
            key.split[3 * i + 1] = part[i].maxN;
            key.split[3 * i + 2] = part[i].minN;
        }
    }
    key.P = pl.P;
    key.SP = pl.SP;
    for (auto &e : h->graphs)
        if (std::memcmp(&e.key, &key, sizeof(key)) == 0) {
            *out = e.exec;
            return GPT_OK;
        }
    cudaStream_t cs = h->cap_stream, bs = h->body_stream;
    cudaGraph_t graph = nullptr;
    GPT_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
    gpt_status st = enqueue_prologue(h, pl, h->ggoal, h->gxu, cs);
    if (st == GPT_OK) {
        cudaError_t e = cudaMemsetAsync(h->d_iter, 0, sizeof(uint32_t), cs);
        cudaStreamCaptureStatus cst;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, &deps, &ndeps);
        cudaGraphConditionalHandle cond;
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&cond, graph, 1u, cudaGraphCondAssignDefault);
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        if (e == cudaSuccess) e = cudaGraphAddNode(&node, graph, deps, ndeps, &cp);
        if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies);
        if (e == cudaSuccess) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            e = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
            if (e == cudaSuccess) {
                st = K > 1 ? enqueue_iteration_split(h, pl, K, bs)
                           : enqueue_iteration(h, pl, h->ggoal, h->glam, h->gxu, bs);
                if (st == GPT_OK) {
                    sqp_continue_kernel<<<1, 1, 0, bs>>>(cond, h->d_active, h->d_iter, pl.SP.sqp_max_iter);
                    e = cudaGetLastError();
                }
                cudaGraph_t body_out = nullptr;
                const cudaError_t e2 = cudaStreamEndCapture(bs, &body_out);
                if (e == cudaSuccess) e = e2;
            }
        }
        if (e != cudaSuccess && st == GPT_OK) st = cuda_err(e, "SQP graph capture");
    }
    cudaGraph_t captured = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(cs, &captured);
    if (st != GPT_OK) {
        if (captured) cudaGraphDestroy(captured);
        return st;
    }
    if (ee != cudaSuccess) return cuda_err(ee, "cudaStreamEndCapture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, captured, 0);
    cudaGraphDestroy(captured);
    if (ei != cudaSuccess) return cuda_err(ei, "cudaGraphInstantiate");
    h->graphs.push_back({key, exec});
    *out = exec;
    return GPT_OK;
}

// The autotuned PCG kernel and launch schedule of this batch shape (gpt_autotune), where the solver
// config leaves the PCG cluster size to the library; a schedule under trial takes precedence.
static void apply_tuned(const gpt_handle *h, const BatchView &bv, int maxN, int minN, SolverParams &SP)
{
    const bool tune_graph = SP.sqp_graph == 1 && !h->trial;  // a graph solve whose branch count is not given
    for (const auto &t : h->tuned)
        if (t.B == bv.B && t.total == bv.total_knots && t.maxN == maxN && t.minN == minN) {
            if (SP.pcg_cluster_size == 0) {
                SP.pcg_cluster_size = t.cluster;
                SP.cta_kkt = t.cta[0];
                SP.cta_schur = t.cta[1];
                SP.cta_merit = t.cta[2];
                SP.cta_dz = t.cta[3];
            }
            if (tune_graph && t.branches > 1) SP.sqp_graph = t.branches;
        }
    if (h->trial) {
        SP.cta_kkt = h->trial_cta[0];
        SP.cta_schur = h->trial_cta[1];
        SP.cta_merit = h->trial_cta[2];
        SP.cta_dz = h->trial_cta[3];
    }
}

// Buffers of gpt_sqp_solve_batched_trace
struct SqpTrace {
    uint32_t iters;
    float *xu;
    double *lam;
    float *dz;
    gpt_iterate_record *rec;
};

static gpt_status sqp_run(gpt_handle *h, uint32_t B, const uint32_t *Ns, const float *d_goal, float *d_lambda,
                          float *d_xu, float *h_rho, float rho_reset, gpt_sqp_stats *h_stats, uint32_t *h_pcg_iters,
                          uint8_t *h_pcg_exit, cudaStream_t s, const SqpTrace *tr = nullptr)
{
    BatchView bv;
    int maxN = 0, minN = 0;
    {
        const gpt_status st = setup_batch(h, B, Ns, h_rho, rho_reset, bv, maxN, minN, s);
        if (st != GPT_OK) return st;
    }
    const ProblemParams P = to_params(h->pc);
    SolverParams SP = to_solver(h->sc);
    apply_tuned(h, bv, maxN, minN, SP);
    const SqpPlan plan{bv, P, SP, maxN, minN, h->num_sms};

    if (SP.sqp_graph && !h->profile && !tr) {
        // one graph launch for the whole solve on handle-owned copies of the caller's buffers
        const size_t nxu = (size_t)NX * bv.total_knots - NC, nl = (size_t)NS * bv.total_knots;
        GPT_CUDA(cudaMemcpyAsync(h->gxu, d_xu, sizeof(float) * nxu, cudaMemcpyDeviceToDevice, s));
        GPT_CUDA(cudaMemcpyAsync(h->glam, d_lambda, sizeof(float) * nl, cudaMemcpyDeviceToDevice, s));
        GPT_CUDA(cudaMemcpyAsync(h->ggoal, d_goal, sizeof(float) * 6 * bv.total_knots, cudaMemcpyDeviceToDevice, s));
        cudaGraphExec_t exec = nullptr;
        {
            const gpt_status st = sqp_graph_for(h, plan, &exec);
            if (st != GPT_OK) return st;
        }
        GPT_CUDA(cudaGraphLaunch(exec, s));
        GPT_CUDA(cudaMemcpyAsync(d_xu, h->gxu, sizeof(float) * nxu, cudaMemcpyDeviceToDevice, s));
        GPT_CUDA(cudaMemcpyAsync(d_lambda, h->glam, sizeof(float) * nl, cudaMemcpyDeviceToDevice, s));
    } else {
        {
            const gpt_status st = enqueue_prologue(h, plan, d_goal, d_xu, s);
            if (st != GPT_OK) return st;
        }
        const size_t T = (size_t)bv.total_knots;
        for (uint32_t it = 0; it < SP.sqp_max_iter; ++it) {
            const bool rec = tr && it < tr->iters;
            if (rec && tr->xu)
                GPT_CUDA(cudaMemcpyAsync(tr->xu + NX * T * it, d_xu, sizeof(float) * (NX * T - NC),
                                         cudaMemcpyDeviceToDevice, s));
            if (rec && tr->rec) GPT_CUDA(launch_trace_record(bv, 0, nullptr, tr->rec + (size_t)B * it, plan.ns, s));
            const gpt_status st = enqueue_iteration(h, plan, d_goal, d_lambda, d_xu, s, true, rec ? h->merits : nullptr);
            if (st != GPT_OK) return st;
            if (rec && tr->lam)
                GPT_CUDA(cudaMemcpyAsync(tr->lam + NS * T * it, h->lam64, sizeof(double) * NS * T,
                                         cudaMemcpyDeviceToDevice, s));
            if (rec && tr->dz)
                GPT_CUDA(cudaMemcpyAsync(tr->dz + NX * T * it, h->dz, sizeof(float) * (NX * T - NC),
                                         cudaMemcpyDeviceToDevice, s));
            if (rec && tr->rec) GPT_CUDA(launch_trace_record(bv, 1, h->merits, tr->rec + (size_t)B * it, plan.ns, s));
            GPT_CUDA(cudaMemcpyAsync(h->h_active, h->d_active, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            GPT_CUDA(cudaEventRecord(h->ev, s));
            GPT_CUDA(cudaEventSynchronize(h->ev));
            if (*h->h_active == 0) break;
        }
    }
    GPT_CUDA(cudaMemcpyAsync(h->h_st, h->st, sizeof(InstState) * B, cudaMemcpyDeviceToHost, s));
    if (h_pcg_iters || h_pcg_exit)
        GPT_CUDA(cudaMemcpyAsync(h->h_pcg_log, h->pcg_log, sizeof(uint32_t) * SP.sqp_max_iter, cudaMemcpyDeviceToHost, s));
    GPT_CUDA(cudaStreamSynchronize(s));
    if (h->profile) collect_phase_times(h);
    bool nonfinite = false, factor = false;
    for (uint32_t b = 0; b < B; ++b) {
        const InstState &st = h->h_st[b];
        if (h_rho) h_rho[b] = st.rho;
        if (st.exit_flags & GPT_EXIT_NONFINITE) nonfinite = true;
        if (st.exit_flags & GPT_EXIT_FACTOR) factor = true;
        if (h_stats) {
            gpt_sqp_stats &o = h_stats[b];
            o.sqp_iters = st.sqp_iters;
            o.exit_flags = st.exit_flags | (st.pcg_maxiter_count ? GPT_EXIT_PCG_MAXITER : 0u);
            o.pcg_iters_total = st.pcg_iters_total;
            o.pcg_maxiter_count = st.pcg_maxiter_count;
            o.ls_fail_count = st.ls_fail_count;
            o.merit_initial = st.merit_init;
            o.merit_final = st.merit0;
            o.rho_final = st.rho;
        }
    }
    if (h_pcg_iters || h_pcg_exit) {
        const uint32_t n = h->h_st[0].sqp_iters;
        for (uint32_t i = 0; i < SP.sqp_max_iter; ++i) {
            const uint32_t v = (i < n) ? h->h_pcg_log[i] : 0u;
            if (h_pcg_iters) h_pcg_iters[i] = v & 0x7fffffffu;
            if (h_pcg_exit) h_pcg_exit[i] = (uint8_t)(v >> 31);
        }
    }
    if (factor)
        return set_err(GPT_ERR_FACTOR, "(Q + rho I) or (R + rho I) not positive definite in at least one instance");
    if (nonfinite) return set_err(GPT_ERR_NONFINITE, "non-finite merit or PCG reduction in at least one instance");
    return GPT_OK;
}

gpt_status gpt_sqp_solve(gpt_handle *h, uint32_t N, const float *d_goal, float *d_lambda, float *d_xu, float *h_rho,
                         float rho_reset, gpt_sqp_stats *h_stats, uint32_t *h_pcg_iters, uint8_t *h_pcg_exit,
                         gpt_stream_t stream)
{
    if (!h || !d_goal || !d_lambda || !d_xu || !h_rho) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    return sqp_run(h, 1, &N, d_goal, d_lambda, d_xu, h_rho, rho_reset, h_stats, h_pcg_iters, h_pcg_exit,
                   (cudaStream_t)stream);
}

gpt_status gpt_sqp_solve_batched(gpt_handle *h, uint32_t B, const uint32_t *h_N, const float *d_goal, float *d_lambda,
                                 float *d_xu, float *h_rho, float rho_reset, gpt_sqp_stats *h_stats,
                                 gpt_stream_t stream)
{
    if (!h || !h_N || !d_goal || !d_lambda || !d_xu) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    return sqp_run(h, B, h_N, d_goal, d_lambda, d_xu, h_rho, rho_reset, h_stats, nullptr, nullptr,
                   (cudaStream_t)stream);
}

gpt_status gpt_sqp_solve_batched_trace(gpt_handle *h, uint32_t B, const uint32_t *h_N, const float *d_goal,
                                       float *d_lambda, float *d_xu, float *h_rho, float rho_reset,
                                       gpt_sqp_stats *h_stats, uint32_t trace_iters, float *d_trace_xu,
                                       double *d_trace_lambda, float *d_trace_dz, gpt_iterate_record *d_trace_rec,
                                       gpt_stream_t stream)
{
    if (!h || !h_N || !d_goal || !d_lambda || !d_xu) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    const SqpTrace tr{trace_iters, d_trace_xu, d_trace_lambda, d_trace_dz, d_trace_rec};
    return sqp_run(h, B, h_N, d_goal, d_lambda, d_xu, h_rho, rho_reset, h_stats, nullptr, nullptr,
                   (cudaStream_t)stream, &tr);
}

gpt_status gpt_autotune(gpt_handle *h, uint32_t B, const uint32_t *h_N, const float *d_goal, const float *d_lambda,
                        const float *d_xu, const float *h_rho, uint32_t *h_cluster_out, uint32_t *h_schedule_out,
                        gpt_stream_t stream)
{
    if (!h || !h_N || !d_goal || !d_lambda || !d_xu || !h_rho) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (B == 0 || B > h->pc.max_batch) return set_err(GPT_ERR_CAPACITY, "batch exceeds handle capacity");
    cudaStream_t s = (cudaStream_t)stream;
    int total = 0, maxN = 0, minN = 1 << 30;
    for (uint32_t b = 0; b < B; ++b) {
        if (!check_n(h, h_N[b])) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
        total += (int)h_N[b];
        maxN = (int)h_N[b] > maxN ? (int)h_N[b] : maxN;
        minN = (int)h_N[b] < minN ? (int)h_N[b] : minN;
    }
    if ((size_t)total > h->cap_knots) return set_err(GPT_ERR_CAPACITY, "total knots exceed workspace");
    // PCG candidates: the smallest cluster that holds the longest horizon (<= 128 knots per CTA) and 2x, 4x it
    int cs0 = 1;
    const int kpc_cap = h->sc.pcg_precond == 2 ? PCG_KPC_STAIR : PCG_KPC_MAX;
    while ((maxN + cs0 - 1) / cs0 > kpc_cap) cs0 *= 2;
    std::vector<uint32_t> cand;
    for (int cs = cs0; cs <= 16 && cs <= 4 * cs0 && cs <= minN; cs *= 2) cand.push_back((uint32_t)cs);
    if (cand.empty()) cand.push_back((uint32_t)cs0);
    if (h->sc.pcg_precond == 1) {  // one 128-thread CTA per instance: two or four factoring warps
        cand.push_back(GPT_PCG_WARP_PAIR);
        cand.push_back(GPT_PCG_WARP_QUAD);
    }
    const gpt_solver_config saved = h->sc;
    const int saved_profile = h->profile;
    h->profile = 0;
    const size_t nxu = (size_t)NX * total - NC, nl = (size_t)NS * total;
    std::vector<float> rho(h_rho, h_rho + B);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    gpt_status st = GPT_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) st = set_err(GPT_ERR_CUDA, "event");
    // two SQP iterations of the batch with a given PCG kernel and launch schedule: the best of two timed
    // repetitions after one warm-up (attributes, graph capture, caches)
    uint32_t branches = 1;  // part-batch branches of the trials (a graph solve: the caller's sqp_graph 1)
    auto time_schedule = [&](uint32_t cluster, const uint8_t *cta) -> float {
        h->sc = saved;
        h->sc.pcg_cluster_size = cluster;
        if (saved.sqp_graph == 1) h->sc.sqp_graph = branches;
        h->sc.sqp_max_iter = saved.sqp_max_iter < 2 ? saved.sqp_max_iter : 2;
        h->trial = true;
        for (int i = 0; i < 4; ++i) h->trial_cta[i] = cta[i];
        float ms_min = 1e30f;
        for (int rep = 0; rep < 3 && st == GPT_OK; ++rep) {
            // the solve updates xu and lambda in place: run it on scratch copies
            cudaError_t e = cudaMemcpyAsync(h->adj_h, d_xu, sizeof(float) * nxu, cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(h->adj_lam, d_lambda, sizeof(float) * nl, cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess) e = cudaEventRecord(e0, s);
            if (e != cudaSuccess) {
                st = cuda_err(e, "autotune");
                break;
            }
            std::vector<float> r = rho;
            st = sqp_run(h, B, h_N, d_goal, h->adj_lam, h->adj_h, r.data(), 1e-3f, nullptr, nullptr, nullptr, s);
            if (st == GPT_ERR_NONFINITE || st == GPT_ERR_FACTOR) st = GPT_OK;  // timing only
            if (st != GPT_OK) break;
            float ms = 0.f;
            e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) {
                st = cuda_err(e, "autotune timing");
                break;
            }
            if (rep > 0 && ms < ms_min) ms_min = ms;
        }
        h->trial = false;
        return ms_min;
    };
    // 1. the PCG kernel / cluster size with the default schedule
    uint8_t cta[4] = {0, 0, 0, 0};
    float best_ms = 1e30f;
    uint32_t best = cand[0];
    for (size_t ci = 0; ci < cand.size() && st == GPT_OK; ++ci) {
        const float ms = time_schedule(cand[ci], cta);
        if (st == GPT_OK && ms < best_ms) {
            best_ms = ms;
            best = cand[ci];
        }
    }
    // 2. the per-knot kernels' grids, one kernel at a time (coordinate descent): CTAs per SM from one
    // resident wave to the default 16 (a smaller grid gives each Schur warp a longer run of knots whose
    // inverses it reuses, and leaves no partial last wave); a change must gain 1 %
    static const uint8_t cta_cand[] = {4, 5, 6, 8};
    for (int which = 0; which < 4 && st == GPT_OK; ++which) {
        uint8_t keep = cta[which];
        for (uint8_t cv : cta_cand) {
            cta[which] = cv;
            const float ms = time_schedule(best, cta);
            if (st != GPT_OK) break;
            if (ms < 0.99f * best_ms) {
                best_ms = ms;
                keep = cv;
            }
        }
        cta[which] = keep;
    }
    // 3. for a graph solve whose branch count the caller left to the library (sqp_graph 1), the number of
    // concurrent part-batch branches per SQP iteration, 1, 2 or 4 (no more than the instances); a change
    // must gain 1 %
    uint32_t best_branches = 1;
    if (saved.sqp_graph == 1 && st == GPT_OK) {
        for (uint32_t kb : {2u, 4u}) {
            if (kb > B) break;
            branches = kb;
            const float ms = time_schedule(best, cta);
            if (st != GPT_OK) break;
            if (ms < 0.99f * best_ms) {
                best_ms = ms;
                best_branches = kb;
            }
        }
        branches = 1;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    h->sc = saved;
    h->profile = saved_profile;
    h->trial = false;
    if (st != GPT_OK) return st;
    bool found = false;
    for (auto &t : h->tuned)
        if (t.B == (int)B && t.total == total && t.maxN == maxN && t.minN == minN) {
            t.cluster = best;
            std::memcpy(t.cta, cta, sizeof(cta));
            t.branches = (uint8_t)best_branches;
            found = true;
        }
    if (!found)
        h->tuned.push_back({(int)B, total, maxN, minN, best, {cta[0], cta[1], cta[2], cta[3]}, (uint8_t)best_branches});
    if (h_cluster_out) *h_cluster_out = best;
    if (h_schedule_out) {
        for (int i = 0; i < 4; ++i) h_schedule_out[i] = (uint32_t)ctas_or_default(cta[i]);
        h_schedule_out[4] = saved.sqp_graph == 1 ? best_branches : saved.sqp_graph;
    }
    return GPT_OK;
}

gpt_status gpt_sqp_adjoint(gpt_handle *h, uint32_t B, const uint32_t *h_N, const float *d_goal, const float *d_xs,
                           const float *d_xu, const float *h_rho, const float *d_grad_xu_next, float *d_xu_next,
                           float *d_grad_goal, float *d_grad_qd, float *d_grad_r, float *d_grad_q_ee,
                           gpt_stream_t stream)
{
    if (!h || !h_N || !d_goal || !d_xs || !d_xu || !h_rho || !d_grad_xu_next || !d_grad_goal || !d_grad_qd ||
        !d_grad_r || !d_grad_q_ee)
        return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (h->sc.pcg_precond == 2) return set_err(GPT_ERR_BAD_ARG, "the adjoint runs with pcg_precond 0 or 1");
    BatchView bv;
    int maxN = 0, minN = 0;
    {
        const gpt_status st = setup_batch(h, B, h_N, h_rho, h_rho[0], bv, maxN, minN, s);
        if (st != GPT_OK) return st;
    }
    const ProblemParams P = to_params(h->pc);
    const SolverParams SP = to_solver(h->sc);
    const int ns = h->num_sms, T = bv.total_knots, nz = NX * T - NC;
    const bool f64 = SP.pcg_precond == 1 && SP.schur_fp64;
    const float *S_rows = f64 ? reinterpret_cast<const float *>(h->S64) : h->S;
    const int fmt = f64 ? 2 : 1;
    GPT_CUDA(cudaMemcpyAsync(h->xs, d_xs, sizeof(float) * NS * B, cudaMemcpyDeviceToDevice, s));
    // ---- the step at xu: K [dz; lambda] = [g; c]
    GPT_CUDA(launch_kkt(bv, P, d_xu, d_goal, h->xs, h->G, h->C, h->g, h->c, ns, s));
    if (f64)
        GPT_CUDA(launch_schur64(bv, h->G, h->C, h->g, h->c, h->S64, h->gamma64, nullptr, h->Ginv64, h->Ginv64c, ns,
                                s));
    else
        GPT_CUDA(launch_schur(1, bv, 0.f, h->G, h->C, h->g, h->c, h->S, nullptr, h->gamma, h->Ginv, h->Ginv64,
                              nullptr, SP.pcg_precond == 0 ? 1 : 0, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->adj_lam, 0, sizeof(float) * NS * T, s));
    GPT_CUDA(launch_pcg(bv, maxN, minN, fmt, (int)SP.pcg_precond, S_rows, nullptr, h->gamma, h->gamma64, h->adj_lam, h->lam64,
                        h->crw, (int)SP.pcg_max_iter, SP.pcg_tol, (int)SP.pcg_exit_mode, nullptr, nullptr, 0,
                        (int)SP.pcg_cluster_size, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->dz, 0, sizeof(float) * NX * T, s));
    GPT_CUDA(launch_dz(bv, h->Ginv, h->Ginv64, f64 ? h->Ginv64c : nullptr, h->C, h->g, nullptr, h->lam64, h->dz, ns,
                       s));
    if (d_xu_next) GPT_CUDA(launch_axpy(nz, -1.f, h->dz, d_xu, d_xu_next, ns, s));
    // ---- adjoint solve K mu = [h; 0], h = dl/d(dz) = -dl/dxu+; same S (recomputed), new gamma
    GPT_CUDA(cudaMemsetAsync(h->adj_h, 0, sizeof(float) * NX * T, s));
    GPT_CUDA(launch_axpy(nz, -1.f, d_grad_xu_next, nullptr, h->adj_h, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->adj_zero, 0, sizeof(float) * NS * T, s));
    if (f64)
        GPT_CUDA(launch_schur64(bv, h->G, h->C, h->adj_h, h->adj_zero, h->S64, h->adj_gamma64, nullptr, h->Ginv64,
                                h->Ginv64c, ns, s));
    else
        GPT_CUDA(launch_schur(1, bv, 0.f, h->G, h->C, h->adj_h, h->adj_zero, h->S, nullptr, h->adj_gamma, h->Ginv,
                              h->Ginv64, nullptr, SP.pcg_precond == 0 ? 1 : 0, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->adj_lam, 0, sizeof(float) * NS * T, s));
    GPT_CUDA(launch_pcg(bv, maxN, minN, fmt, (int)SP.pcg_precond, S_rows, nullptr, h->adj_gamma, h->adj_gamma64, h->adj_lam,
                        h->adj_lam64, h->crw, (int)SP.pcg_max_iter, SP.pcg_tol, (int)SP.pcg_exit_mode, nullptr,
                        nullptr, 0, (int)SP.pcg_cluster_size, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->adj_mu, 0, sizeof(float) * NX * T, s));
    GPT_CUDA(launch_dz(bv, h->Ginv, h->Ginv64, f64 ? h->Ginv64c : nullptr, h->C, h->adj_h, nullptr, h->adj_lam64,
                       h->adj_mu, ns, s));
    // ---- dl/dtheta = mu_z^T (dg/dtheta - dG/dtheta dz)
    GPT_CUDA(launch_adjoint_grad(bv, P, d_xu, d_goal, h->dz, h->adj_mu, d_grad_goal, h->adj_part, d_grad_qd,
                                 d_grad_r, d_grad_q_ee, ns, s));
    GPT_CUDA(cudaMemcpyAsync(h->h_st, h->st, sizeof(InstState) * B, cudaMemcpyDeviceToHost, s));
    GPT_CUDA(cudaStreamSynchronize(s));
    for (uint32_t b = 0; b < B; ++b) {
        const InstState &st = h->h_st[b];
        if (st.exit_flags & GPT_EXIT_FACTOR)
            return set_err(GPT_ERR_FACTOR, "(Q + rho I) or (R + rho I) not positive definite in the adjoint");
        if (st.exit_flags & 4u) return set_err(GPT_ERR_NONFINITE, "non-finite value in an adjoint solve");
        if (st.pcg_maxiter_count) return set_err(GPT_ERR_NONFINITE, "PCG reached pcg_max_iter in the adjoint");
    }
    return GPT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// MPC tracking loop (toplevel.cuh:507-796)
// ---------------------------------------------------------------------------

namespace {

TrackParams track_params(float timestep, float sim_step, float shift_threshold, double sim_us)
{
    TrackParams tp;
    tp.sim_us = sim_us;
    tp.shift_threshold = (double)(shift_threshold > 0.f ? shift_threshold : timestep);
    tp.timestep = (double)timestep;
    tp.sim_step = sim_step;
    const double t = sim_us * 1e-6;
    tp.n_sub = (uint32_t)(t / (double)sim_step);  // integrator.cuh:383
    tp.sim_last = (float)fmod(t, (double)sim_step);  // integrator.cuh:395
    return tp;
}

// Updates the shared clock runs before the longest trajectory is done: the host image of
// track_clock_kernel's arithmetic (the same doubles in the same order).
uint32_t track_update_count(const TrackParams &tp, uint32_t max_steps, uint32_t max_updates)
{
    double ts = 0.0;
    bool shifted = false;
    uint32_t off = 0, u = 0;
    while (u < max_updates && off < max_steps) {
        ts += tp.sim_us * 1e-6;
        if (!shifted && ts > tp.shift_threshold) {
            off++;
            shifted = true;
        }
        if (ts > tp.timestep) {
            shifted = false;
            ts = fmod(ts, tp.timestep);
        }
        u++;
    }
    return u;
}

}  // namespace

// One solve of every active instance on the handle's working buffers (gxu, glam, ggoal):
// the cached graph, or the host loop when graphs are off or profiling is on.
static gpt_status solve_on_workspace(gpt_handle *h, const SqpPlan &pl, cudaStream_t s)
{
    if (pl.SP.sqp_graph && !h->profile) {
        cudaGraphExec_t exec = nullptr;
        const gpt_status st = sqp_graph_for(h, pl, &exec);
        if (st != GPT_OK) return st;
        GPT_CUDA(cudaGraphLaunch(exec, s));
        return GPT_OK;
    }
    {
        const gpt_status st = enqueue_prologue(h, pl, h->ggoal, h->gxu, s);
        if (st != GPT_OK) return st;
    }
    for (uint32_t it = 0; it < pl.SP.sqp_max_iter; ++it) {
        const gpt_status st = enqueue_iteration(h, pl, h->ggoal, h->glam, h->gxu, s);
        if (st != GPT_OK) return st;
        GPT_CUDA(cudaMemcpyAsync(h->h_active, h->d_active, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        GPT_CUDA(cudaEventRecord(h->ev, s));
        GPT_CUDA(cudaEventSynchronize(h->ev));
        if (*h->h_active == 0) break;
    }
    if (h->profile) collect_phase_times(h);
    return GPT_OK;
}

extern "C" {

void gpt_default_track_config(gpt_track_config *o)
{
    if (!o) return;
    o->sim_period_us = 2000.f;      // perform_experiment.sh:29,46
    o->sim_step = 2e-4f;            // integrator.cuh:378
    o->shift_threshold = 0.f;       // settings.cuh:29 (1 * timestep)
    o->max_control_updates = 100000;  // toplevel.cuh:515
    o->jitter_solves = 0;
    o->rho_reset = 1e-3f;           // toplevel.cuh:579
}

}  // extern "C"

// The adjoint of one update's solve at its solution xu (the handle's gxu), on the loss of the update's
// horizon l = 1/2 sum_k |p(q_k+) - p*_k|^2 at xu+ = xu - dz: the steps of gpt_sqp_adjoint with the
// loss gradient formed on the device, the weight gradients added to d_wgrad and l to d_loss.  The
// solve's per-instance state is saved and restored around it.
static gpt_status enqueue_track_adjoint(gpt_handle *h, const SqpPlan &pl, float *d_wgrad, float *d_loss,
                                        cudaStream_t s)
{
    const BatchView &bv = pl.bv;
    const SolverParams &SP = pl.SP;
    const int ns = h->num_sms, T = bv.total_knots;
    const bool f64 = SP.pcg_precond == 1 && SP.schur_fp64;
    const float *S_rows = f64 ? reinterpret_cast<const float *>(h->S64) : h->S;
    const int fmt = f64 ? 2 : 1;
    GPT_CUDA(launch_track_adj_begin(bv, h->trk_rows, h->trk_clk, h->trk_stbak, s));
    // the step at the solution: K [dz; lambda] = [g; c]
    GPT_CUDA(launch_kkt(bv, pl.P, h->gxu, h->ggoal, h->xs, h->G, h->C, h->g, h->c, ns, s));
    if (f64)
        GPT_CUDA(launch_schur64(bv, h->G, h->C, h->g, h->c, h->S64, h->gamma64, nullptr, h->Ginv64, h->Ginv64c, ns,
                                s));
    else
        GPT_CUDA(launch_schur(1, bv, 0.f, h->G, h->C, h->g, h->c, h->S, nullptr, h->gamma, h->Ginv, h->Ginv64,
                              nullptr, SP.pcg_precond == 0 ? 1 : 0, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->adj_lam, 0, sizeof(float) * NS * T, s));
    GPT_CUDA(launch_pcg(bv, pl.maxN, pl.minN, fmt, (int)SP.pcg_precond, S_rows, nullptr, h->gamma, h->gamma64,
                        h->adj_lam, h->lam64, h->crw, (int)SP.pcg_max_iter, SP.pcg_tol, (int)SP.pcg_exit_mode, nullptr,
                        nullptr, 0, (int)SP.pcg_cluster_size, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->dz, 0, sizeof(float) * NX * T, s));
    GPT_CUDA(launch_dz(bv, h->Ginv, h->Ginv64, f64 ? h->Ginv64c : nullptr, h->C, h->g, nullptr, h->lam64, h->dz, ns,
                       s));
    // the adjoint solve K mu = [h; 0], h = dl/d(dz)
    GPT_CUDA(cudaMemsetAsync(h->adj_h, 0, sizeof(float) * NX * T, s));
    GPT_CUDA(launch_track_loss_grad(bv, h->gxu, h->dz, h->ggoal, h->adj_h, h->trk_kloss, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->adj_zero, 0, sizeof(float) * NS * T, s));
    if (f64)
        GPT_CUDA(launch_schur64(bv, h->G, h->C, h->adj_h, h->adj_zero, h->S64, h->adj_gamma64, nullptr, h->Ginv64,
                                h->Ginv64c, ns, s));
    else
        GPT_CUDA(launch_schur(1, bv, 0.f, h->G, h->C, h->adj_h, h->adj_zero, h->S, nullptr, h->adj_gamma, h->Ginv,
                              h->Ginv64, nullptr, SP.pcg_precond == 0 ? 1 : 0, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->adj_lam, 0, sizeof(float) * NS * T, s));
    GPT_CUDA(launch_pcg(bv, pl.maxN, pl.minN, fmt, (int)SP.pcg_precond, S_rows, nullptr, h->adj_gamma,
                        h->adj_gamma64, h->adj_lam, h->adj_lam64, h->crw, (int)SP.pcg_max_iter, SP.pcg_tol,
                        (int)SP.pcg_exit_mode, nullptr, nullptr, 0, (int)SP.pcg_cluster_size, ns, s));
    GPT_CUDA(cudaMemsetAsync(h->adj_mu, 0, sizeof(float) * NX * T, s));
    GPT_CUDA(launch_dz(bv, h->Ginv, h->Ginv64, f64 ? h->Ginv64c : nullptr, h->C, h->adj_h, nullptr, h->adj_lam64,
                       h->adj_mu, ns, s));
    // dl/dtheta = mu_z^T (dg/dtheta - dG/dtheta dz), added to d_wgrad
    GPT_CUDA(launch_adjoint_grad(bv, pl.P, h->gxu, h->ggoal, h->dz, h->adj_mu, h->trk_ggrad, h->adj_part, nullptr,
                                 nullptr, nullptr, ns, s, d_wgrad));
    GPT_CUDA(launch_track_adj_end(bv, h->trk_stbak, h->trk_kloss, d_loss, h->trk_inst, s));
    return GPT_OK;
}

// gpt_track_batched, and with d_wgrad non-null gpt_track_batched_adjoint
static gpt_status track_impl(gpt_handle *h, uint32_t B, const uint32_t *h_N, const uint32_t *h_S,
                             const float *d_eePos_traj, const float *d_xu_traj, float *d_xs,
                             const gpt_track_config *tc_in, float *d_err, uint32_t *d_log, uint32_t log_cap,
                             float *d_wgrad, float *d_loss, uint32_t *h_adj_fail, gpt_track_stats *h_stats,
                             cudaStream_t s)
{
    gpt_track_config tc;
    gpt_default_track_config(&tc);
    if (tc_in) tc = *tc_in;
    if (!(tc.sim_period_us > 0.f) || !(tc.sim_step > 0.f) || !(tc.shift_threshold >= 0.f) || !(tc.rho_reset > 0.f))
        return set_err(GPT_ERR_BAD_ARG, "sim_period_us, sim_step and rho_reset must be positive");
    if ((double)tc.sim_period_us * 1e-6 / (double)tc.sim_step > 1e6)
        return set_err(GPT_ERR_BAD_ARG, "more than 1e6 plant steps per control update");
    if (B == 0 || B > h->pc.max_batch) return set_err(GPT_ERR_CAPACITY, "batch exceeds handle capacity");
    uint32_t maxS = 0;
    h->h_trk_rows[0] = 0;
    for (uint32_t b = 0; b < B; ++b) {
        if (h_S[b] < h_N[b])
            return set_err(GPT_ERR_BAD_ARG, "traj_steps must be >= knot_points (runme.cu:151 skips shorter trajectories)");
        if ((uint64_t)h->h_trk_rows[b] + h_S[b] > 0x7fffffffu) return set_err(GPT_ERR_BAD_ARG, "trajectories too long");
        h->h_trk_rows[b + 1] = h->h_trk_rows[b] + (int)h_S[b];
        maxS = h_S[b] > maxS ? h_S[b] : maxS;
    }
    BatchView bv;
    int maxN = 0, minN = 0;
    {
        const gpt_status st = setup_batch(h, B, h_N, nullptr, tc.rho_reset, bv, maxN, minN, s);
        if (st != GPT_OK) return st;
    }
    const ProblemParams P = to_params(h->pc);
    SolverParams SP = to_solver(h->sc);
    apply_tuned(h, bv, maxN, minN, SP);
    const SqpPlan plan{bv, P, SP, maxN, minN, h->num_sms};
    if (d_wgrad && SP.pcg_precond == 2) return set_err(GPT_ERR_BAD_ARG, "the adjoint runs with pcg_precond 0 or 1");
    const TrackParams tp = track_params(h->pc.timestep, tc.sim_step, tc.shift_threshold, (double)tc.sim_period_us);
    const uint32_t n_updates = track_update_count(tp, maxS, tc.max_control_updates);
    const int ns = h->num_sms;

    GPT_CUDA(cudaMemcpyAsync(h->trk_rows, h->h_trk_rows, sizeof(int) * (B + 1), cudaMemcpyHostToDevice, s));
    GPT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(float) * (size_t)h->h_trk_rows[B], s));
    if (d_wgrad) GPT_CUDA(cudaMemsetAsync(d_wgrad, 0, sizeof(float) * 15 * B, s));
    if (d_loss) GPT_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(float) * B, s));
    GPT_CUDA(launch_track_start(bv, h->trk_rows, d_eePos_traj, d_xu_traj, h->gxu, h->trk_xu_old, h->ggoal, h->glam,
                                h->trk_clk, h->trk_inst, 1e-3f, 0, ns, s));
    if (tc.jitter_solves > 0) {  // toplevel.cuh:581-592
        SolverParams SPj = SP;
        SPj.pcg_tol = 1e-11f;
        SPj.pcg_max_iter = 10000;
        const SqpPlan pj{bv, P, SPj, maxN, minN, ns};
        for (uint32_t j = 0; j < tc.jitter_solves; ++j) {
            GPT_CUDA(launch_track_prep(bv, h->trk_rows, h->trk_clk, 1e-3f, 1, s));
            const gpt_status st = solve_on_workspace(h, pj, s);
            if (st != GPT_OK) return st;
            GPT_CUDA(launch_track_start(bv, h->trk_rows, d_eePos_traj, d_xu_traj, h->gxu, h->trk_xu_old, h->ggoal,
                                        h->glam, h->trk_clk, h->trk_inst, j + 1 == tc.jitter_solves ? 1e-3f : -1.f,
                                        1, ns, s));
        }
    }
    for (uint32_t u = 0; u < n_updates; ++u) {
        GPT_CUDA(launch_track_prep(bv, h->trk_rows, h->trk_clk, tc.rho_reset, 0, s));
        const gpt_status st = solve_on_workspace(h, plan, s);
        if (st != GPT_OK) return st;
        if (d_wgrad) {
            const gpt_status sa = enqueue_track_adjoint(h, plan, d_wgrad, d_loss, s);
            if (sa != GPT_OK) return sa;
        }
        GPT_CUDA(launch_track_tail(bv, h->trk_rows, h->trk_clk, tp, d_eePos_traj, d_xu_traj, d_xs, h->gxu,
                                   h->trk_xu_old, h->ggoal, h->glam, h->adj_h, d_err, h->trk_inst, d_log, log_cap, s));
    }
    GPT_CUDA(launch_track_final(bv, d_xs, h->ggoal, h->trk_inst, s));
    GPT_CUDA(cudaMemcpyAsync(h->h_trk_inst, h->trk_inst, sizeof(TrackInst) * B, cudaMemcpyDeviceToHost, s));
    GPT_CUDA(cudaStreamSynchronize(s));
    bool nonfinite = false;
    for (uint32_t b = 0; b < B; ++b) {
        const TrackInst &ti = h->h_trk_inst[b];
        if (ti.nonfinite) nonfinite = true;
        if (h_adj_fail) h_adj_fail[b] = ti.adj_fail;
        if (!h_stats) continue;
        gpt_track_stats &o = h_stats[b];
        o.control_updates = ti.updates;
        o.shifts = ti.shifts;
        o.sqp_iters_total = ti.sqp_iters;
        o.pcg_iters_total = ti.pcg_iters;
        o.ls_fail_total = ti.ls_fail;
        o.pcg_maxiter_total = ti.pcg_maxiter;
        o.rho_exits = ti.rho_exits;
        o.nonfinite = ti.nonfinite;
        o.tracking_error_mean = ti.shifts ? ti.err_sum / (float)ti.shifts : 0.f;
        o.final_tracking_error = ti.final_err;
        o.rho_final = ti.rho;
    }
    if (nonfinite) return set_err(GPT_ERR_NONFINITE, "non-finite merit or PCG reduction in a tracking solve");
    return GPT_OK;
}

extern "C" {

gpt_status gpt_track_batched(gpt_handle *h, uint32_t B, const uint32_t *h_N, const uint32_t *h_S,
                             const float *d_eePos_traj, const float *d_xu_traj, float *d_xs,
                             const gpt_track_config *tc, float *d_err, uint32_t *d_log, uint32_t log_cap,
                             gpt_track_stats *h_stats, gpt_stream_t stream)
{
    if (!h || !h_N || !h_S || !d_eePos_traj || !d_xu_traj || !d_xs || !d_err)
        return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    return track_impl(h, B, h_N, h_S, d_eePos_traj, d_xu_traj, d_xs, tc, d_err, d_log, log_cap, nullptr, nullptr,
                      nullptr, h_stats, (cudaStream_t)stream);
}

gpt_status gpt_track_batched_adjoint(gpt_handle *h, uint32_t B, const uint32_t *h_N, const uint32_t *h_S,
                                     const float *d_eePos_traj, const float *d_xu_traj, float *d_xs,
                                     const gpt_track_config *tc, float *d_err, uint32_t *d_log, uint32_t log_cap,
                                     float *d_weight_grad, float *d_loss, uint32_t *h_adjoint_fail,
                                     gpt_track_stats *h_stats, gpt_stream_t stream)
{
    if (!h || !h_N || !h_S || !d_eePos_traj || !d_xu_traj || !d_xs || !d_err || !d_weight_grad)
        return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    return track_impl(h, B, h_N, h_S, d_eePos_traj, d_xu_traj, d_xs, tc, d_err, d_log, log_cap, d_weight_grad,
                      d_loss, h_adjoint_fail, h_stats, (cudaStream_t)stream);
}

gpt_status gpt_track(gpt_handle *h, uint32_t N, uint32_t S, const float *d_eePos_traj, const float *d_xu_traj,
                     float *d_xs, const gpt_track_config *tc, float *d_err, uint32_t *d_log, uint32_t log_cap,
                     gpt_track_stats *h_stats, gpt_stream_t stream)
{
    return gpt_track_batched(h, 1, &N, &S, d_eePos_traj, d_xu_traj, d_xs, tc, d_err, d_log, log_cap, h_stats, stream);
}

gpt_status gpt_simulate(gpt_handle *h, uint32_t N, float *d_xs, const float *d_xu, double time_offset_us,
                        double sim_time_us, float sim_step, gpt_stream_t stream)
{
    if (!h || !d_xs || !d_xu) return set_err(GPT_ERR_BAD_ARG, "null argument");
    DeviceGuard dg(h->device);
    if (!check_n(h, N)) return set_err(GPT_ERR_BAD_ARG, "knot_points out of range");
    if (!(sim_step > 0.f) || !(sim_time_us >= 0.0) || !(time_offset_us >= 0.0) ||
        sim_time_us * 1e-6 / (double)sim_step > 1e6)
        return set_err(GPT_ERR_BAD_ARG, "sim_step must be positive, times non-negative, <= 1e6 plant steps");
    const TrackParams tp = track_params(h->pc.timestep, sim_step, 0.f, sim_time_us);
    GPT_CUDA(launch_simulate_one((int)N, tp, time_offset_us, d_xs, d_xu, (cudaStream_t)stream));
    return GPT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// rigid-body library kernels and trajectory files
// ---------------------------------------------------------------------------

extern "C" {

gpt_status gpt_end_effector_positions(uint32_t n, const float *d_x, uint32_t stride, float *d_pose,
                                      gpt_stream_t stream)
{
    if (n == 0) return GPT_OK;
    if (!d_x || !d_pose) return set_err(GPT_ERR_BAD_ARG, "null argument");
    if (stride < 7 || n > (1u << 28)) return set_err(GPT_ERR_BAD_ARG, "row_stride must be >= 7 and n <= 2^28");
    GPT_CUDA(launch_ee_pose(n, d_x, stride, d_pose, (cudaStream_t)stream));
    return GPT_OK;
}

gpt_status gpt_forward_dynamics(uint32_t n, const float *d_xu, uint32_t stride, float *d_qdd, gpt_stream_t stream)
{
    if (n == 0) return GPT_OK;
    if (!d_xu || !d_qdd) return set_err(GPT_ERR_BAD_ARG, "null argument");
    if (stride < (uint32_t)NX || n > (1u << 28)) return set_err(GPT_ERR_BAD_ARG, "row_stride must be >= 21 and n <= 2^28");
    GPT_CUDA(launch_fd(n, d_xu, stride, d_qdd, (cudaStream_t)stream));
    return GPT_OK;
}

gpt_status gpt_forward_dynamics_gradient(uint32_t n, const float *d_xu, uint32_t stride, float *d_qdd, float *d_df,
                                         gpt_stream_t stream)
{
    if (n == 0) return GPT_OK;
    if (!d_xu || !d_qdd || !d_df) return set_err(GPT_ERR_BAD_ARG, "null argument");
    if (stride < (uint32_t)NX || n > (1u << 26)) return set_err(GPT_ERR_BAD_ARG, "row_stride must be >= 21 and n <= 2^26");
    GPT_CUDA(launch_fd_grad(n, d_xu, stride, d_qdd, d_df, (cudaStream_t)stream));
    return GPT_OK;
}

gpt_status gpt_read_csv(const char *path, float *h_out, size_t capacity, uint32_t *h_rows, uint32_t *h_cols)
{
    if (!path || !h_rows || !h_cols) return set_err(GPT_ERR_BAD_ARG, "null argument");
    *h_rows = 0;
    *h_cols = 0;
    FILE *f = std::fopen(path, "r");
    if (!f) return set_err(GPT_ERR_BAD_ARG, std::string("cannot open ") + path);
    std::vector<float> vals;
    std::string line;
    size_t rows = 0, cols = 0;
    bool ragged = false;
    int ch;
    while (true) {
        line.clear();
        while ((ch = std::fgetc(f)) != EOF && ch != '\n') line.push_back((char)ch);
        if (line.empty() && ch == EOF) break;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) {
            if (ch == EOF) break;
            continue;
        }
        // comma-separated fields, each parsed from its leading float (std::stof); like
        // std::getline(ss, val, ','), a trailing comma ends the row without an empty field
        size_t n = 0, pos = 0;
        while (pos < line.size()) {
            const size_t end = line.find(',', pos);
            const std::string field = line.substr(pos, end == std::string::npos ? std::string::npos : end - pos);
            vals.push_back(std::strtof(field.c_str(), nullptr));
            ++n;
            if (end == std::string::npos) break;
            pos = end + 1;
        }
        if (rows == 0) cols = n;
        else if (n != cols) ragged = true;
        ++rows;
        if (ch == EOF) break;
    }
    std::fclose(f);
    if (ragged) return set_err(GPT_ERR_BAD_ARG, "rows of unequal length");
    *h_rows = (uint32_t)rows;
    *h_cols = (uint32_t)cols;
    if (!h_out) return GPT_OK;
    if (capacity < vals.size()) return set_err(GPT_ERR_CAPACITY, "output capacity below rows x cols");
    std::copy(vals.begin(), vals.end(), h_out);
    return GPT_OK;
}

}  // extern "C"
