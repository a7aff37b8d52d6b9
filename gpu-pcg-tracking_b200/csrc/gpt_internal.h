// gpt_internal.h -- launchers shared between the kernel files and the C-ABI.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "gpt_common.cuh"

namespace gpt {

constexpr int MAX_PCG_KNOTS = 512;  // horizon limit of the library (16-CTA cluster x 32 knots)
constexpr int PCG_KPC_MAX = 128;    // knots per CTA held in shared memory by the PCG
constexpr int PCG_KPC_STAIR = 64;   // with the stair preconditioner (its Pinv blocks staged too)
constexpr int PCG_WARP_PAIR = 32;   // pcg_cluster_size value selecting pcg_pair_kernel (one 128-thread CTA per instance)
constexpr int PCG_WARP_QUAD = 64;   // pcg_cluster_size value selecting pcg_quad_kernel (four warps factor four parts)

// SQP control constants (settings.cuh:31-50 and the -D flags of perform_experiment.sh:42-58)
struct SolverParams {
    uint32_t sqp_max_iter;
    uint32_t pcg_max_iter;
    float pcg_tol;
    uint32_t pcg_exit_mode;
    float rho_factor, rho_max, rho_min;
    uint32_t pcg_cluster_size;  // 0: chosen from N and the batch size
    uint32_t pcg_precond;       // 0 block-Jacobi (reference), 1 chunk block-tridiagonal LDL^T
    uint32_t schur_fp64;        // with pcg_precond 1: FP64 Schur formation and rows
    uint32_t sqp_graph;         // the SQP loop as one CUDA graph with a device-side while loop
    // launch schedule of the per-knot kernels: CTAs per SM of the grid-stride launches (KKT, FP64 Schur,
    // merit, dz); the grid is ctas_per_sm x SMs CTAs, each warp taking knots strided by the grid (KKT,
    // merit, dz) or a contiguous run of total / grid-warps knots (Schur, whose inverses a run shares).
    // 0 = 16.  Chosen by gpt_autotune.
    uint8_t cta_kkt, cta_schur, cta_merit, cta_dz;
};
inline int ctas_or_default(uint8_t v) { return v ? (int)v : 16; }

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize >= smem_bytes, and NonPortableClusterSizeAllowed when
// cluster16) for func on the CURRENT device, once per (kernel, device); thread-safe.  Function
// attributes apply to the device that is current when they are set, so a per-process flag is not enough
// when handles live on several devices.
cudaError_t ensure_func_attrs(const void *func, size_t smem_bytes, bool cluster16 = false);

// full_g false: only the position block of each Q_k is written (the SQP loop, after launch_kkt_gconst
// wrote the rest of G for the same view and weights)
cudaError_t launch_kkt(const BatchView &bv, const ProblemParams &P, const float *xu, const float *goal,
                       const float *xs, float *G, float *C, float *g, float *c, int num_sms, cudaStream_t s,
                       int ctas_per_sm = 16, bool full_g = true);
cudaError_t launch_kkt_gconst(const BatchView &bv, const ProblemParams &P, float *G, int num_sms, cudaStream_t s);
// Ginv64 (optional) receives the inverses in FP64; need_pinv = 0 skips the theta inversion in mode 1
cudaError_t launch_schur(int mode, const BatchView &bv, float rho_scalar, const float *G, const float *C,
                         const float *g, const float *c, float *S, float *Pinv, float *gamma, float *Ginv,
                         double *Ginv64, float *csc_val, int need_pinv, int num_sms, cudaStream_t s);
size_t pcg_cluster_smem_bytes(int kpc);
int pcg_pick_cluster(int maxN, int B, int num_sms, int requested);
// fmt 0: S and Pinv in the reference 3-block layout; fmt 1: packed rows (PK floats per knot) in S
// precond 0: block-Jacobi with the given Pinv; 1: exact block-tridiagonal LDL^T of each CTA's chunk;
// 2: the stair preconditioner (Pinv's diagonal and off-diagonal blocks of gpt_form_ss, fmt 0 only)
// cr_ws: FP64 workspace of 2 x 196 doubles per knot of the batch (the cyclic-reduction couplings of
// precond 1, the warp-pair kernel's factors and vectors, the partitioned kernel's factors, vectors and
// coupling blocks; unused by precond 0)
// fmt 0: reference 3-block rows (S, Pinv floats); 1: packed FP32 rows (PK); 2: packed FP64 rows (PK64,
// S points at doubles) with FP64 gamma64 -- chain preconditioner only.  cluster_size PCG_WARP_PAIR runs
// pcg_pair_kernel (precond 1, fmt 1 or 2; cr_ws holds its factors and FP64 vectors)
cudaError_t launch_pcg(const BatchView &bv, int max_n_knots, int min_n_knots, int fmt, int precond, const float *S,
                       const float *Pinv, const float *gamma, const double *gamma64, float *lambda, double *lambda64,
                       double *cr_ws, int max_iter, float tol, int exit_mode, uint32_t *out_iters, uint32_t *pcg_log,
                       int log_stride, int cluster_size, int num_sms, cudaStream_t s);
// lambda64 (optional) replaces lambda when given; Ginv64c (optional): the compact inverses of
// launch_schur64 (GC64 doubles per knot), with Ginv64 holding only the blocks its flags name
cudaError_t launch_dz(const BatchView &bv, const float *Ginv, const double *Ginv64, const double *Ginv64c,
                      const float *C, const float *g, const float *lambda, const double *lambda64, float *dz,
                      int num_sms, cudaStream_t s, int ctas_per_sm = 16);
cudaError_t launch_merit(const BatchView &bv, const ProblemParams &P, int n_alpha, const float *xu, const float *dz,
                         const float *goal, const float *xs, float *knot_merit, int num_sms, cudaStream_t s,
                         int ctas_per_sm = 16);
cudaError_t launch_accept(const BatchView &bv, int mode, const SolverParams &SP, const float *knot_merit,
                          const float *dz, float *xu, float *merits_out, uint32_t *active_count, int num_sms,
                          cudaStream_t s);
cudaError_t launch_init(const BatchView &bv, const float *xu, float *xs, int num_sms, cudaStream_t s);
// FP64 Schur complement for the exact-preconditioner PCG: packed rows (PK64 doubles per knot), gamma
// (FP64), the inverses in compact form (Ginv64c, GC64 doubles per knot; a block that is not
// (block) diagonal in the full layout of Ginv64 instead; Ginv FP32 in the full layout too when
// non-null); rho from bv.st
cudaError_t launch_schur64(const BatchView &bv, const float *G, const float *C, const float *g, const float *c,
                           double *S64, double *gamma64, float *Ginv, double *Ginv64, double *Ginv64c, int num_sms,
                           cudaStream_t s, int ctas_per_sm = 16);
// adjoint of the SQP step (gpt_adjoint.cu): per-knot goal gradients, per-instance weight gradients;
// part holds adjoint_part_floats() floats per knot
// (wacc non-null: the 15 weight gradients of each active instance are added to wacc[15 b ..] instead of
// written to grad_qd / grad_r / grad_qee)
cudaError_t launch_adjoint_grad(const BatchView &bv, const ProblemParams &P, const float *xu, const float *goal,
                                const float *dz, const float *mu, float *grad_goal, float *part, float *grad_qd,
                                float *grad_r, float *grad_qee, int num_sms, cudaStream_t s, float *wacc = nullptr);
cudaError_t launch_axpy(int n, float alpha, const float *x, const float *a, float *out, int num_sms, cudaStream_t s);
size_t adjoint_part_floats();
// reference 3-block FP32 rows -> FP64 packed rows (PK64) and gamma64 (input of the warp-pair PCG)
cudaError_t launch_pack_rows64(int N, const float *S, const float *gamma, double *S64, double *gamma64, int num_sms,
                               cudaStream_t s);

// MPC tracking loop (gpt_track.cu).  The loop's clock is shared by the batch: every instance
// advances on the same schedule; instance b stops once the trajectory offset reaches its length.
struct TrackClock {
    double time_since;     // time since the last timestep (toplevel.cuh:524)
    double prev_sim_us;    // previous update's simulated time (toplevel.cuh:523)
    double sim_offset_us;  // this update's plant time offset into the previous solution
    uint32_t shifted, traj_offset, start_offset, do_shift, updates;
};
struct TrackInst {  // per-instance totals over the loop
    uint32_t updates, sqp_iters, pcg_iters, ls_fail, pcg_maxiter, rho_exits, nonfinite, shifts;
    float err_sum, final_err, rho;
    uint32_t adj_fail;  // updates whose adjoint solve failed (gpt_track_batched_adjoint)
};
struct TrackParams {
    double sim_us;           // SIMULATION_PERIOD
    double shift_threshold;  // SHIFT_THRESHOLD (s)
    double timestep;         // the solver's timestep, as double (track's arithmetic)
    float sim_step;          // plant step, 2e-4 s
    float sim_last;          // fmod(sim time, sim_step): the final partial step
    uint32_t n_sub;          // floor(sim time / sim_step)
};
cudaError_t launch_track_start(const BatchView &bv, const int *rows, const float *eePos_traj, const float *xu_traj,
                               float *xu, float *xu_old, float *goal, float *lambda, TrackClock *clk, TrackInst *inst,
                               float rho0, int reset_xu_only, int num_sms, cudaStream_t s);
cudaError_t launch_track_prep(const BatchView &bv, const int *rows, const TrackClock *clk, float rho_reset,
                              int all_live, cudaStream_t s);
cudaError_t launch_track_tail(const BatchView &bv, const int *rows, TrackClock *clk, const TrackParams &tp,
                              const float *eePos_traj, const float *xu_traj, float *xs, float *xu, float *xu_old,
                              float *goal, float *lambda, float *tmp, float *errors, TrackInst *inst,
                              uint32_t *iters_log, uint32_t log_cap, cudaStream_t s);
cudaError_t launch_track_final(const BatchView &bv, const float *xs, const float *goal, TrackInst *inst, cudaStream_t s);
// the adjoint of each update's solve (gpt_track_batched_adjoint): begin saves the per-solve state and
// marks the instances that track this update active; loss_grad writes h = dl/d(dz) = -dl/dxu+ of the
// update's horizon loss l = 1/2 sum_k |p(q_k - dz_q,k) - p*_k|^2 (q entries only) and each knot's
// term of l; end adds each live instance's l to loss, counts failed adjoint solves and restores the state
cudaError_t launch_track_adj_begin(const BatchView &bv, const int *rows, const TrackClock *clk, InstState *bak,
                                   cudaStream_t s);
cudaError_t launch_track_loss_grad(const BatchView &bv, const float *xu, const float *dz, const float *goal, float *h,
                                   float *kloss, int num_sms, cudaStream_t s);
cudaError_t launch_track_adj_end(const BatchView &bv, const InstState *bak, const float *kloss, float *loss,
                                 TrackInst *inst, cudaStream_t s);
// stair preconditioner's off-diagonal Pinv blocks (gato_form_ss_inner), reference 3-block rows
cudaError_t launch_form_ss(const BatchView &bv, const float *S, float *Pinv, int num_sms, cudaStream_t s);
// batched rigid-body library kernels (gpt_grid.cu)
cudaError_t launch_ee_pose(uint32_t n, const float *x, uint32_t stride, float *pose, cudaStream_t s);
cudaError_t launch_fd(uint32_t n, const float *xu, uint32_t stride, float *qdd, cudaStream_t s);
cudaError_t launch_fd_grad(uint32_t n, const float *xu, uint32_t stride, float *qdd, float *df, cudaStream_t s);
cudaError_t launch_simulate_one(int N, const TrackParams &tp, double t0_us, float *xs, const float *xu,
                                cudaStream_t s);

}  // namespace gpt

#include "../../include/gpt.h"

namespace gpt {
// for C-ABI entry points defined outside gpt_api.cu: the error text gpt_last_error()
// returns, and the device-side form of a problem config
gpt_status record_error(gpt_status st, const char *msg);
// per-iteration scalars of gpt_sqp_solve_batched_trace: phase 0 (before an iteration) records rho,
// the iterate's merit and the activity; phase 1 (after it) the line-search merits (merits, 8 per
// instance), the accepted step (the accept kernel's argmin), the next rho and the PCG count
cudaError_t launch_trace_record(const BatchView &bv, int phase, const float *merits, gpt_iterate_record *rec,
                                int num_sms, cudaStream_t s);
ProblemParams problem_params(const gpt_problem_config &pc);
}  // namespace gpt
