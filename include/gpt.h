/*
 * gpt.h -- C ABI of the B200-native SQP inner loop for 7-DOF iiwa
 * end-effector tracking (a drop-in for gpu-pcg-tracking's sqpSolve path).
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream, never
 * exits, and returns a gpt_status.  Device pointers are named d_*, host
 * pointers h_*.  All floating-point buffers are float32 in the reference's
 * layouts (column-major blocks, knots contiguous):
 *
 *   xu        [21N-7]      x_0 u_0 x_1 u_1 ... x_{N-1}      (toplevel.cuh:512)
 *   eePos     [6N]         goal xyz + rpy per knot           (runme.cu:153-157)
 *   lambda    [14N]        Schur-system multipliers (warm start, in/out)
 *   G         [245N-49]    {Q_k, R_k}           (toplevel.cuh:46)
 *   C         [294(N-1)]   {-A_k, -B_k}         (toplevel.cuh:47)
 *   g         [21N-7]      {q_k, r_k}           (toplevel.cuh:48)
 *   c         [14N]        defects              (toplevel.cuh:49)
 *   S, Pinv   [588N]       3 blocks per row     (toplevel.cuh:103,124)
 *   gamma     [14N]
 *   dz        [21N-7]                           (toplevel.cuh:50)
 *
 * Batched calls concatenate instances knot by knot: instance b with horizon
 * N_b starts at knot K_b = N_0 + ... + N_{b-1}, i.e. at float offset 21 K_b
 * of xu (slot of 21 N_b floats, the last 7 unused), 6 K_b of eePos and
 * 14 K_b of lambda.
 */
#ifndef GPT_H
#define GPT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *gpt_stream_t; /* same type as cudaStream_t */
typedef struct gpt_handle gpt_handle;

typedef enum gpt_status {
    GPT_OK = 0,
    GPT_ERR_BAD_ARG = 1,     /* null pointer, size out of range, wrong state/control size */
    GPT_ERR_CUDA = 2,        /* a CUDA runtime call failed; see gpt_last_error() */
    GPT_ERR_NO_DEVICE = 3,   /* no CUDA device / library built without a usable GPU */
    GPT_ERR_CAPACITY = 4,    /* request exceeds the handle's preallocated workspace */
    GPT_ERR_NONFINITE = 5,   /* a NaN/Inf appeared (reported per instance in gpt_sqp_stats) */
    GPT_ERR_FACTOR = 6       /* a factorisation failed (matrix not definite) */
} gpt_status;

/* gpt_sqp_stats.exit_flags bits */
#define GPT_EXIT_RHO_MAX 1u      /* line search failed until rho > rho_max (toplevel.cuh:396-405) */
#define GPT_EXIT_PCG_MAXITER 2u  /* at least one PCG solve hit its iteration limit */
#define GPT_EXIT_NONFINITE 4u    /* NaN/Inf in a merit or a PCG reduction */
#define GPT_EXIT_ITER_LIMIT 8u   /* SQP_MAX_ITER iterations done (toplevel.cuh:254) */
#define GPT_EXIT_FACTOR 16u      /* (Q + rho I) or (R + rho I) was not positive definite (a non-positive or vanishing
                                    pivot in the Schur complement's inverses, e.g. rho = 0 with a rank-deficient
                                    cost block); the instance stops and the call returns GPT_ERR_FACTOR */

/* Problem description; the reference's compile-time macros become fields.
 * Replaces settings.cuh and the -D flags of perform_experiment.sh:42-58. */
typedef struct gpt_problem_config {
    uint32_t state_size;       /* must be 14 (settings.cuh:4) */
    uint32_t control_size;     /* must be 7 (grid::NUM_JOINTS) */
    uint32_t max_knot_points;  /* capacity: largest horizon N (2..512) */
    uint32_t max_batch;        /* capacity: instances per batched call */
    float timestep;            /* runme.cu:65 uses 1/64 */
    uint32_t integrator;       /* 0 explicit Euler (reference default), 1 semi-implicit */
    float q_ee;                /* end-effector position weight (1 in the reference) */
    float qd_cost;             /* QD_COST */
    float r_cost;              /* R_COST */
    float mu;                  /* merit penalty, 10 in toplevel.cuh:54 */
    uint32_t ref_terminal;     /* 1 (reference): terminal Q,q at x_{N-2} with the target the reference's kernel
                                  actually reads, Q_{N-2}[0][0..2] (goal_{N-1} is overwritten in its shared
                                  buffer, schur.cuh:413-425, iiwa_eepos_plant.cuh:396-401);
                                  0: at x_{N-1} with target goal_{N-1} */
} gpt_problem_config;

/* SQP / PCG controls (settings.cuh:31-50; pcg_config of GPU-PCG, toplevel.cuh:573-576) */
typedef struct gpt_solver_config {
    uint32_t sqp_max_iter;     /* SQP_MAX_ITER, 40 */
    uint32_t pcg_max_iter;     /* PCG_MAX_ITER */
    float pcg_exit_tol;        /* PCG_EXIT_TOL */
    uint32_t pcg_exit_mode;    /* 0: ||r||_2 <= tol ||gamma||_2; 1: |r^T Pinv r| < tol */
    float rho_factor;          /* RHO_FACTOR */
    float rho_max;             /* RHO_MAX */
    float rho_min;             /* RHO_MIN */
    uint32_t pcg_cluster_size; /* CTAs per instance in the PCG (1,2,4,8,16); GPT_PCG_WARP_PAIR / GPT_PCG_WARP_QUAD:
                                  one 128-thread CTA per instance, factorisation by two / four warps (pcg_precond 1
                                  only); 0 = chosen by the library (gpt_autotune's choice for the batch shape, else
                                  1 ... 16) */
    uint32_t pcg_precond;      /* 0: block-Jacobi Pinv (the reference's, oldschur.cuh:926-933);
                                  1 (default): exact block-tridiagonal LDL^T of each CTA's chunk of knots */
    uint32_t schur_fp64;       /* SQP loop and adjoint with pcg_precond 1: 1 (default) forms and stores the
                                  Schur complement in FP64; 0 in FP32 as the reference does (schur.cuh:391-524).
                                  FP32 formation moves the solution by ~cond(S) x 1e-7 (~1e-2 at cond 1e7) */
    uint32_t sqp_graph;        /* 1 (default): a solve runs as one CUDA graph (built on the first call of each
                                  batch shape and cached) whose while node repeats the SQP iteration on the
                                  device, split in the part-batch branches gpt_autotune chose for the shape
                                  (one when it was not tuned); K = 2 .. 8: the same graph with the batch split
                                  in K parts whose iterations run on concurrent branches (one part's PCG
                                  overlaps the others' KKT, Schur and merit kernels; identical results); 0:
                                  one host
                                  synchronisation per SQP iteration, as the reference loop.  Profiling
                                  (gpt_set_profiling) uses the host loop. */
} gpt_solver_config;

/* One sqpSolve's outcome (the reference returns a tuple, toplevel.cuh:502) */
typedef struct gpt_sqp_stats {
    uint32_t sqp_iters;          /* sqp_iter */
    uint32_t exit_flags;         /* GPT_EXIT_* */
    uint32_t pcg_iters_total;
    uint32_t pcg_maxiter_count;  /* number of PCG solves that stopped at pcg_max_iter */
    uint32_t ls_fail_count;
    float merit_initial;
    float merit_final;
    float rho_final;
} gpt_sqp_stats;

/* pcg_cluster_size value: the PCG of one instance in one 128-thread CTA whose first two warps factor S
 * from both ends of the horizon at once (twisted block LDL^T), so that all instances of a large batch run
 * concurrently; same iteration and preconditioner (exact inverse of S) as pcg_cluster_size 1. */
#define GPT_PCG_WARP_PAIR 32u

/* pcg_cluster_size value: the PCG of one instance in one 128-thread CTA whose four warps each factor about a
 * quarter of the horizon (partitioned block LDL^T: three separator knots, a 3-block reduced system), so every
 * SM sub-partition factors and each warp's chain is half the warp-pair kernel's; same iteration and
 * preconditioner (exact inverse of S) as pcg_cluster_size 1. */
#define GPT_PCG_WARP_QUAD 64u

/* Default configs: the reference's logged experiment settings (dt 1/64, Euler,
 * QD = R = 1e-4, RHO_FACTOR 1.2, RHO_MAX 10, RHO_MIN 1e-3, SQP_MAX_ITER 40). */
void gpt_default_problem_config(gpt_problem_config *out);
void gpt_default_solver_config(gpt_solver_config *out);

/* Handle with a workspace sized for max_batch x max_knot_points; no
 * allocation happens inside the solve calls.  Replaces the per-call
 * cudaMalloc/cublasCreate of sqpSolve (toplevel.cuh:67-141) and
 * gato_plant::initializeDynamicsConstMem (rbdfiles/iiwa_eepos_plant.cuh:66-70). */
gpt_status gpt_create(const gpt_problem_config *problem, const gpt_solver_config *solver, gpt_handle **out);
gpt_status gpt_destroy(gpt_handle *h);
gpt_status gpt_set_solver_config(gpt_handle *h, const gpt_solver_config *solver);

/* Cost weights of later calls: end-effector position weight, QD_COST and
 * R_COST (no reference counterpart: the reference compiles them in,
 * iiwa_eepos_plant.cuh:58-64). */
gpt_status gpt_set_cost_weights(gpt_handle *h, float q_ee, float qd_cost, float r_cost);
const char *gpt_last_error(void);
const char *gpt_version(void);

/*
 * One SQP solve of one instance: replaces
 *   sqpSolve<T>(state_size, control_size, knot_points, timestep, d_eePos_traj, d_lambda, d_xu,
 *               d_dynMem_const, pcg_config&, T& rho, T rho_reset)      (toplevel.cuh:24-25)
 * d_xu and d_lambda are updated in place; *h_rho is in/out like the
 * reference's T& rho.  h_pcg_iters / h_pcg_exit (optional, length
 * sqp_max_iter) receive the per-iteration PCG iteration counts and max-iter
 * flags (the tuple's pcg_iter_vec / pcg_exit_vec).  Stream-ordered; returns
 * after the solve completed (the stats are host values).
 */
gpt_status gpt_sqp_solve(gpt_handle *h, uint32_t knot_points, const float *d_eePos_traj, float *d_lambda,
                         float *d_xu, float *h_rho, float rho_reset, gpt_sqp_stats *h_stats,
                         uint32_t *h_pcg_iters, uint8_t *h_pcg_exit, gpt_stream_t stream);

/* Many independent instances of uneven horizon in one call (no reference
 * counterpart; the reference solves one instance per sqpSolve).  h_rho and
 * h_stats have `batch` entries. */
gpt_status gpt_sqp_solve_batched(gpt_handle *h, uint32_t batch, const uint32_t *h_knot_points,
                                 const float *d_eePos_traj, float *d_lambda, float *d_xu, float *h_rho,
                                 float rho_reset, gpt_sqp_stats *h_stats, gpt_stream_t stream);

/* Scalars of one SQP iteration of one instance, recorded by gpt_sqp_solve_batched_trace */
typedef struct gpt_iterate_record {
    float rho;          /* rho of this iteration's Schur complement ((Q + rho I), (R + rho I)) */
    float rho_next;     /* rho after the schedule of toplevel.cuh:396-412 (the next iteration's) */
    float merit_prev;   /* merit of the iterate: the line search must go below it (toplevel.cuh:384-392) */
    float merits[8];    /* line-search merits of xu + alpha_p dz, alpha_p = -2^-p (toplevel.cuh:357-374) */
    float alpha;        /* accepted step; 0 when the line search failed (xu unchanged) */
    uint32_t active;    /* 1 when the instance ran this iteration; the other fields are then defined */
    uint32_t pcg_iters; /* PCG iterations of this iteration's linear solve */
} gpt_iterate_record;

/* gpt_sqp_solve_batched with every SQP iterate recorded (no reference counterpart: the reference
 * returns only per-iteration PCG counts, toplevel.cuh:502).  Same kernels and results; the loop is
 * driven from the host (one synchronisation per iteration).  For the first trace_iters iterations
 * it writes, per iteration i (T = total knots of the batch, batch layout of gpt_sqp_solve_batched):
 *   d_trace_xu     [trace_iters][21 T]     xu at the start of iteration i
 *   d_trace_lambda [trace_iters][14 T]     the FP64 multipliers of iteration i's linear solve (dz's input)
 *   d_trace_dz     [trace_iters][21 T]     the step dz of iteration i
 *   d_trace_rec    [trace_iters][batch]    the iteration's scalars
 * Any of the four may be NULL.  Vectors of an instance with rec.active == 0 in iteration i are not
 * written. */
gpt_status gpt_sqp_solve_batched_trace(gpt_handle *h, uint32_t batch, const uint32_t *h_knot_points,
                                       const float *d_eePos_traj, float *d_lambda, float *d_xu, float *h_rho,
                                       float rho_reset, gpt_sqp_stats *h_stats, uint32_t trace_iters,
                                       float *d_trace_xu, double *d_trace_lambda, float *d_trace_dz,
                                       gpt_iterate_record *d_trace_rec, gpt_stream_t stream);

/* Autotuner (no reference counterpart).  Picks, by timing two SQP iterations of this batch (on copies of
 * d_xu and d_lambda; the inputs are not modified), the schedule of the batch shape (instances, total knots,
 * longest and shortest horizon), which later solves of that shape use while pcg_cluster_size is 0:
 *   1. the PCG kernel: cluster sizes from the smallest that holds the longest horizon in <= 128 knots per
 *      CTA (64 with the stair preconditioner) to four times it, up to 16 and the shortest horizon, and,
 *      with pcg_precond 1, GPT_PCG_WARP_PAIR and GPT_PCG_WARP_QUAD;
 *   2. then, one kernel at a time, the grid of the per-knot kernels -- KKT formation, FP64 Schur complement,
 *      line-search merit, dz recovery -- as CTAs per SM in {4, 5, 6, 8, 16} (16 is the default; a change
 *      must gain 1 %);
 *   3. then, when the handle's sqp_graph is 1 (a graph solve whose branch count is left to the library),
 *      the part-batch branches per graph iteration in {1, 2, 4} (at most the batch; a change must gain
 *      1 %), which later graph solves of the shape use while sqp_graph stays 1.
 * h_cluster_out (optional) receives the PCG choice, h_schedule_out (optional, 5 entries) the CTAs per SM of
 * the KKT, Schur, merit and dz launches and the branches per graph iteration (the tuned count with
 * sqp_graph 1, else sqp_graph itself). */
gpt_status gpt_autotune(gpt_handle *h, uint32_t batch, const uint32_t *h_knot_points, const float *d_eePos_traj,
                        const float *d_lambda, const float *d_xu, const float *h_rho, uint32_t *h_cluster_out,
                        uint32_t *h_schedule_out, gpt_stream_t stream);

/* Adjoint of the SQP step (no reference counterpart).  At the iterate d_xu
 * (typically a solve's result) with per-instance rho h_rho and initial states
 * d_xs (14 per instance, x_0 of the solve's initial guess), the step solves
 * K [dz; lambda] = [g; c] (the KKT system of gato_form_kkt,
 * oldschur.cuh:966-1092) and maps xu to xu+ = xu - dz (the first line-search
 * step, toplevel.cuh:409), written to d_xu_next when non-NULL.  Given
 * d_grad_xu_next = dl/dxu+ (xu layout), one extra Schur right-hand side and
 * PCG solve with the same Schur matrix (K is symmetric) give the gradients of
 * l with respect to
 *   d_grad_eePos  the goal trajectory (6 per knot: xyz; rpy entries are 0),
 *   d_grad_qd     the 7 joint-velocity weights (QD_COST per joint), per instance,
 *   d_grad_r      the 7 control weights (R_COST per joint), per instance,
 *   d_grad_q_ee   the end-effector position weight, per instance.
 * Exact derivatives of that map (the SQP's own KKT matrix, with the
 * reference's terminal target when ref_terminal is set); at a converged
 * iterate xu+ = xu, so they are the one-step implicit derivatives of the
 * solution.  Per-knot dynamics and kinematics are recomputed, not stored.
 * Uses the handle's solver settings for both PCG solves. */
gpt_status gpt_sqp_adjoint(gpt_handle *h, uint32_t batch, const uint32_t *h_knot_points, const float *d_eePos_traj,
                           const float *d_xs, const float *d_xu, const float *h_rho, const float *d_grad_xu_next,
                           float *d_xu_next, float *d_grad_eePos, float *d_grad_qd, float *d_grad_r,
                           float *d_grad_q_ee, gpt_stream_t stream);

/* ---- the MPC tracking loop around the solve ---- */

/* Controls of the tracking loop: settings.cuh:26-29,59 and the -DSIMULATION_PERIOD flag of
 * perform_experiment.sh:46, toplevel.cuh:514-592, integrator.cuh:365-398.  The reference's
 * CONST_UPDATE_FREQ 1 mode: every control update simulates a fixed plant time. */
typedef struct gpt_track_config {
    float sim_period_us;          /* SIMULATION_PERIOD: plant time per control update (2000 in the logged runs) */
    float sim_step;               /* plant explicit-Euler step, 2e-4 s (integrator.cuh:378) */
    float shift_threshold;        /* SHIFT_THRESHOLD in seconds (settings.cuh:29: 1 * timestep); 0 = timestep */
    uint32_t max_control_updates; /* 100000 (toplevel.cuh:515) */
    uint32_t jitter_solves;       /* REMOVE_JITTERS (settings.cuh:59): solves from the trajectory at PCG
                                     tolerance 1e-11 / 10000 iterations before tracking, which warm lambda
                                     (toplevel.cuh:581-592; the reference runs 100); 0 = none */
    float rho_reset;              /* 1e-3 (toplevel.cuh:579) */
} gpt_track_config;

/* One instance's tracking run (the reference returns per-update vectors and the final error,
 * toplevel.cuh:810-815) */
typedef struct gpt_track_stats {
    uint32_t control_updates;     /* control updates this instance ran */
    uint32_t shifts;              /* trajectory offset reached (traj_steps when the run completed) */
    uint32_t sqp_iters_total;
    uint32_t pcg_iters_total;
    uint32_t ls_fail_total;
    uint32_t pcg_maxiter_total;
    uint32_t rho_exits;           /* solves that ended with rho > rho_max */
    uint32_t nonfinite;           /* solves that met a NaN/Inf */
    float tracking_error_mean;    /* mean of the per-shift errors */
    float final_tracking_error;   /* after the loop (toplevel.cuh:789-794) */
    float rho_final;
} gpt_track_stats;

void gpt_default_track_config(gpt_track_config *out);

/*
 * Receding-horizon tracking of a precomputed trajectory: replaces
 *   track<T, R>(state_size, control_size, knot_points, traj_steps, timestep, d_eePos_traj, d_xu_traj,
 *               d_xs, start_state_ind, goal_state_ind, test_iter, pcg_exit_tol, test_output_prefix)
 *                                                                      (toplevel.cuh:507-510)
 * Each control update solves the SQP (the handle's solver settings; sqp_max_iter stands in for the
 * reference's wall-clock cap SQP_MAX_TIME_US), simulates the plant (explicit Euler at sim_step) for
 * sim_period_us with the previous solution's controls, and once per timestep records the tracking
 * error sum_{i<3} |p(x_s)_i - goal_0,i| and shifts xu, the goal window and lambda one knot along
 * the trajectory (toplevel.cuh:600-726).  The run ends when the offset reaches traj_steps.
 *   d_eePos_traj  [6 traj_steps]   goal rows (runme.cu:145-150)
 *   d_xu_traj     [21 traj_steps]  x_k, u_k rows (runme.cu:152-157); traj_steps >= knot_points
 *   d_xs          [14]             plant state, in/out (the reference's d_xs)
 *   d_tracking_errors [traj_steps] one error per shift
 *   d_sqp_iters_log (optional)     SQP iterations of each update, first log_capacity updates
 *                                  (the returned sqp_iters vector of the reference)
 * The loop's working xu, lambda and goal window live in the handle (no allocation). */
gpt_status gpt_track(gpt_handle *h, uint32_t knot_points, uint32_t traj_steps, const float *d_eePos_traj,
                     const float *d_xu_traj, float *d_xs, const gpt_track_config *tc, float *d_tracking_errors,
                     uint32_t *d_sqp_iters_log, uint32_t log_capacity, gpt_track_stats *h_stats,
                     gpt_stream_t stream);

/* Many tracking runs at once (no reference counterpart): instance b has horizon h_knot_points[b]
 * and owns trajectory rows R_b .. R_b + h_traj_steps[b] - 1 of d_eePos_traj / d_xu_traj and of
 * d_tracking_errors (R_b = sum of the earlier traj_steps), 14 floats of d_xs, log_capacity
 * entries of d_sqp_iters_log and one h_stats entry.  Every update is one batched solve plus one
 * simulation / shift launch for the batch; all instances share the update clock and an instance
 * stops once the offset reaches its traj_steps. */
gpt_status gpt_track_batched(gpt_handle *h, uint32_t batch, const uint32_t *h_knot_points,
                             const uint32_t *h_traj_steps, const float *d_eePos_traj, const float *d_xu_traj,
                             float *d_xs, const gpt_track_config *tc, float *d_tracking_errors,
                             uint32_t *d_sqp_iters_log, uint32_t log_capacity, gpt_track_stats *h_stats,
                             gpt_stream_t stream);

/* gpt_track_batched with the adjoint of every control update's solve (no reference counterpart):
 * after an update's solve, the one-step adjoint of gpt_sqp_adjoint at the update's solution xu, on
 * that update's predicted tracking loss l = 1/2 sum_k |p(q_k+) - p*_k|^2 over the horizon at
 * xu+ = xu - dz (the solution's next SQP step) against the update's goal window, accumulated over
 * the updates each instance tracks:
 *   d_weight_grad [15 batch]  per instance dl/dqd (7), dl/dr (7), dl/dq_ee, summed over its updates
 *   d_loss        [batch]     sum of l over its updates (may be NULL)
 *   h_adjoint_fail [batch]    updates whose adjoint solve failed: factorisation, non-finite value or
 *                             PCG iteration cap (may be NULL)
 * Both device arrays are overwritten.  The forward run (tracking errors, logs, statistics, plant
 * state) equals gpt_track_batched's bit for bit.  Needs pcg_precond 0 or 1. */
gpt_status gpt_track_batched_adjoint(gpt_handle *h, uint32_t batch, const uint32_t *h_knot_points,
                                     const uint32_t *h_traj_steps, const float *d_eePos_traj,
                                     const float *d_xu_traj, float *d_xs, const gpt_track_config *tc,
                                     float *d_tracking_errors, uint32_t *d_sqp_iters_log, uint32_t log_capacity,
                                     float *d_weight_grad, float *d_loss, uint32_t *h_adjoint_fail,
                                     gpt_track_stats *h_stats, gpt_stream_t stream);

/* simple_simulate (integrator.cuh:365-398): advances the plant state d_xs (14) by sim_time_us of
 * explicit-Euler steps of sim_step seconds (plus the remainder step), applying the control of
 * knot floor(t / timestep) of d_xu (21N-7), t starting time_offset_us into the horizon. */
gpt_status gpt_simulate(gpt_handle *h, uint32_t knot_points, float *d_xs, const float *d_xu, double time_offset_us,
                        double sim_time_us, float sim_step, gpt_stream_t stream);

/* ---- rigid-body library kernels and trajectory files (no handle) ---- */

/* end_effector_positions_kernel (rbdfiles/iiwa_eepos_grid.cuh:2091-2110) for n rows at once (the
 * reference launches it once per row, generateeepos.cu:101-107): the end-effector xyz and roll,
 * pitch, yaw of joint vector d_x[i * row_stride + 0..6] -> d_eePos[6 i .. 6 i + 5].  row_stride 21
 * reads the rows of a trajectory (x, u), 14 plain states. */
gpt_status gpt_end_effector_positions(uint32_t n, const float *d_x, uint32_t row_stride, float *d_eePos,
                                      gpt_stream_t stream);

/* forward_dynamics (rbdfiles/iiwa_eepos_grid.cuh:4351-4395, gravity 0) for n rows at once:
 * qdd = M(q)^{-1} (u - c(q, qd)) of the row [q (7), qd (7), u (7)] at d_xu[i * row_stride]
 * -> d_qdd[7 i .. 7 i + 6]; row_stride >= 21. */
gpt_status gpt_forward_dynamics(uint32_t n, const float *d_xu, uint32_t row_stride, float *d_qdd,
                                gpt_stream_t stream);

/* forwardDynamicsAndGradient (rbdfiles/iiwa_eepos_plant.cuh:130-160) for n rows at once: qdd
 * (7 per row) and df/du = [-M^{-1} dID/dq, -M^{-1} dID/dqd, M^{-1}] (7 x 21 column-major, 147 per
 * row) of the row [q, qd, u] at d_xu[i * row_stride]; row_stride >= 21. */
gpt_status gpt_forward_dynamics_gradient(uint32_t n, const float *d_xu, uint32_t row_stride, float *d_qdd,
                                         float *d_dfdu, gpt_stream_t stream);

/* readCSVToVecVec (runme.cu:18-44, generateeepos.cu:14-40): a text file of comma-separated floats,
 * one row per line, parsed like std::stof, flattened row by row into h_out (host).  *h_rows and
 * *h_cols receive the shape; with h_out NULL only the shape is returned.  Rows of unequal length
 * (GPT_ERR_BAD_ARG) and a capacity (in floats) below rows x cols (GPT_ERR_CAPACITY, shape still
 * returned) are errors; an unreadable file is GPT_ERR_BAD_ARG. */
gpt_status gpt_read_csv(const char *path, float *h_out, size_t capacity, uint32_t *h_rows, uint32_t *h_cols);

/* ---- the reference's kernels, one instance, device buffers, stream-ordered ---- */

/* gato_form_kkt (schur.cuh:391-524); d_xs = x_s (14) */
gpt_status gpt_form_kkt(gpt_handle *h, uint32_t knot_points, const float *d_xu, const float *d_eePos_traj,
                        const float *d_xs, float *d_G, float *d_C, float *d_g, float *d_c, gpt_stream_t stream);

/* form_schur -> gato_form_schur_jacobi (schur.cuh:545-559, oldschur.cuh:518-963).
 * d_Ginv (245N-49) receives (Q+rho I)^-1 and (R+rho I)^-1, which the reference
 * writes over d_G (schur.cuh:236-256); d_Ginv64 (optional) the same in FP64. */
gpt_status gpt_form_schur(gpt_handle *h, uint32_t knot_points, float rho, const float *d_G, const float *d_C,
                          const float *d_g, const float *d_c, float *d_S, float *d_Pinv, float *d_gamma,
                          float *d_Ginv, double *d_Ginv64, gpt_stream_t stream);

/* form_schur_qdl (schur.cuh:528-542): upper-triangle CSC values (nnz = 196(N-1)+105N) */
gpt_status gpt_form_schur_csc(gpt_handle *h, uint32_t knot_points, float rho, const float *d_G, const float *d_C,
                              const float *d_g, const float *d_c, float *d_val, float *d_gamma, float *d_Ginv,
                              gpt_stream_t stream);

/* gato_form_ss_inner (oldschur.cuh:334-494): the stair ("SS") preconditioner.  Given S and the
 * block-Jacobi d_Pinv of gpt_form_schur (theta_k^{-1} in the diagonal blocks), fills Pinv's
 * off-diagonal blocks: left_k = -theta_k^{-1} S[k].left theta_{k-1}^{-1}, right_k =
 * -theta_k^{-1} S[k+1].left^T theta_{k+1}^{-1}.  The reference ships this kernel without calling
 * it; the SQP loop here uses the exact block-tridiagonal preconditioner instead. */
gpt_status gpt_form_ss(gpt_handle *h, uint32_t knot_points, const float *d_S, float *d_Pinv, gpt_stream_t stream);

/* prep_csr (utils.cuh:84-118): CSC column pointers [14N+1] and row indices [nnz] (host arrays) */
gpt_status gpt_prep_csr(uint32_t knot_points, int32_t *h_col_ptr, int32_t *h_row_ind);

/* GPU-PCG pcg<T,STATE_SIZE,KNOT_POINTS> launch (toplevel.cuh:135-157,292-294):
 * solves S lambda = gamma from the warm start in d_lambda (updated in place,
 * FP32).  d_lambda64 (optional, 14N doubles) receives the FP64 iterate; at
 * N >= ~64 only it can carry a relative residual near 1e-5.  With
 * pcg_cluster_size GPT_PCG_WARP_PAIR, S and gamma are first converted (exactly)
 * to FP64 packed rows in the handle's workspace. */
gpt_status gpt_pcg(gpt_handle *h, uint32_t knot_points, const float *d_S, const float *d_Pinv,
                   const float *d_gamma, float *d_lambda, double *d_lambda64, uint32_t max_iter, float exit_tol,
                   uint32_t exit_mode, uint32_t *h_iters, uint8_t *h_maxiter_exit, gpt_stream_t stream);

/* compute_dz (schur.cuh:562-566, oldschur.cuh:966-1105) from Ginv; the FP64
 * inputs d_Ginv64 / d_lambda64 (optional) are used instead of the FP32 ones
 * when given */
gpt_status gpt_compute_dz(gpt_handle *h, uint32_t knot_points, const float *d_Ginv, const double *d_Ginv64,
                          const float *d_C, const float *d_g, const float *d_lambda, const double *d_lambda64,
                          float *d_dz, gpt_stream_t stream);

/* compute_merit (merit.cuh:99-145): merit of d_xu -> *d_merit (one float) */
gpt_status gpt_compute_merit(gpt_handle *h, uint32_t knot_points, const float *d_xu, const float *d_eePos_traj,
                             float *d_merit, gpt_stream_t stream);

/* ls_gato_compute_merit x 8 (merit.cuh:16-94, toplevel.cuh:357-374): merits of
 * d_xu + alpha_p d_dz, alpha_p = -2^-p, p = 0..7 -> d_merits[8] */
gpt_status gpt_ls_compute_merit(gpt_handle *h, uint32_t knot_points, const float *d_xs, const float *d_xu,
                                const float *d_eePos_traj, const float *d_dz, float *d_merits,
                                gpt_stream_t stream);

/* The same 8 line-search merits without a handle and without allocating.  No
 * counterpart in the reference.  For callers that cannot allocate device
 * memory: a real-time control loop that allocates only at start-up, or a
 * plug-in whose host framework owns every device allocation (gpt_create
 * allocates the handle's workspace).  The scratch is a fixed array of
 * 8 x GPT_NOALLOC_MAX_KNOTS floats (16 KiB) inside the library, held on every
 * GPU that loads it until the process exits; knot_points above
 * GPT_NOALLOC_MAX_KNOTS returns GPT_ERR_BAD_ARG.  The first call on each device
 * looks up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  That address is
 * cached for the life of the process: after cudaDeviceReset on a device, this
 * entry point must not be called on that device again.  All calls share
 * the array: calls whose kernels overlap on the GPU (other streams, other host
 * threads) race.  pc->max_knot_points and max_batch are not used. */
#define GPT_NOALLOC_MAX_KNOTS 512
gpt_status gpt_ls_compute_merit_noalloc(const gpt_problem_config *pc, uint32_t knot_points, const float *d_xs,
                                        const float *d_xu, const float *d_eePos_traj, const float *d_dz,
                                        float *d_merits, gpt_stream_t stream);

/* ---- instrumentation (no reference counterpart; the reference times with
 * clock_gettime around host syncs, toplevel.cuh:36-38,219-222,286-303) ---- */

/* SQP-loop phases timed with CUDA events on the launch stream */
#define GPT_PHASE_INIT 0   /* x_s copy + merit of the initial iterate */
#define GPT_PHASE_KKT 1    /* KKT formation */
#define GPT_PHASE_SCHUR 2  /* Schur complement + preconditioner */
#define GPT_PHASE_PCG 3    /* PCG solve */
#define GPT_PHASE_DZ 4     /* dz recovery */
#define GPT_PHASE_MERIT 5  /* 8-step line-search merits */
#define GPT_PHASE_ACCEPT 6 /* merit reduction, rho schedule, step update */
#define GPT_NUM_PHASES 7

/* When enabled, every SQP-loop launch is bracketed by CUDA events. */
gpt_status gpt_set_profiling(gpt_handle *h, int enable);
/* Accumulated device milliseconds and launch counts per phase (arrays of
 * GPT_NUM_PHASES); reset != 0 clears them. */
gpt_status gpt_get_phase_stats(gpt_handle *h, double *h_ms, uint64_t *h_launches, int reset);

#ifdef __cplusplus
}
#endif

#endif /* GPT_H */
