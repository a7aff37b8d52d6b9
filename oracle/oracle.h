/*
 * oracle/oracle.h -- TEST INFRASTRUCTURE, not the product.
 *
 * CPU restatement of the reference's SQP inner loop for 7-DOF iiwa
 * end-effector tracking (gpu-pcg-tracking: toplevel.cuh sqpSolve and the
 * kernels it launches).  It exists only to check the CUDA product: tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may call it, nothing
 * else.  Every function cites the reference file:line it follows.
 *
 * The file oracle.c is compiled twice: with GPT_REAL=float (symbols orc_f32_*)
 * and GPT_REAL=double (symbols orc_f64_*).
 *
 * Layouts (s = 14 state, c = 7 control, N knots; all matrices column-major):
 *   xu    [21N-7]    x_0 u_0 x_1 u_1 ... x_{N-1}              (toplevel.cuh:512)
 *   goal  [6N]       end-effector xyz+rpy per knot            (runme.cu:153-157)
 *   G     [245N-49]  {Q_k 14x14, R_k 7x7} per knot, last knot Q only
 *   C     [294(N-1)] {-A_k 14x14, -B_k 14x7}
 *   g     [21N-7]    {q_k, r_k}
 *   c     [14N]      c_0 = x_0 - x_s, c_{k+1} = x_{k+1} - f(x_k,u_k)
 *   S     [588N]     block row k = [left, diag, right] 14x14 blocks (utils.cuh:121-150)
 *   Pinv  [588N]     same layout, block-Jacobi: only diag blocks non-zero
 */
#ifndef GPT_ORACLE_H
#define GPT_ORACLE_H

#include <stdint.h>

typedef struct {
    double dt;          /* timestep (runme.cu:65 uses 1/64) */
    int integrator;     /* 0 explicit Euler (reference default), 1 semi-implicit */
    double q_ee;        /* weight on 0.5*|p(q)-p*|^2 (implicitly 1 in the reference) */
    double qd_cost;     /* QD_COST (iiwa_eepos_plant.cuh:58-60) */
    double r_cost;      /* R_COST  (iiwa_eepos_plant.cuh:62-64) */
    double mu;          /* merit penalty, 10 (toplevel.cuh:54) */
    int ref_terminal;   /* 1: terminal Q,q evaluated at x_{N-2} with target Q_{N-2}[0][0..2], as
                           the reference's kernel computes (goal_{N-1} is overwritten in its shared
                           buffer: schur.cuh:413-425, iiwa_eepos_plant.cuh:396-401);
                           0: at x_{N-1} with target goal_{N-1} */
} orc_params;

typedef struct {
    int sqp_iters;          /* sqp_iter (toplevel.cuh:400,435) */
    int rho_exit;           /* 1 if the loop stopped because rho > rho_max */
    int ls_fail_count;
    int pcg_iters_total;
    int pcg_maxiter_count;
    int linsys_count;
    double merit_final;
    double rho_final;
} orc_stats;

typedef struct {
    int linsys;             /* 0 PCG (block-Jacobi), 1 LDL^T of the CSC Schur matrix (qdldl path),
                               2 FP64 banded Cholesky */
    int sqp_max_iter;       /* SQP_MAX_ITER (settings.cuh:31-37) */
    int pcg_max_iter;
    double pcg_tol;
    int pcg_exit_mode;      /* 0: ||r||_2 <= tol*||gamma||_2, 1: |r^T Pinv r| < tol */
    double rho_factor, rho_max, rho_min;   /* RHO_FACTOR, RHO_MAX, RHO_MIN (settings.cuh:50) */
} orc_solver;

/* MPC tracking loop controls (toplevel.cuh:507-596, settings.cuh:26-29, integrator.cuh:365-398) */
typedef struct {
    double sim_period_us;     /* SIMULATION_PERIOD: plant time simulated per control update (CONST_UPDATE_FREQ 1) */
    double sim_step;          /* plant integration step, 2e-4 s, held as float (integrator.cuh:378) */
    double shift_threshold;   /* SHIFT_THRESHOLD in s (settings.cuh:29: 1 * timestep) */
    int max_control_updates;  /* 100000 (toplevel.cuh:515) */
    int jitter_solves;        /* REMOVE_JITTERS: solves at tol 1e-11 before tracking (toplevel.cuh:581-592) */
    double rho_reset;         /* 1e-3 (toplevel.cuh:579) */
} orc_track_cfg;

typedef struct {
    int control_updates;      /* control_update_step at exit */
    int shifts;               /* traj_offset at exit */
    int sqp_iters_total;
    int pcg_iters_total;
    int ls_fail_total;
    int rho_exits;
    double final_error;       /* cur_tracking_error after the loop (toplevel.cuh:789-794) */
    double rho_final;
} orc_track_stats;

#endif
