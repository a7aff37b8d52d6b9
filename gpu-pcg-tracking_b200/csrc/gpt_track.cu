// gpt_track.cu -- the MPC tracking loop around the SQP solve, on the device.
//
//   track_start_kernel  track's set-up (toplevel.cuh:545-552, 578): xu, xu_old and the goal window
//                       from the trajectory, lambda = 0, rho = rho_0
//   track_prep_kernel   per-update start of a solve: the rho schedule carries over (T& rho,
//                       toplevel.cuh:617), drho = 1 (toplevel.cuh:89), finished instances inactive
//   track_clock_kernel  the loop's time bookkeeping (toplevel.cuh:628-724), shared by the batch
//   track_sim_kernel    simple_simulate (integrator.cuh:365-398): explicit-Euler plant steps of
//                       simple_integrator_kernel (integrator.cuh:306-331), 4 instances per warp
//   track_post_kernel   xu_old <- xu, tracking error, just_shift of xu / goal / lambda with the
//                       trajectory fills, x_0 <- x_s (toplevel.cuh:660-726), one block per instance
//   track_final_kernel  the final tracking error (toplevel.cuh:789-794)
//
// Instance b of a batch owns trajectory rows [rows[b], rows[b+1]) of eePos_traj (6 floats per row)
// and xu_traj (21 floats per row: x_k then u_k, runme.cu:145-161).
#include "gpt_common.cuh"
#include "gpt_dyn.cuh"
#include "gpt_internal.h"

namespace gpt {

// Control slot of plant time t: floor(t / timestep) (integrator.cuh:380-388), clamped to the
// horizon's last control (the reference reads past the horizon there).
__device__ __forceinline__ int track_slot(double t, double timestep, int N)
{
    const unsigned co = (unsigned)(t / timestep);
    return (int)co > N - 2 ? N - 2 : (int)co;
}

__global__ void track_start_kernel(BatchView bv, const int *__restrict__ rows, const float *__restrict__ eePos_traj,
                                   const float *__restrict__ xu_traj, float *__restrict__ xu, float *__restrict__ xu_old,
                                   float *__restrict__ goal, float *__restrict__ lambda, TrackClock *clk,
                                   TrackInst *inst, float rho0, int reset_xu_only)
{
    if (blockIdx.x == 0 && threadIdx.x == 0 && !reset_xu_only) *clk = TrackClock{};
    for (int b = blockIdx.x; b < bv.B; b += gridDim.x) {
        const int N = bv.N(b), kb = bv.off(b), r0 = rows[b];
        const float *tr = xu_traj + (size_t)NX * r0;
        for (int i = threadIdx.x; i < NX * N - NC; i += blockDim.x) {
            const float v = tr[i];
            xu[(size_t)NX * kb + i] = v;
            if (!reset_xu_only) xu_old[(size_t)NX * kb + i] = v;
        }
        if (reset_xu_only) {
            if (threadIdx.x == 0) bv.st[b].rho = rho0;
            continue;
        }
        for (int i = threadIdx.x; i < 6 * N; i += blockDim.x) goal[(size_t)6 * kb + i] = eePos_traj[(size_t)6 * r0 + i];
        for (int i = threadIdx.x; i < NS * N; i += blockDim.x) lambda[(size_t)NS * kb + i] = 0.f;
        if (threadIdx.x == 0) {
            bv.st[b].rho = rho0;
            inst[b] = TrackInst{};
        }
    }
}

// all_live: every instance solves (the warm-up solves before tracking); otherwise instance b
// solves while the shared trajectory offset is below its trajectory length.
__global__ void track_prep_kernel(BatchView bv, const int *__restrict__ rows, const TrackClock *__restrict__ clk,
                                  float rho_reset, int all_live)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bv.B) return;
    InstState &s = bv.st[b];
    const float rho = s.rho;
    const uint32_t live = all_live ? 1u : (clk->traj_offset < (uint32_t)(rows[b + 1] - rows[b]) ? 1u : 0u);
    s = InstState{};
    s.rho = rho;
    s.drho = 1.f;
    s.rho_reset = rho_reset;
    s.active = live;
}

// One update's time bookkeeping (toplevel.cuh:628-724, CONST_UPDATE_FREQ 1): the plant runs
// sim_period_us from the previous update's offset; the goal window shifts once the time since the
// last timestep passes the threshold, and the timer wraps once it passes the timestep.
__global__ void track_clock_kernel(TrackClock *clk, TrackParams tp)
{
    TrackClock c = *clk;
    c.sim_offset_us = c.prev_sim_us;
    c.start_offset = c.traj_offset;
    c.time_since += tp.sim_us * 1e-6;
    c.do_shift = 0u;
    if (!c.shifted && c.time_since > tp.shift_threshold) {
        c.do_shift = 1u;
        c.traj_offset++;
        c.shifted = 1u;
    }
    if (c.time_since > tp.timestep) {
        c.shifted = 0u;
        c.time_since = fmod(c.time_since, tp.timestep);
    }
    c.prev_sim_us = tp.sim_us;
    c.updates++;
    *clk = c;
}

// One explicit-Euler plant step x <- x + h [qd; M^{-1}(u - c(q, qd))] by a group of 8 lanes
// (fd_group).  Every lane holds the whole state (q, qd) and the control u.
__device__ __forceinline__ void plant_step_group(float (&q)[NQ], float (&qd)[NQ], const float (&u)[NC], float h,
                                                 int m, int base)
{
    double col[NQ];
    fd_group(q, qd, u, col, m, base);
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const float qdd = (float)__shfl_sync(0xffffffffu, col[i], base + 7);
        q[i] = q[i] + h * qd[i];
        qd[i] = qd[i] + h * qdd;
    }
}

__global__ void __launch_bounds__(128)
    track_sim_kernel(BatchView bv, const int *__restrict__ rows, const TrackClock *__restrict__ clk, TrackParams tp,
                     float *__restrict__ xs, const float *__restrict__ xu_old)
{
    const int lane = threadIdx.x & 31, m = lane & 7, base = lane & ~7;
    const int b_raw = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    // lanes of a group past the batch or of a finished instance follow instance 0's data (all
    // lanes take part in the shuffles) and store nothing
    bool live = b_raw < bv.B;
    const int b = live ? b_raw : 0;
    const uint32_t start_offset = clk->start_offset;
    live = live && start_offset < (uint32_t)(rows[b + 1] - rows[b]);
    const int N = bv.N(b), kb = bv.off(b);
    float q[NQ], qd[NQ], u[NC];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        q[i] = xs[(size_t)NS * b + i];
        qd[i] = xs[(size_t)NS * b + NQ + i];
    }
    const double t0 = clk->sim_offset_us * 1e-6;
    const float *xo = xu_old + (size_t)NX * kb;
    int co = track_slot(t0, tp.timestep, N);
    for (uint32_t step = 0; step < tp.n_sub; ++step) {
        co = track_slot(t0 + (double)((float)step * tp.sim_step), tp.timestep, N);
#pragma unroll
        for (int i = 0; i < NC; ++i) u[i] = xo[NX * co + NS + i];
        plant_step_group(q, qd, u, tp.sim_step, m, base);
    }
#pragma unroll
    for (int i = 0; i < NC; ++i) u[i] = xo[NX * co + NS + i];
    plant_step_group(q, qd, u, tp.sim_last, m, base);
    if (live && m < NQ) {
        float qm = 0.f, qdm = 0.f;
#pragma unroll
        for (int i = 0; i < NQ; ++i)
            if (i == m) { qm = q[i]; qdm = qd[i]; }
        xs[(size_t)NS * b + m] = qm;
        xs[(size_t)NS * b + NQ + m] = qdm;
    }
}

// sum_{i<3} |p(q)_i - goal_i| (toplevel.cuh:674-681)
__device__ __forceinline__ float track_error(const float *x, const float *goal)
{
    JointTrig t;
    joint_trig(x, t);
    float p[3];
    fk_lane<false>(t, p, nullptr);
    return fabsf(p[0] - goal[0]) + fabsf(p[1] - goal[1]) + fabsf(p[2] - goal[2]);
}

constexpr int POST_THREADS = 256;

__global__ void __launch_bounds__(POST_THREADS)
    track_post_kernel(BatchView bv, const int *__restrict__ rows, const TrackClock *__restrict__ clk,
                      const float *__restrict__ eePos_traj, const float *__restrict__ xu_traj,
                      const float *__restrict__ xs, float *__restrict__ xu, float *__restrict__ xu_old,
                      float *__restrict__ goal, float *__restrict__ lambda, float *__restrict__ tmp,
                      float *__restrict__ errors, TrackInst *__restrict__ inst, uint32_t *__restrict__ iters_log,
                      uint32_t log_cap)
{
    const int b = blockIdx.x;
    if (b >= bv.B) return;
    const int S = rows[b + 1] - rows[b];
    const uint32_t start_offset = clk->start_offset;
    if (start_offset >= (uint32_t)S) return;  // finished before this update (block-uniform)
    const int N = bv.N(b), kb = bv.off(b), len = NX * N - NC;
    const bool shift = clk->do_shift != 0u;
    const int T = (int)clk->traj_offset;  // after the increment of this update's shift
    float *x = xu + (size_t)NX * kb, *xo = xu_old + (size_t)NX * kb;
    float *gl = goal + (size_t)6 * kb, *lm = lambda + (size_t)NS * kb, *sc = tmp + (size_t)NX * kb;
    for (int i = threadIdx.x; i < len; i += POST_THREADS) xo[i] = x[i];
    if (shift) {
        for (int i = threadIdx.x; i < 6 * N; i += POST_THREADS) sc[i] = gl[i];
        for (int i = threadIdx.x; i < NS * N; i += POST_THREADS) sc[6 * N + i] = lm[i];
        if (threadIdx.x == 0) {
            const float e = track_error(xs + (size_t)NS * b, gl);
            errors[rows[b] + (int)start_offset] = e;
            inst[b].err_sum += e;
        }
    }
    __syncthreads();
    if (shift) {
        const float *tr = xu_traj + (size_t)NX * rows[b];
        const bool inside = T + N < S;
        // just_shift (integrator.cuh:299-304): knot k <- knot k+1 up to x_{N-1} -> x_{N-2}
        // (indices below len - NX); then u_{N-2} (len - NX .. len - NS) from the trajectory
        for (int i = threadIdx.x; i < len - NS; i += POST_THREADS) {
            float v;
            if (i < len - NX) {
                v = xo[i + NX];
            } else if (inside) {
                v = tr[NX * T - NC + (i - (len - NX))];  // u_{N-2}: row T-1's control
            } else {
                v = 0.f;
            }
            x[i] = v;
        }
        // x_{N-1}: trajectory row T inside the trajectory, else its last q with zero velocity
        for (int i = threadIdx.x; i < NS; i += POST_THREADS) {
            float v;
            if (inside) v = tr[NX * T + i];
            else v = (i < NQ) ? tr[NX * (S - 1) + i] : 0.f;
            x[len - NS + i] = v;
        }
        const int row = inside ? T + N - 1 : S - 1;
        for (int i = threadIdx.x; i < 6 * N; i += POST_THREADS)
            gl[i] = (i < 6 * (N - 1)) ? sc[i + 6] : eePos_traj[(size_t)6 * (rows[b] + row) + (i - 6 * (N - 1))];
        for (int i = threadIdx.x; i < NS * (N - 1); i += POST_THREADS) lm[i] = sc[6 * N + NS + i];
    }
    __syncthreads();
    if (threadIdx.x < NS) x[threadIdx.x] = xs[(size_t)NS * b + threadIdx.x];
    if (threadIdx.x == 0) {
        const InstState &s = bv.st[b];
        TrackInst &ti = inst[b];
        if (iters_log && ti.updates < log_cap) iters_log[(size_t)log_cap * b + ti.updates] = s.sqp_iters;
        ti.updates++;
        ti.sqp_iters += s.sqp_iters;
        ti.pcg_iters += s.pcg_iters_total;
        ti.ls_fail += s.ls_fail_count;
        ti.pcg_maxiter += s.pcg_maxiter_count;
        ti.rho_exits += (s.exit_flags & 1u) ? 1u : 0u;
        ti.nonfinite += (s.exit_flags & 4u) ? 1u : 0u;
        ti.shifts = shift ? (uint32_t)T : ti.shifts;
    }
}

__global__ void track_final_kernel(BatchView bv, const float *__restrict__ xs, const float *__restrict__ goal,
                                   TrackInst *__restrict__ inst)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bv.B) return;
    inst[b].final_err = track_error(xs + (size_t)NS * b, goal + (size_t)6 * bv.off(b));
    inst[b].rho = bv.st[b].rho;
}

cudaError_t launch_track_start(const BatchView &bv, const int *rows, const float *eePos_traj, const float *xu_traj,
                               float *xu, float *xu_old, float *goal, float *lambda, TrackClock *clk, TrackInst *inst,
                               float rho0, int reset_xu_only, int num_sms, cudaStream_t s)
{
    int blocks = bv.B < num_sms * 8 ? bv.B : num_sms * 8;
    track_start_kernel<<<blocks, 256, 0, s>>>(bv, rows, eePos_traj, xu_traj, xu, xu_old, goal, lambda, clk, inst,
                                              rho0, reset_xu_only);
    return cudaGetLastError();
}

cudaError_t launch_track_prep(const BatchView &bv, const int *rows, const TrackClock *clk, float rho_reset,
                              int all_live, cudaStream_t s)
{
    track_prep_kernel<<<(bv.B + 127) / 128, 128, 0, s>>>(bv, rows, clk, rho_reset, all_live);
    return cudaGetLastError();
}

cudaError_t launch_track_tail(const BatchView &bv, const int *rows, TrackClock *clk, const TrackParams &tp,
                              const float *eePos_traj, const float *xu_traj, float *xs, float *xu, float *xu_old,
                              float *goal, float *lambda, float *tmp, float *errors, TrackInst *inst,
                              uint32_t *iters_log, uint32_t log_cap, cudaStream_t s)
{
    track_clock_kernel<<<1, 1, 0, s>>>(clk, tp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // one warp (4 instances) per CTA: the kernel is a dependent chain per instance, so the
    // instances spread over as many SMs as possible
    track_sim_kernel<<<(bv.B + 3) / 4, 32, 0, s>>>(bv, rows, clk, tp, xs, xu_old);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    track_post_kernel<<<bv.B, POST_THREADS, 0, s>>>(bv, rows, clk, eePos_traj, xu_traj, xs, xu, xu_old, goal, lambda,
                                                    tmp, errors, inst, iters_log, log_cap);
    return cudaGetLastError();
}

cudaError_t launch_track_final(const BatchView &bv, const float *xs, const float *goal, TrackInst *inst, cudaStream_t s)
{
    track_final_kernel<<<(bv.B + 63) / 64, 64, 0, s>>>(bv, xs, goal, inst);
    return cudaGetLastError();
}

// ---- the adjoint of each update's solve (gpt_track_batched_adjoint; no reference counterpart)

// Saves every instance's per-solve state (the adjoint's KKT, Schur and PCG launches reuse the
// solve's kernels, which count into it) and marks the instances that track this update active.
__global__ void track_adj_begin_kernel(BatchView bv, const int *__restrict__ rows, const TrackClock *__restrict__ clk,
                                       InstState *__restrict__ bak)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bv.B) return;
    InstState &s = bv.st[b];
    bak[b] = s;
    s.active = clk->traj_offset < (uint32_t)(rows[b + 1] - rows[b]) ? 1u : 0u;
    s.exit_flags = 0u;
    s.pcg_maxiter_count = 0u;
}

// One thread per knot of an active instance: q+ = q - dz_q, p = p(q+), e = p - p*_k;
// kloss_k = |e|^2 / 2 and h_q = -J(q+)^T e (the adjoint right-hand side dl/d(dz) = -dl/dxu+).
__global__ void track_loss_grad_kernel(BatchView bv, const float *__restrict__ xu, const float *__restrict__ dz,
                                       const float *__restrict__ goal, float *__restrict__ h,
                                       float *__restrict__ kloss)
{
    for (int j = bv.j0 + blockIdx.x * blockDim.x + threadIdx.x; j < bv.j0 + bv.total_knots;
         j += gridDim.x * blockDim.x) {
        if (!bv.active(bv.inst(j))) continue;
        float q[NQ];
#pragma unroll
        for (int i = 0; i < NQ; ++i) q[i] = xu[(size_t)NX * j + i] - dz[(size_t)NX * j + i];
        JointTrig t;
        joint_trig(q, t);
        float p[3], J[3 * NQ];
        fk_lane<true>(t, p, J);
        const float e0 = p[0] - goal[(size_t)6 * j], e1 = p[1] - goal[(size_t)6 * j + 1],
                    e2 = p[2] - goal[(size_t)6 * j + 2];
        kloss[j] = 0.5f * (e0 * e0 + e1 * e1 + e2 * e2);
#pragma unroll
        for (int i = 0; i < NQ; ++i) h[(size_t)NX * j + i] = -(J[3 * i] * e0 + J[3 * i + 1] * e1 + J[3 * i + 2] * e2);
    }
}

// Per instance: loss[b] += the update's loss (a fixed-order FP64 sum of the knots' terms) and one
// more failed update when an adjoint solve stopped (factorisation, non-finite value, PCG cap); then
// the saved per-solve state comes back.
__global__ void track_adj_end_kernel(BatchView bv, const InstState *__restrict__ bak, const float *__restrict__ kloss,
                                     float *__restrict__ loss, TrackInst *__restrict__ inst)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bv.B) return;
    InstState &s = bv.st[b];
    if (s.active) {
        const int kb = bv.off(b), N = bv.N(b);
        double a = 0.0;
        for (int k = 0; k < N; ++k) a += (double)kloss[kb + k];
        if (loss) loss[b] += (float)a;
        if ((s.exit_flags & (GPT_EXIT_NONFINITE | GPT_EXIT_FACTOR)) || s.pcg_maxiter_count) inst[b].adj_fail++;
    }
    s = bak[b];
}

cudaError_t launch_track_adj_begin(const BatchView &bv, const int *rows, const TrackClock *clk, InstState *bak,
                                   cudaStream_t s)
{
    track_adj_begin_kernel<<<(bv.B + 127) / 128, 128, 0, s>>>(bv, rows, clk, bak);
    return cudaGetLastError();
}

cudaError_t launch_track_loss_grad(const BatchView &bv, const float *xu, const float *dz, const float *goal, float *h,
                                   float *kloss, int num_sms, cudaStream_t s)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    int blocks = (bv.total_knots + 127) / 128;
    if (blocks > num_sms * 8) blocks = num_sms * 8;
    track_loss_grad_kernel<<<blocks, 128, 0, s>>>(bv, xu, dz, goal, h, kloss);
    return cudaGetLastError();
}

cudaError_t launch_track_adj_end(const BatchView &bv, const InstState *bak, const float *kloss, float *loss,
                                 TrackInst *inst, cudaStream_t s)
{
    track_adj_end_kernel<<<(bv.B + 127) / 128, 128, 0, s>>>(bv, bak, kloss, loss, inst);
    return cudaGetLastError();
}

// simple_simulate of one state over one horizon (the gpt_simulate entry point): the clock
// holds the time offset; one group of 8 lanes.
__global__ void simulate_one_kernel(int N, TrackParams tp, double t0_us, float *__restrict__ xs,
                                    const float *__restrict__ xu)
{
    const int lane = threadIdx.x & 31, m = lane & 7, base = lane & ~7;
    float q[NQ], qd[NQ], u[NC];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        q[i] = xs[i];
        qd[i] = xs[NQ + i];
    }
    const double t0 = t0_us * 1e-6;
    int co = track_slot(t0, tp.timestep, N);
    for (uint32_t step = 0; step < tp.n_sub; ++step) {
        co = track_slot(t0 + (double)((float)step * tp.sim_step), tp.timestep, N);
#pragma unroll
        for (int i = 0; i < NC; ++i) u[i] = xu[NX * co + NS + i];
        plant_step_group(q, qd, u, tp.sim_step, m, base);
    }
#pragma unroll
    for (int i = 0; i < NC; ++i) u[i] = xu[NX * co + NS + i];
    plant_step_group(q, qd, u, tp.sim_last, m, base);
    __syncwarp();
    if (lane < NQ) {
        float qm = 0.f, qdm = 0.f;
#pragma unroll
        for (int i = 0; i < NQ; ++i)
            if (i == lane) { qm = q[i]; qdm = qd[i]; }
        xs[lane] = qm;
        xs[NQ + lane] = qdm;
    }
}

cudaError_t launch_simulate_one(int N, const TrackParams &tp, double t0_us, float *xs, const float *xu,
                                cudaStream_t s)
{
    simulate_one_kernel<<<1, 32, 0, s>>>(N, tp, t0_us, xs, xu);
    return cudaGetLastError();
}

}  // namespace gpt
