// gpt_adjoint.cu -- gradients of a loss of the SQP step with respect to the
// cost weights and the end-effector goal (the adjoint of the KKT solve).
//
// No reference counterpart (the reference has no derivatives of its solve).
// At an iterate xu the SQP step solves K(theta) [dz; lambda] = [g(theta); c]
// (the KKT system of gato_form_kkt / oldschur.cuh:966-1092) and proposes
// xu+ = xu - dz (the first line-search step, alpha_0 = -1, toplevel.cuh:409).
// For a loss l(xu+) with h = dl/d(dz) = -dl/dxu+, the adjoint solve
// K mu = [h; 0] (K is symmetric, so the same Schur complement and PCG serve)
// gives dl/dtheta = mu_z^T (dg/dtheta - dG/dtheta dz).  theta enters only the
// cost blocks of knot k through
//   v_k = q_ee J_k^T (p(q_k) - p*_k)            position-cost gradient (7)
//   Q_k = [v_k v_k^T, 0; 0, diag(qd)],  q_k = [v_k; qd .* qdot_k]
//   R_k = diag(r),  r_k = r .* u_k
// so with a = mu_q, d = dz_q the position part reduces to the adjoint of v_k,
//   w_k = a (1 - v_k^T d) - d (a^T v_k),
// and dl/dp*_k = -q_ee J_k w_k, dl/dq_ee = sum_k w_k^T J_k^T (p_k - p*_k),
// dl/dqd_i = sum_k mu_{k,7+i} (qdot_{k,i} - dz_{k,7+i}),
// dl/dr_i = sum_{k<N-1} mu_{k,u,i} (u_{k,i} - dz_{k,u,i}).
// The terminal block follows the forward model: with ref_terminal it is
// evaluated at x_{N-2} with target t = (a0^2, a0 a1, a0 a2), a = v_{N-2}
// (the reference kernel's overwritten goal), whose derivative flows back into
// v_{N-2}; otherwise at x_{N-1} with target p*_{N-1}.  Per-knot forward-kinematic
// quantities are recomputed, not stored.
#include "gpt_common.cuh"
#include "gpt_dyn.cuh"
#include "gpt_internal.h"

namespace gpt {

constexpr int ADJ_WARPS = 4;
constexpr int ADJ_PART = 16;  // per-knot partials: qd 0..6, r 7..13, q_ee 14

struct AdjWarpSmem {
    float x[2][NS];      // x_k and x_{k+1}
    float u[NC];
    float goal[12];      // p*_k, p*_{k+1} (xyz + rpy)
    float mu[2][NS];     // mu_z state parts of knots k, k+1
    float muu[NC];
    float d[2][NS];      // dz state parts of knots k, k+1
    float du[NC];
    float p[2][3], J[2][21];
};

__device__ __forceinline__ void adj_v(const float *J, const float *p, const float *t, float qee, float *v)
{
#pragma unroll
    for (int i = 0; i < NQ; ++i)
        v[i] = qee * (J[3 * i] * (p[0] - t[0]) + J[3 * i + 1] * (p[1] - t[1]) + J[3 * i + 2] * (p[2] - t[2]));
}

// w = a (1 - v.d) - d (a.v): the adjoint of v in a^T v - a^T (v v^T) d
__device__ __forceinline__ void adj_w(const float *a, const float *d, const float *v, float *w)
{
    double vd = 0.0, av = 0.0;
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        vd += (double)v[i] * d[i];
        av += (double)a[i] * v[i];
    }
#pragma unroll
    for (int i = 0; i < NQ; ++i) w[i] = (float)((double)a[i] * (1.0 - vd) - (double)d[i] * av);
}

__global__ void __launch_bounds__(32 * ADJ_WARPS)
    adjoint_grad_kernel(BatchView bv, ProblemParams P, const float *__restrict__ xu, const float *__restrict__ goal,
                        const float *__restrict__ dz, const float *__restrict__ mu, float *__restrict__ grad_goal,
                        float *__restrict__ part)
{
    __shared__ AdjWarpSmem smem_all[ADJ_WARPS];
    const int lane = threadIdx.x & 31;
    AdjWarpSmem &sm = smem_all[threadIdx.x >> 5];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = bv.j0 + gw; j < bv.j0 + bv.total_knots; j += nw) {
        const int b = bv.inst(j);
        if (!bv.active(b)) continue;
        const int N = bv.N(b), k = j - bv.off(b);
        float *pk = part + (size_t)ADJ_PART * j;
        if (k == N - 1) continue;  // the terminal knot is handled with knot N-2
        const bool terminal = (k == N - 2);
        // ---- stage x_k, u_k, x_{k+1}, goals, mu and dz of knots k, k+1
        for (int i = lane; i < NX + NS; i += 32) {
            const size_t o = (size_t)NX * j + i;
            if (i < NS) {
                sm.x[0][i] = xu[o];
                sm.mu[0][i] = mu[o];
                sm.d[0][i] = dz[o];
            } else if (i < NX) {
                sm.u[i - NS] = xu[o];
                sm.muu[i - NS] = mu[o];
                sm.du[i - NS] = dz[o];
            } else {
                sm.x[1][i - NX] = xu[o];
                sm.mu[1][i - NX] = mu[o];
                sm.d[1][i - NX] = dz[o];
            }
        }
        if (lane < 12) sm.goal[lane] = goal[(size_t)6 * j + lane];
        __syncwarp();
        // ---- forward kinematics and position Jacobian: lane 0 at x_k, lane 1 at x_{k+1}
        if (lane == 0 || (lane == 1 && terminal && !P.ref_terminal)) {
            JointTrig t;
            joint_trig(sm.x[lane], t);
            fk_lane<true>(t, sm.p[lane], sm.J[lane]);
        }
        __syncwarp();
        if (lane == 0) {
            const float qee = P.q_ee;
            float v[NQ], w[NQ], e[3];
            for (int dd = 0; dd < 3; ++dd) e[dd] = sm.p[0][dd] - sm.goal[dd];
            adj_v(sm.J[0], sm.p[0], sm.goal, qee, v);
            adj_w(sm.mu[0], sm.d[0], v, w);
            double gq = 0.0;                                  // d l / d q_ee
            float gg_next[3] = {0.f, 0.f, 0.f};               // d l / d p*_{k+1} (terminal, spec mode)
            double qd_part[NQ], r_part[NC];
#pragma unroll
            for (int i = 0; i < NQ; ++i)
                qd_part[i] = (double)sm.mu[0][NQ + i] * ((double)sm.x[0][NQ + i] - (double)sm.d[0][NQ + i]);
#pragma unroll
            for (int i = 0; i < NC; ++i) r_part[i] = (double)sm.muu[i] * ((double)sm.u[i] - (double)sm.du[i]);
            if (terminal) {
                // terminal cost block (knot N-1)
                const int which = P.ref_terminal ? 0 : 1;
                const float *xt = P.ref_terminal ? sm.x[0] : sm.x[1];
                float tt[3];
                if (P.ref_terminal) {
                    const float a0 = v[0];
                    tt[0] = a0 * a0;
                    tt[1] = a0 * v[1];
                    tt[2] = a0 * v[2];
                } else {
                    tt[0] = sm.goal[6];
                    tt[1] = sm.goal[7];
                    tt[2] = sm.goal[8];
                }
                float vt[NQ], wt[NQ];
                adj_v(sm.J[which], sm.p[which], tt, qee, vt);
                adj_w(sm.mu[1], sm.d[1], vt, wt);
                // d l / d target = -q_ee J_t w_t
                float gt[3];
                for (int dd = 0; dd < 3; ++dd) {
                    double a = 0.0;
#pragma unroll
                    for (int i = 0; i < NQ; ++i) a += (double)sm.J[which][3 * i + dd] * wt[i];
                    gt[dd] = (float)(-(double)qee * a);
                }
                // direct q_ee dependence of v_t = q_ee J_t^T (p_t - t)
                for (int i = 0; i < NQ; ++i) {
                    double a = 0.0;
                    for (int dd = 0; dd < 3; ++dd)
                        a += (double)sm.J[which][3 * i + dd] * ((double)sm.p[which][dd] - (double)tt[dd]);
                    gq += (double)wt[i] * a;
                }
                if (P.ref_terminal) {
                    // t = (a0^2, a0 a1, a0 a2) with a = v_{N-2}: the target's adjoint flows into w_{N-2}
                    w[0] += 2.f * v[0] * gt[0] + v[1] * gt[1] + v[2] * gt[2];
                    w[1] += v[0] * gt[1];
                    w[2] += v[0] * gt[2];
                } else {
                    for (int dd = 0; dd < 3; ++dd) gg_next[dd] = gt[dd];
                }
                // terminal velocity cost qd .* qdot_t
#pragma unroll
                for (int i = 0; i < NQ; ++i)
                    qd_part[i] += (double)sm.mu[1][NQ + i] * ((double)xt[NQ + i] - (double)sm.d[1][NQ + i]);
            }
            // knot k: d l / d p*_k = -q_ee J_k w_k and the q_ee term w_k^T J_k^T e_k
            for (int dd = 0; dd < 3; ++dd) {
                double a = 0.0;
#pragma unroll
                for (int i = 0; i < NQ; ++i) a += (double)sm.J[0][3 * i + dd] * w[i];
                grad_goal[(size_t)6 * j + dd] = (float)(-(double)qee * a);
            }
            for (int i = 0; i < NQ; ++i) {
                double a = 0.0;
                for (int dd = 0; dd < 3; ++dd) a += (double)sm.J[0][3 * i + dd] * e[dd];
                gq += (double)w[i] * a;
            }
            for (int dd = 3; dd < 6; ++dd) grad_goal[(size_t)6 * j + dd] = 0.f;
            if (terminal) {
                for (int dd = 0; dd < 3; ++dd) grad_goal[(size_t)6 * (j + 1) + dd] = gg_next[dd];
                for (int dd = 3; dd < 6; ++dd) grad_goal[(size_t)6 * (j + 1) + dd] = 0.f;
            }
#pragma unroll
            for (int i = 0; i < NQ; ++i) pk[i] = (float)qd_part[i];
#pragma unroll
            for (int i = 0; i < NC; ++i) pk[NQ + i] = (float)r_part[i];
            pk[14] = (float)gq;
        }
        __syncwarp();
    }
}

// per instance: fixed-order FP64 sums of the per-knot partials (knots 0..N-2)
// (wacc: added to wacc[15 b + t] instead)
__global__ void adjoint_reduce_kernel(BatchView bv, const float *__restrict__ part, float *__restrict__ grad_qd,
                                      float *__restrict__ grad_r, float *__restrict__ grad_qee, float *__restrict__ wacc)
{
    const int b = bv.b0 + (int)blockIdx.x;
    if (b >= bv.b0 + bv.B || !bv.active(b)) return;
    const int t = threadIdx.x;  // 0..14
    if (t >= 15) return;
    const int N = bv.N(b), kb = bv.off(b);
    double a = 0.0;
    for (int k = 0; k < N - 1; ++k) a += (double)part[(size_t)ADJ_PART * (kb + k) + t];
    if (wacc) wacc[(size_t)15 * b + t] += (float)a;
    else if (t < NQ) grad_qd[(size_t)NQ * b + t] = (float)a;
    else if (t < NQ + NC) grad_r[(size_t)NC * b + t - NQ] = (float)a;
    else grad_qee[b] = (float)a;
}

// out = a + alpha * x (a == nullptr: out = alpha * x)
__global__ void axpy_kernel(int n, float alpha, const float *__restrict__ x, const float *__restrict__ a,
                            float *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = a ? fmaf(alpha, x[i], a[i]) : alpha * x[i];
}

cudaError_t launch_adjoint_grad(const BatchView &bv, const ProblemParams &P, const float *xu, const float *goal,
                                const float *dz, const float *mu, float *grad_goal, float *part, float *grad_qd,
                                float *grad_r, float *grad_qee, int num_sms, cudaStream_t s, float *wacc)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    int blocks = (bv.total_knots + ADJ_WARPS - 1) / ADJ_WARPS;
    if (blocks > num_sms * 16) blocks = num_sms * 16;
    adjoint_grad_kernel<<<blocks, 32 * ADJ_WARPS, 0, s>>>(bv, P, xu, goal, dz, mu, grad_goal, part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    adjoint_reduce_kernel<<<bv.B, 32, 0, s>>>(bv, part, grad_qd, grad_r, grad_qee, wacc);
    return cudaGetLastError();
}

cudaError_t launch_axpy(int n, float alpha, const float *x, const float *a, float *out, int num_sms, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    int blocks = (n + 255) / 256;
    if (blocks > num_sms * 8) blocks = num_sms * 8;
    axpy_kernel<<<blocks, 256, 0, s>>>(n, alpha, x, a, out);
    return cudaGetLastError();
}

size_t adjoint_part_floats() { return ADJ_PART; }

}  // namespace gpt
