// gpt_kkt.cu -- KKT formation: one half-warp per knot.
//
// Replaces gato_form_kkt (schur.cuh:391-524) with the per-knot pieces it
// calls: integratorAndGradient (integrator.cuh:159-183), the plant's
// forwardDynamicsAndGradient (rbdfiles/iiwa_eepos_plant.cuh:126-156) and
// trackingCostGradientAndHessian[_lastblock] (iiwa_eepos_plant.cuh:295-401).
//
// Per knot k < N-1 the half-warp computes, with no block-wide barrier:
//   lanes 0..6   M(q) e_j  (inverse dynamics with qd = 0, qdd = e_j)
//   lane  7      c(q, qd)  (bias force)
//   lanes 0..14  FP64 Gauss-Jordan on [M | I | u - c]: Minv columns and qdd = Minv (u - c)
//   lanes 0..13  d ID(q, qd, qdd) / d(q_j | qd_j)  (forward-mode RNEA tangent)
//   all lanes    df/du = [-Minv dID/dx, Minv], A_k, B_k, defect, cost terms
// and writes the reference blocks G_k = {Q_k, R_k}, C_k = {-A_k, -B_k},
// g_k = {q_k, r_k}, c_{k+1}.  The half-warp of knot N-2 also writes the terminal
// Q_{N-1}, q_{N-1} and c_0 = x_0 - x_s (schur.cuh:429-479).  Inside the SQP loop
// (FULL_G false) only the knot-dependent 7x7 position block of Q_k is written: the
// rest of G (the velocity diagonal, R, the zeros) depends on the cost weights only and
// is written once per solve by gconst_kernel.
#include "gpt_common.cuh"
#include "gpt_dyn.cuh"
#include "gpt_internal.h"

namespace gpt {

struct KktWarpSmem {
    float x[NS], u[NC], xn[NS];
    float goal[12];
    float M[CC];
    float cbias[NQ];
    float Minv[CC];
    float qdd[NQ];
    float dfdu[NQ * NX];   // [dqdd/dq dqdd/dqd dqdd/du], col-major 7x21
    float ee[2][3];
    float J[2][21];
    float qv[2][NS];
    JointTrig trig;  // sin, cos of q_k, computed once per knot
};

constexpr int KKT_WARPS = 4;

// Two knots per warp, one per half-warp (lanes hl = 0..15): the dynamics phases keep at most 14
// lanes of a knot busy, so a knot per half-warp halves their instructions per knot.  A half-warp
// without a knot (odd count, last knot of an instance, inactive instance) computes on knot 0's data
// and writes nothing, so both halves take every __syncwarp.  Four CTAs per SM (16 warps; the
// kernel fits 128 registers without spilling).
// The knot a half-warp takes in pair step jp, and the inputs it stages: lane hl loads entries hl,
// hl + 16 and hl + 32 of x_k, u_k, x_{k+1} and entry hl of goal_k, goal_{k+1} (the next step's are
// loaded while the current step computes).
struct KktKnot {
    int j, b, N, k, jj;
    bool valid;
};
__device__ __forceinline__ KktKnot kkt_knot(const BatchView &bv, int jp, int half)
{
    KktKnot kn;
    kn.j = bv.j0 + 2 * jp + half;
    kn.valid = kn.j < bv.j0 + bv.total_knots;
    kn.b = 0;
    kn.N = 2;
    kn.k = 0;
    if (kn.valid) {
        kn.b = bv.inst(kn.j);
        kn.N = bv.N(kn.b);
        kn.k = kn.j - bv.off(kn.b);
        kn.valid = (kn.k < kn.N - 1) && bv.active(kn.b);
    }
    kn.jj = kn.valid ? kn.j : bv.j0;  // the view's first knot always has a successor (N >= 2)
    return kn;
}
__device__ __forceinline__ void kkt_fetch(const float *xu, const float *goal, int jj, int hl, float (&v)[4])
{
    const float *xk = xu + (size_t)NX * jj;
#pragma unroll
    for (int q = 0; q < 3; ++q) v[q] = (hl + 16 * q < NX + NS) ? __ldg(xk + hl + 16 * q) : 0.f;
    v[3] = hl < 12 ? __ldg(goal + (size_t)6 * jj + hl) : 0.f;
}

template <bool FULL_G>
__global__ void __launch_bounds__(32 * KKT_WARPS, 4) kkt_kernel(BatchView bv, ProblemParams P, const float *__restrict__ xu,
                                                           const float *__restrict__ goal,
                                                           const float *__restrict__ xs, float *__restrict__ G,
                                                           float *__restrict__ Cm, float *__restrict__ g,
                                                           float *__restrict__ c)
{
    __shared__ KktWarpSmem smem_all[2 * KKT_WARPS];
    const int lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
    KktWarpSmem &sm = smem_all[2 * (threadIdx.x >> 5) + half];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;

    float pv[4];
    kkt_fetch(xu, goal, kkt_knot(bv, gw, half).jj, hl, pv);
    for (int jp = gw; 2 * jp < bv.total_knots; jp += nw) {
        const KktKnot kn = kkt_knot(bv, jp, half);
        const int j = kn.j, b = kn.b, N = kn.N, k = kn.k;
        const bool valid = kn.valid;
        const bool terminal = valid && (k == N - 2);

        // ---- stage x_k, u_k, x_{k+1}, goal_k, goal_{k+1} (fetched during the previous step)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int i = hl + 16 * q;
            if (i < NS) sm.x[i] = pv[q];
            else if (i < NX) sm.u[i - NS] = pv[q];
            else if (i < NX + NS) sm.xn[i - NX] = pv[q];
        }
        if (hl < 12) sm.goal[hl] = pv[3];
        if (2 * (jp + nw) < bv.total_knots) kkt_fetch(xu, goal, kkt_knot(bv, jp + nw, half).jj, hl, pv);
        __syncwarp();
        if (hl < NQ) sincosf(sm.x[hl], &sm.trig.s[hl], &sm.trig.c[hl]);
        __syncwarp();
        const JointTrig trig = sm.trig;

        // ---- mass-matrix columns (lanes 0..6) and bias force (lane 7)
        {
            float qd[NQ], qdd[NQ], tau[NQ];
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                qd[i] = (hl == 7) ? sm.x[NQ + i] : 0.f;
                qdd[i] = (hl == i) ? 1.f : 0.f;
            }
            rnea<false>(trig, qd, qdd, -1, -1, tau, nullptr);
            if (hl < NQ) {
#pragma unroll
                for (int r = 0; r < NQ; ++r) sm.M[NQ * hl + r] = tau[r];
            } else if (hl == NQ) {
#pragma unroll
                for (int r = 0; r < NQ; ++r) sm.cbias[r] = tau[r];
            }
        }
        __syncwarp();

        // ---- Minv (lanes 7..13) and qdd = Minv (u - c) (lane 14): Gauss-Jordan on [M | I | u - c] in FP64
        {
            double col[NQ];
#pragma unroll
            for (int r = 0; r < NQ; ++r) {
                double v = 0.0;
                if (hl < NQ) v = 0.5 * ((double)sm.M[NQ * hl + r] + (double)sm.M[NQ * r + hl]);  // symmetric part
                else if (hl < 2 * NQ) v = (r == hl - NQ) ? 1.0 : 0.0;
                else if (hl == 2 * NQ) v = (double)sm.u[r] - (double)sm.cbias[r];
                col[r] = v;
            }
            gj7_group(col, 16 * half);
            if (hl >= NQ && hl < 2 * NQ) {
                // Minv column hl - 7: kept for the products below, and dqdd/du's column of df/du
#pragma unroll
                for (int r = 0; r < NQ; ++r) {
                    sm.Minv[NQ * (hl - NQ) + r] = (float)col[r];
                    sm.dfdu[SC + NQ * (hl - NQ) + r] = (float)col[r];
                }
            } else if (hl == 2 * NQ) {
#pragma unroll
                for (int r = 0; r < NQ; ++r) sm.qdd[r] = (float)col[r];
            }
        }
        __syncwarp();

        // ---- dID/dq_j, dID/dqd_j at (q, qd, qdd), lanes 0..13 (lane hl: direction hl of x)
        float dtau[NQ];
        {
            float qd[NQ], qdd[NQ], tau[NQ];
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                qd[i] = sm.x[NQ + i];
                qdd[i] = sm.qdd[i];
            }
            const int dq_dir = (hl < NQ) ? hl : -1;
            const int dqd_dir = (hl >= NQ && hl < NS) ? hl - NQ : -1;
            rnea<true>(trig, qd, qdd, dq_dir, dqd_dir, tau, dtau);
        }
        // ---- df/du (iiwa_eepos_plant.cuh:142-155): lane hl < 14 forms column hl of -Minv dID/dx from its
        // own tangent; the Minv columns came from the elimination
        if (hl < NS) {
#pragma unroll 1
            for (int r = 0; r < NQ; ++r) {
                float acc = 0.f;
#pragma unroll
                for (int t = 0; t < NQ; ++t) acc += sm.Minv[r + NQ * t] * dtau[t];
                sm.dfdu[NQ * hl + r] = -acc;
            }
        }
        // ---- end-effector position and Jacobian (lane 0 at x_k, lane 1 at the terminal state)
        if (hl == 0) {
            fk_lane<true>(trig, sm.ee[0], sm.J[0]);
        } else if (hl == 1 && terminal && !P.ref_terminal) {
            JointTrig t2;
            joint_trig(sm.xn, t2);
            fk_lane<true>(t2, sm.ee[1], sm.J[1]);
        }
        __syncwarp();

        // ---- cost gradient (iiwa_eepos_plant.cuh:329-354)
        if (hl < NS) {
            float v;
            if (hl < NQ) {
                const float *J = sm.J[0];
                v = P.q_ee * (J[3 * hl] * (sm.ee[0][0] - sm.goal[0]) + J[3 * hl + 1] * (sm.ee[0][1] - sm.goal[1]) +
                              J[3 * hl + 2] * (sm.ee[0][2] - sm.goal[2]));
            } else {
                v = P.qd_cost * sm.x[hl];
            }
            sm.qv[0][hl] = v;
        }
        __syncwarp();
        if (terminal && hl < NS) {
            const int i = hl;
            const int which = P.ref_terminal ? 0 : 1;
            const float *xt = P.ref_terminal ? sm.x : sm.xn;
            // terminal target: goal_{N-1}; in the reference's layout (ref_terminal) the kernel
            // reserves 6 shared floats for the goal but copies 12 (schur.cuh:413-425), so
            // goal_{N-1} lands on Q_{N-2}'s first row and is overwritten by q_0 q_j before the
            // terminal cost call reads it (iiwa_eepos_plant.cuh:396-401)
            float t0 = sm.goal[6], t1 = sm.goal[7], t2 = sm.goal[8];
            if (P.ref_terminal) {
                const float q0 = sm.qv[0][0];
                t0 = q0 * q0;
                t1 = q0 * sm.qv[0][1];
                t2 = q0 * sm.qv[0][2];
            }
            float v;
            if (i < NQ) {
                const float *J = sm.J[which];
                v = P.q_ee * (J[3 * i] * (sm.ee[which][0] - t0) + J[3 * i + 1] * (sm.ee[which][1] - t1) +
                              J[3 * i + 2] * (sm.ee[which][2] - t2));
            } else {
                v = P.qd_cost * xt[i];
            }
            sm.qv[1][i] = v;
        }
        __syncwarp();

        if (valid) {
            // ---- C_k = {-A_k, -B_k} (integrator.cuh:85-126, sign from schur.cuh:519-520): lane r writes row r
            // of the 21 columns (each store a contiguous column of 14 floats per half-warp)
            float *Ck = Cm + (size_t)C_STRIDE * j;
            const float dt = P.dt;
            if (hl < NS) {
                const int r = hl, rq = r < NQ ? r : r - NQ;
                if (P.integrator == 0) {
#pragma unroll
                    for (int col = 0; col < NS; ++col) {
                        float val = (float)(r == col);
                        if (r < NQ && r == col - NQ) val += dt;
                        if (r >= NQ) val += dt * sm.dfdu[col * NQ + r - NQ];
                        Ck[r + NS * col] = -val;
                    }
#pragma unroll
                    for (int col = 0; col < NC; ++col)
                        Ck[SS + r + NS * col] = -((r >= NQ) ? dt * sm.dfdu[(NS + col) * NQ + r - NQ] : 0.f);
                } else {
                    const float dtv = (r == rq) ? dt : 1.f;
#pragma unroll
                    for (int col = 0; col < NS; ++col)
                        Ck[r + NS * col] = -((float)(r == col) + dt * (float)(r == col - NQ) +
                                             dt * sm.dfdu[col * NQ + rq] * dtv);
#pragma unroll
                    for (int col = 0; col < NC; ++col) Ck[SS + r + NS * col] = -(dt * sm.dfdu[SC + col * NQ + rq] * dtv);
                }
            }
            // ---- defect c_{k+1} = x_{k+1} - f(x_k, u_k)  (integrator.cuh:25-83)
            if (hl < NQ) {
                const float q = sm.x[hl], qd = sm.x[NQ + hl], a = sm.qdd[hl];
                float nq, nqd;
                if (P.integrator == 0) {
                    nq = q + dt * qd;
                    nqd = qd + dt * a;
                } else {
                    nqd = qd + dt * a;
                    nq = q + dt * nqd;
                }
                float *cn = c + (size_t)NS * (j + 1);
                cn[hl] = sm.xn[hl] - nq;
                cn[NQ + hl] = sm.xn[NQ + hl] - nqd;
            }
            // ---- G_k = {Q_k, R_k}, g_k = {q_k, r_k}
            float *Gk = G + (size_t)G_STRIDE * j;
            if constexpr (FULL_G) {
                for (int e = hl; e < G_STRIDE; e += 16) {
                    float v;
                    if (e < SS) {
                        const int i = e / NS, jq = e - NS * i;
                        v = (i < NQ && jq < NQ) ? sm.qv[0][i] * sm.qv[0][jq] : ((i == jq) ? P.qd_cost : 0.f);
                    } else {
                        v = ((e - SS) % (NC + 1) == 0) ? P.r_cost : 0.f;
                    }
                    Gk[e] = v;
                }
            } else if (hl < NQ) {
#pragma unroll
                for (int i = 0; i < NQ; ++i) Gk[NS * i + hl] = sm.qv[0][i] * sm.qv[0][hl];
            }
            for (int e = hl; e < NX; e += 16)
                g[(size_t)NX * j + e] = (e < NS) ? sm.qv[0][e] : P.r_cost * sm.u[e - NS];
            if (terminal) {
                float *Gt = G + (size_t)G_STRIDE * (j + 1);
                if constexpr (FULL_G) {
                    for (int e = hl; e < SS; e += 16) {
                        const int i = e / NS, jq = e - NS * i;
                        Gt[e] = (i < NQ && jq < NQ) ? sm.qv[1][i] * sm.qv[1][jq] : ((i == jq) ? P.qd_cost : 0.f);
                    }
                } else if (hl < NQ) {
#pragma unroll
                    for (int i = 0; i < NQ; ++i) Gt[NS * i + hl] = sm.qv[1][i] * sm.qv[1][hl];
                }
                if (hl < NS) {
                    g[(size_t)NX * (j + 1) + hl] = sm.qv[1][hl];
                    const int j0 = j - k;
                    c[(size_t)NS * j0 + hl] = xu[(size_t)NX * j0 + hl] - xs[(size_t)NS * b + hl];
                }
            }
        }
        __syncwarp();
    }
}

// The cost-weight-only entries of G for every knot of the view: Q's velocity diagonal and zeros outside
// the position block, R = r_cost I (the terminal knot has no R).  One thread per entry.
__global__ void gconst_kernel(BatchView bv, float qd_cost, float r_cost, float *__restrict__ G)
{
    const size_t n = (size_t)G_STRIDE * bv.total_knots;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int e = (int)(t % G_STRIDE);
        const int j = bv.j0 + (int)(t / G_STRIDE);
        const int b = bv.inst(j);
        if (!bv.active(b)) continue;
        const bool last = j - bv.off(b) == bv.N(b) - 1;
        float *Gk = G + (size_t)G_STRIDE * j;
        if (e < SS) {
            const int i = e / NS, jq = e - NS * i;
            if (i < NQ && jq < NQ) continue;  // the position block: kkt_kernel's
            Gk[e] = (i == jq) ? qd_cost : 0.f;
        } else if (!last) {
            Gk[e] = ((e - SS) % (NC + 1) == 0) ? r_cost : 0.f;
        }
    }
}

cudaError_t launch_kkt(const BatchView &bv, const ProblemParams &P, const float *xu, const float *goal,
                       const float *xs, float *G, float *C, float *g, float *c, int num_sms, cudaStream_t s,
                       int ctas_per_sm, bool full_g)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    int warps = (bv.total_knots + 1) / 2;  // two knots per warp
    int blocks = (warps + KKT_WARPS - 1) / KKT_WARPS;
    const int cap = num_sms * ctas_per_sm;
    if (blocks > cap) blocks = cap;
    if (full_g)
        kkt_kernel<true><<<blocks, 32 * KKT_WARPS, 0, s>>>(bv, P, xu, goal, xs, G, C, g, c);
    else
        kkt_kernel<false><<<blocks, 32 * KKT_WARPS, 0, s>>>(bv, P, xu, goal, xs, G, C, g, c);
    return cudaGetLastError();
}

cudaError_t launch_kkt_gconst(const BatchView &bv, const ProblemParams &P, float *G, int num_sms, cudaStream_t s)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    const size_t n = (size_t)G_STRIDE * bv.total_knots;
    size_t blocks = (n + 255) / 256;
    if (blocks > (size_t)num_sms * 8) blocks = (size_t)num_sms * 8;
    gconst_kernel<<<(unsigned)blocks, 256, 0, s>>>(bv, P.qd_cost, P.r_cost, G);
    return cudaGetLastError();
}

}  // namespace gpt
