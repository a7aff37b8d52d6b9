// gpt_grid.cu -- batched rigid-body library kernels of the iiwa14 (the standalone GRiD kernels the
// reference ships, rbdfiles/iiwa_eepos_grid.cuh, called one state per launch there):
//
//   ee_pose_kernel  end_effector_positions_kernel (:2091-2110, inner :2015-2090): xyz + roll /
//                   pitch / yaw per row, one thread per row (generateeepos.cu:101-107 launches it
//                   once per trajectory row)
//   fd_kernel       forward_dynamics (:4351-4395): qdd = M^{-1}(u - c(q, qd)), gravity 0, one group
//                   of 8 lanes per row (fd_group)
//   fd_grad_kernel  forwardDynamicsAndGradient (rbdfiles/iiwa_eepos_plant.cuh:130-160): qdd and
//                   df/du = [-M^{-1} dID/dq, -M^{-1} dID/dqd, M^{-1}] (7 x 21, column-major), one
//                   half-warp per row with the lane roles of kkt_kernel
//
// Rows are read with a caller-given stride, so the rows of a trajectory (21 floats: x, u) and plain
// states (14 floats) are both accepted.
#include "gpt_common.cuh"
#include "gpt_dyn.cuh"
#include "gpt_internal.h"

namespace gpt {

__global__ void __launch_bounds__(128) ee_pose_kernel(uint32_t n, const float *__restrict__ x, uint32_t stride,
                                                      float *__restrict__ pose)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float q[NQ];
#pragma unroll
    for (int j = 0; j < NQ; ++j) q[j] = x[(size_t)stride * i + j];
    JointTrig t;
    joint_trig(q, t);
    float p[6];
    fk_pose_lane(t, p);
#pragma unroll
    for (int j = 0; j < 6; ++j) pose[(size_t)6 * i + j] = p[j];
}

__global__ void __launch_bounds__(128) fd_kernel(uint32_t n, const float *__restrict__ xu, uint32_t stride,
                                                 float *__restrict__ qdd)
{
    const int lane = threadIdx.x & 31, m = lane & 7, base = lane & ~7;
    const uint32_t raw = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const bool live = raw < n;
    const uint32_t i = live ? raw : 0u;  // groups past the end follow row 0 (all lanes shuffle) and store nothing
    float q[NQ], qd[NQ], u[NC];
    const float *r = xu + (size_t)stride * i;
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
        q[j] = r[j];
        qd[j] = r[NQ + j];
        u[j] = r[NS + j];
    }
    double col[NQ];
    fd_group(q, qd, u, col, m, base);
    if (live && m == 7) {
#pragma unroll
        for (int j = 0; j < NQ; ++j) qdd[(size_t)NQ * i + j] = (float)col[j];
    }
}

struct FdgSmem {
    float x[NS], u[NC];
    JointTrig trig;
    float M[CC], cb[NQ], Minv[CC], qdd[NQ], dc[NQ * NS];
};
constexpr int FDG_WARPS = 4;

__global__ void __launch_bounds__(32 * FDG_WARPS)
    fd_grad_kernel(uint32_t n, const float *__restrict__ xu, uint32_t stride, float *__restrict__ qdd_out,
                   float *__restrict__ df_out)
{
    __shared__ FdgSmem sm_all[2 * FDG_WARPS];
    const int lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
    FdgSmem &sm = sm_all[2 * (threadIdx.x >> 5) + half];
    const uint32_t raw = (blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const bool live = raw < n;
    const uint32_t row = live ? raw : 0u;  // half-warps past the end follow row 0 and store nothing
    for (int i = hl; i < NX; i += 16) {
        const float v = xu[(size_t)stride * row + i];
        if (i < NS) sm.x[i] = v;
        else sm.u[i - NS] = v;
    }
    __syncwarp();
    if (hl < NQ) sincosf(sm.x[hl], &sm.trig.s[hl], &sm.trig.c[hl]);
    __syncwarp();
    const JointTrig trig = sm.trig;
    {  // mass-matrix columns (lanes 0..6), bias force (lane 7)
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
            for (int r = 0; r < NQ; ++r) sm.cb[r] = tau[r];
        }
    }
    __syncwarp();
    {  // Minv (lanes 7..13), qdd (lane 14): FP64 Gauss-Jordan on [M | I | u - c]
        double col[NQ];
#pragma unroll
        for (int r = 0; r < NQ; ++r) {
            double v = 0.0;
            if (hl < NQ) v = 0.5 * ((double)sm.M[NQ * hl + r] + (double)sm.M[NQ * r + hl]);
            else if (hl < 2 * NQ) v = (r == hl - NQ) ? 1.0 : 0.0;
            else if (hl == 2 * NQ) v = (double)sm.u[r] - (double)sm.cb[r];
            col[r] = v;
        }
        gj7_group(col, 16 * half);
        if (hl >= NQ && hl < 2 * NQ) {
#pragma unroll
            for (int r = 0; r < NQ; ++r) sm.Minv[NQ * (hl - NQ) + r] = (float)col[r];
        } else if (hl == 2 * NQ) {
#pragma unroll
            for (int r = 0; r < NQ; ++r) sm.qdd[r] = (float)col[r];
        }
    }
    __syncwarp();
    {  // dID/dq_j (lanes 0..6), dID/dqd_j (lanes 7..13) at (q, qd, qdd)
        float qd[NQ], qdd[NQ], tau[NQ], dtau[NQ];
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            qd[i] = sm.x[NQ + i];
            qdd[i] = sm.qdd[i];
        }
        const int dq_dir = (hl < NQ) ? hl : -1;
        const int dqd_dir = (hl >= NQ && hl < NS) ? hl - NQ : -1;
        rnea<true>(trig, qd, qdd, dq_dir, dqd_dir, tau, dtau);
        if (hl < NS) {
#pragma unroll
            for (int r = 0; r < NQ; ++r) sm.dc[NQ * hl + r] = dtau[r];
        }
    }
    __syncwarp();
    if (!live) return;
    if (hl < NQ) qdd_out[(size_t)NQ * row + hl] = sm.qdd[hl];
    for (int e = hl; e < NQ * NX; e += 16) {
        float v;
        if (e < NQ * NS) {
            const int col = e / NQ, r = e - NQ * col;
            float acc = 0.f;
#pragma unroll
            for (int t = 0; t < NQ; ++t) acc += sm.Minv[r + NQ * t] * sm.dc[NQ * col + t];
            v = -acc;
        } else {
            v = sm.Minv[e - NQ * NS];
        }
        df_out[(size_t)NQ * NX * row + e] = v;
    }
}

cudaError_t launch_fd_grad(uint32_t n, const float *xu, uint32_t stride, float *qdd, float *df, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    fd_grad_kernel<<<(unsigned)(((size_t)n * 16 + 32 * FDG_WARPS - 1) / (32 * FDG_WARPS)), 32 * FDG_WARPS, 0, s>>>(
        n, xu, stride, qdd, df);
    return cudaGetLastError();
}

cudaError_t launch_ee_pose(uint32_t n, const float *x, uint32_t stride, float *pose, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    ee_pose_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, x, stride, pose);
    return cudaGetLastError();
}

cudaError_t launch_fd(uint32_t n, const float *xu, uint32_t stride, float *qdd, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    fd_kernel<<<(unsigned)(((size_t)n * 8 + 127) / 128), 128, 0, s>>>(n, xu, stride, qdd);
    return cudaGetLastError();
}

}  // namespace gpt
