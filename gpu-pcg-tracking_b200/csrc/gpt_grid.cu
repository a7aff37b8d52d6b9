// gpt_grid.cu -- batched rigid-body library kernels of the iiwa14 (the standalone GRiD kernels the
// reference ships, rbdfiles/iiwa_eepos_grid.cuh, called one state per launch there):
//
//   ee_pose_kernel  end_effector_positions_kernel (:2091-2110, inner :2015-2090): xyz + roll /
//                   pitch / yaw per row, one thread per row (generateeepos.cu:101-107 launches it
//                   once per trajectory row)
//   fd_kernel       forward_dynamics (:4351-4395): qdd = M^{-1}(u - c(q, qd)), gravity 0, one group
//                   of 8 lanes per row (fd_group)
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
