// glass.cuh -- project-written stand-in for the two GLASS routines the
// reference's kernels call (glass::copy, glass::reduce).  GLASS is a git
// submodule of the reference (.gitmodules:4-6) that is empty in its tree;
// these are restated from the call sites' use of them (schur.cuh:424-521,
// merit.cuh:74-88, integrator.cuh:215, iiwa_eepos_plant.cuh:286):
//   copy(n, x, y)         y[i] = x[i]           (threads of the group stride over i)
//   copy(n, alpha, x, y)  y[i] = alpha * x[i]
//   reduce(n, x)          x[0] = sum of x[0..n-1] (in place, group-synchronised)
// Test infrastructure only: it lets the reference's own kernels be compiled
// and run as a parity oracle.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>

namespace glass {

template <typename T>
__device__ void copy(uint32_t n, const T *x, T *y,
                     cooperative_groups::thread_group g = cooperative_groups::this_thread_block())
{
    for (uint32_t i = g.thread_rank(); i < n; i += g.size()) y[i] = x[i];
}

template <typename T>
__device__ void copy(uint32_t n, T alpha, const T *x, T *y,
                     cooperative_groups::thread_group g = cooperative_groups::this_thread_block())
{
    for (uint32_t i = g.thread_rank(); i < n; i += g.size()) y[i] = alpha * x[i];
}

// pairwise halving: after each round the first ceil(len/2) entries hold the partial sums
template <typename T>
__device__ void reduce(uint32_t n, T *x, cooperative_groups::thread_group g = cooperative_groups::this_thread_block())
{
    g.sync();
    uint32_t len = n;
    while (len > 1) {
        const uint32_t half = (len + 1) / 2;
        for (uint32_t i = g.thread_rank(); i + half < len; i += g.size()) x[i] += x[i + half];
        g.sync();
        len = half;
    }
}

}  // namespace glass
