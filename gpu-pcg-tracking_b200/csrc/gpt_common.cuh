// gpt_common.cuh -- layouts, batch descriptors and small device helpers shared
// by the kernels of the SQP inner loop.
//
// Buffers keep the reference's per-knot block layouts (toplevel.cuh:42-50,
// utils.cuh:121-187) so single-instance calls accept reference-sized buffers.
// A batch concatenates instances knot by knot: knot j of the batch belongs to
// instance b = knot_inst[j], local index k = j - knot_off[b], and every
// per-knot block of every buffer sits at (stride * j).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gpt {

constexpr int NQ = 7;            // joints
constexpr int NS = 14;           // state size (settings.cuh:4)
constexpr int NC = 7;            // control size
constexpr int NX = NS + NC;      // 21 floats of xu per knot
constexpr int SS = NS * NS;      // 196
constexpr int SC = NS * NC;      // 98
constexpr int CC = NC * NC;      // 49
constexpr int G_STRIDE = SS + CC;        // 245 (toplevel.cuh:46)
constexpr int C_STRIDE = SS + SC;        // 294 (toplevel.cuh:47)
constexpr int S_STRIDE = 3 * SS;         // 588 (toplevel.cuh:103)
constexpr int NUM_ALPHAS = 8;            // toplevel.cuh:55
constexpr int PK = 408;                  // packed Schur row for the PCG: left 196 + tri 105 + Pinv tri 105 + 2
constexpr int PK64 = 302;                // FP64 packed Schur row: left 196 + diagonal lower triangle 105 + 1 pad (doubles)
// Compact FP64 inverses of a knot's cost blocks (doubles; the FP64 Schur kernel's output for dz):
// [0] flags (1: (Q + rho I)^{-1} is not block diagonal, 2: (R + rho I)^{-1} is not diagonal -- that
// block is then in the full-layout buffer of G_STRIDE doubles per knot instead), [1, 50) the
// position block's inverse (7 x 7, column-major), [50, 57) the velocity diagonal, [57, 64) the
// control diagonal (zero for an instance's last knot).
constexpr int GC64 = 64, GC_POS = 1, GC_VEL = 50, GC_CTL = 57;
constexpr int MAX_KNOTS = 1024;          // per-instance horizon limit of the library

// Per-instance SQP state kept on the device across the phases of one solve.
struct InstState {
    float rho, drho, merit0, merit_init;
    float rho_reset;
    uint32_t active;          // 1 while the SQP loop of this instance runs
    uint32_t sqp_iters;
    uint32_t exit_flags;      // GPT_EXIT_* bits (include/gpt.h)
    uint32_t pcg_iters_total;
    uint32_t pcg_maxiter_count;
    uint32_t ls_fail_count;
    uint32_t last_pcg_iters;
    uint32_t last_pcg_exit;
    uint32_t pad[3];
};

struct BatchView {
    int B;                   // instances
    int total_knots;         // sum of horizons
    const int *knot_off;     // [B+1] prefix offsets, nullptr => single instance of total_knots
    const int *knot_inst;    // [total_knots] owning instance, nullptr => single instance
    InstState *st;           // [B] or nullptr (always active)
    // A view of a contiguous sub-range of a batch: instances b0 .. b0+B-1, owning knots
    // j0 .. j0+total_knots-1.  Instance and knot indices stay those of the whole batch.
    int j0 = 0, b0 = 0;

    __device__ __forceinline__ int inst(int j) const { return knot_inst ? knot_inst[j] : 0; }
    __device__ __forceinline__ int off(int b) const { return knot_off ? knot_off[b] : 0; }
    __device__ __forceinline__ int N(int b) const
    {
        return knot_off ? knot_off[b + 1] - knot_off[b] : total_knots;
    }
    __device__ __forceinline__ bool active(int b) const { return st == nullptr || st[b].active != 0; }
};

// Physical problem parameters (the reference's compile-time macros, runtime here).
struct ProblemParams {
    float dt;          // timestep (runme.cu:65)
    int integrator;    // 0 explicit Euler, 1 semi-implicit Euler (integrator.cuh:25-126)
    float q_ee;        // end-effector position weight
    float qd_cost;     // QD_COST
    float r_cost;      // R_COST
    float mu;          // merit penalty (toplevel.cuh:54)
    int ref_terminal;  // 1: terminal Q,q at x_{N-2}, target Q_{N-2}[0][0..2], as the reference's kernel computes
};

// Reciprocal by two Newton-Raphson steps r <- r + r (1 - x r) from the PTX approximation
// rcp.approx.ftz.f64 (quadratic convergence: a seed accurate to ~2^-20 reaches FP64 rounding);
// x is a positive pivot of an SPD elimination, far from the FP64 range limits
__device__ __forceinline__ double rcp_newton(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

// FP64 tensor-core MMA (mma.sync m8n8k4, the FP64 shape; tcgen05 has no FP64 kind): d += a b for an
// 8x4 by 4x8 tile pair.  Fragments: a = A(g, t), b = B(t, g), d = D(g, 2t + {0, 1}), with
// g = lane >> 2, t = lane & 3.
__device__ __forceinline__ void mma884_f64(double (&d)[2], double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}
// c[I][J] += sum over k < 4 KS of A(8I + g, k) B(k, 8J + g'), one warp: TI x TJ output tiles of 8x8,
// operands read through the element accessors A(i, k), B(k, j) (which return 0 in the padding)
template <int TI, int TJ, int KS, class FA, class FB>
__device__ __forceinline__ void warp_dmma(FA A, FB B, double (&c)[TI][TJ][2], int lane)
{
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kk = 0; kk < KS; ++kk) {
        const int k = 4 * kk + t;
        double a[TI], b[TJ];
#pragma unroll
        for (int I = 0; I < TI; ++I) a[I] = A(8 * I + g, k);
#pragma unroll
        for (int J = 0; J < TJ; ++J) b[J] = B(k, 8 * J + g);
#pragma unroll
        for (int I = 0; I < TI; ++I)
#pragma unroll
            for (int J = 0; J < TJ; ++J) mma884_f64(c[I][J], a[I], b[J]);
    }
}
// hand each element (i, j, value) of the tiles to st
template <int TI, int TJ, class F>
__device__ __forceinline__ void warp_dmma_store(const double (&c)[TI][TJ][2], F st, int lane)
{
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int I = 0; I < TI; ++I)
#pragma unroll
        for (int J = 0; J < TJ; ++J)
#pragma unroll
            for (int e = 0; e < 2; ++e) st(8 * I + g, 8 * J + 2 * t + e, c[I][J][e]);
}

// Asynchronous global -> shared copies (cp.async): 16 bytes (both addresses 16-byte aligned, L1
// bypassed) or 4 bytes; a thread's copies form groups (commit) it can wait for (all but the newest N).
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(sdst)),
                 "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *sdst, const void *gsrc)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(sdst)),
                 "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace gpt
