// gpt_merit.cu -- primal step recovery, merit / line search and the SQP
// accept-and-update step, all on the device.
//
//   dz_kernel      oldschur.cuh:966-1105 (compute_dz), one warp per knot
//   merit_kernel   merit.cuh:16-94 (ls_gato_compute_merit, all 8 step sizes in
//                  one launch) and merit.cuh:99-145 (compute_merit, alpha = 0);
//                  one warp per knot, lanes = (step size, mass-matrix column)
//   accept_kernel  toplevel.cuh:377-444: argmin merit, rho schedule, the
//                  saxpy xu += alpha dz (cuBLAS in the reference) -- one block
//                  per instance, deterministic fixed-order merit sums
#include "gpt_common.cuh"
#include "gpt_dyn.cuh"
#include "gpt_internal.h"

namespace gpt {

constexpr int DZ_WARPS = 4;

// dz from lambda (FP32 or, when lambda64 is given, FP64).  The right-hand sides
// q_k - lambda_k - (-A_k)^T lambda_{k+1} and r_k - (-B_k)^T lambda_{k+1} cancel
// heavily, so they are accumulated in FP64 before the inverses apply.  Every input of a
// knot is loaded in one batch (the kernel is bound by load latency) and staged in shared memory.
// COMPACT: the inverses come as launch_schur64's compact blocks (GC64 doubles per knot: the position
// block, the velocity and control diagonals -- a quarter of the full layout's bytes); a block its
// flags mark as not (block) diagonal is read from the full layout instead.  The sums are those of
// the full layout term by term (the skipped terms are exact zeros).
template <bool COMPACT>
struct DzWarpSmem {
    double gi[COMPACT ? GC64 : G_STRIDE];  // (Q + rho I)^{-1}, (R + rho I)^{-1}
    double lv[2 * NS];                     // lambda_k, lambda_{k+1}
    double s[NX];
    float cm[C_STRIDE];  // -A_k, -B_k
    float gv[NX];
};

template <bool COMPACT>
__global__ void __launch_bounds__(32 * DZ_WARPS)
    dz_kernel(BatchView bv, const float *__restrict__ Ginv, const double *__restrict__ Ginv64,
              const double *__restrict__ Ginv64c, const float *__restrict__ Cm, const float *__restrict__ g,
              const float *__restrict__ lambda, const double *__restrict__ lambda64, float *__restrict__ dz)
{
    __shared__ DzWarpSmem<COMPACT> sm_all[DZ_WARPS];
    const int lane = threadIdx.x & 31;
    DzWarpSmem<COMPACT> &sm = sm_all[threadIdx.x >> 5];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    constexpr int GIN = COMPACT ? GC64 : G_STRIDE;
    for (int j = bv.j0 + gw; j < bv.j0 + bv.total_knots; j += nw) {
        const int b = bv.inst(j);
        if (!bv.active(b)) continue;
        const int N = bv.N(b), k = j - bv.off(b);
        const bool last = (k == N - 1);
        const float *Cj = Cm + (size_t)C_STRIDE * j;
        const int nl = last ? NS : 2 * NS;
        // ---- all loads of the knot, then the shared-memory stores
        constexpr int NGI = (GIN + 31) / 32, NCM = (C_STRIDE + 31) / 32;
        // the last knot's block has no R part (buffers of 245N - 49)
        const int ngi = COMPACT ? GC64 : (last ? SS : G_STRIDE);
        double gi[NGI];
        float cm[NCM];
#pragma unroll
        for (int i = 0; i < NGI; ++i) {
            const int e = lane + 32 * i;
            gi[i] = 0.0;
            if (COMPACT)
                gi[i] = Ginv64c[(size_t)GC64 * j + e];
            else if (e < ngi)
                gi[i] = Ginv64 ? Ginv64[(size_t)G_STRIDE * j + e] : (double)Ginv[(size_t)G_STRIDE * j + e];
        }
#pragma unroll
        for (int i = 0; i < NCM; ++i) {
            const int e = lane + 32 * i;
            cm[i] = (!last && e < C_STRIDE) ? Cj[e] : 0.f;
        }
        double lvv = 0.0;
        if (lane < nl) lvv = lambda64 ? lambda64[(size_t)NS * j + lane] : (double)lambda[(size_t)NS * j + lane];
        float gvv = 0.f;
        if (lane < NX && (lane < NS || !last)) gvv = g[(size_t)NX * j + lane];
#pragma unroll
        for (int i = 0; i < NGI; ++i) {
            const int e = lane + 32 * i;
            if (e < GIN) sm.gi[e] = gi[i];
        }
#pragma unroll
        for (int i = 0; i < NCM; ++i) {
            const int e = lane + 32 * i;
            if (e < C_STRIDE) sm.cm[e] = cm[i];
        }
        if (lane < 2 * NS) sm.lv[lane] = lvv;
        if (lane < NX) sm.gv[lane] = gvv;
        __syncwarp();
        if (lane < NS) {
            // q_k - (lambda_k + (-A_k)^T lambda_{k+1})
            double a = 0.0;
            if (!last) {
#pragma unroll
                for (int t = 0; t < NS; ++t) a = fma((double)sm.cm[lane * NS + t], sm.lv[NS + t], a);
            }
            sm.s[lane] = (double)sm.gv[lane] - (sm.lv[lane] + a);
        } else if (lane < NX && !last) {
            // r_k - (-B_k)^T lambda_{k+1}
            const int i = lane - NS;
            double a = 0.0;
#pragma unroll
            for (int t = 0; t < NS; ++t) a = fma((double)sm.cm[SS + i * NS + t], sm.lv[NS + t], a);
            sm.s[lane] = (double)sm.gv[lane] - a;
        }
        __syncwarp();
        const int flags = COMPACT ? (int)sm.gi[0] : 0;
        const double *full = COMPACT ? Ginv64 + (size_t)G_STRIDE * j : nullptr;  // the flagged blocks
        if (lane < NS) {
            double a = 0.0;
            if (!COMPACT) {
#pragma unroll
                for (int t = 0; t < NS; ++t) a = fma(sm.gi[lane + NS * t], sm.s[t], a);
            } else if (flags & 1) {
                for (int t = 0; t < NS; ++t) a = fma(full[lane + NS * t], sm.s[t], a);
            } else if (lane < NC) {
#pragma unroll
                for (int t = 0; t < NC; ++t) a = fma(sm.gi[GC_POS + lane + NC * t], sm.s[t], a);
            } else {
                a = sm.gi[GC_VEL + lane - NC] * sm.s[lane];
            }
            dz[(size_t)NX * j + lane] = (float)a;
        } else if (lane < NX && !last) {
            const int i = lane - NS;
            double a = 0.0;
            if (!COMPACT) {
#pragma unroll
                for (int t = 0; t < NC; ++t) a = fma(sm.gi[SS + i + NC * t], sm.s[NS + t], a);
            } else if (flags & 2) {
                for (int t = 0; t < NC; ++t) a = fma(full[SS + i + NC * t], sm.s[NS + t], a);
            } else {
                a = sm.gi[GC_CTL + i] * sm.s[lane];
            }
            dz[(size_t)NX * j + lane] = (float)a;
        }
        __syncwarp();
    }
}

cudaError_t launch_dz(const BatchView &bv, const float *Ginv, const double *Ginv64, const double *Ginv64c,
                      const float *C, const float *g, const float *lambda, const double *lambda64, float *dz,
                      int num_sms, cudaStream_t s, int ctas_per_sm)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    if (Ginv64c && !Ginv64) return cudaErrorInvalidValue;
    int blocks = (bv.total_knots + DZ_WARPS - 1) / DZ_WARPS;
    if (blocks > num_sms * ctas_per_sm) blocks = num_sms * ctas_per_sm;
    if (Ginv64c)
        dz_kernel<true><<<blocks, 32 * DZ_WARPS, 0, s>>>(bv, Ginv, Ginv64, Ginv64c, C, g, lambda, lambda64, dz);
    else
        dz_kernel<false><<<blocks, 32 * DZ_WARPS, 0, s>>>(bv, Ginv, Ginv64, nullptr, C, g, lambda, lambda64, dz);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// merit
// ------------------------------------------------------------------------

constexpr int MERIT_WARPS = 4;

__device__ __forceinline__ float alpha_of(int a, int n_alpha)
{
    return n_alpha == 1 ? 0.f : -1.f / (float)(1 << a);  // toplevel.cuh:409, merit.cuh:47
}

// One lane per (knot, step size): with the 8 line-search step sizes a warp takes 4 knots, for the
// merit of the iterate (n_alpha = 1) 32.  The lane evaluates its candidate xu + alpha dz at its knot:
// the tracking cost (iiwa_eepos_plant.cuh:240-290; forward kinematics for the end-effector term) and
// the defect ||x_{k+1} - f(x_k, u_k)||_1 (integrator.cuh:187-219) with q'' = M^{-1} (u - c(q, q')):
// M by its lower-triangle columns at zero velocity, c by one inverse-dynamics pass, the 7x7 solve by
// an FP32 Cholesky refined in FP64.  The last knot: the line search adds ||x_0 + alpha dz_0 - x_s||_1,
// the iterate's merit no defect (merit.cuh:68-77,135-137).  No shared memory and no warp synchronisation:
// the lanes of a knot read the same addresses (one transaction per warp load).  Four CTAs per SM:
// 128 registers without spilling (the unbounded build took 136, which let three fit).
__global__ void __launch_bounds__(32 * MERIT_WARPS, 4)
    merit_kernel(BatchView bv, ProblemParams P, int n_alpha, const float *__restrict__ xu,
                 const float *__restrict__ dz, const float *__restrict__ goal, const float *__restrict__ xs,
                 float *__restrict__ knot_merit)
{
    const int lane = threadIdx.x & 31;
    const int per = n_alpha > 1 ? NUM_ALPHAS : 1;  // lanes per knot
    const int kpw = 32 / per;                      // knots per warp
    const int slot = lane / per, a = lane - per * slot;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int jend = bv.j0 + bv.total_knots;
    for (int j0 = bv.j0 + gw * kpw; j0 < jend; j0 += nw * kpw) {
        const int j = j0 + slot;
        if (j >= jend) continue;
        const int b = bv.inst(j);
        if (!bv.active(b)) continue;
        const int N = bv.N(b), k = j - bv.off(b);
        const bool last = (k == N - 1);
        const float al = alpha_of(a, n_alpha);
        const bool step = n_alpha > 1;
        const float *xj = xu + (size_t)NX * j;
        const float *dj = step ? dz + (size_t)NX * j : nullptr;
        float q[NQ], qd[NQ];
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            q[i] = step ? fmaf(al, dj[i], xj[i]) : xj[i];
            qd[i] = step ? fmaf(al, dj[NQ + i], xj[NQ + i]) : xj[NQ + i];
        }
        JointTrig t;
        joint_trig(q, t);
        // tracking cost
        float J = 0.f;
#pragma unroll
        for (int i = 0; i < NQ; ++i) J += 0.5f * (P.qd_cost * qd[i] * qd[i]);
        float dsum = 0.f;
        if (!last) {
            float u[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i) {
                u[i] = step ? fmaf(al, dj[NS + i], xj[NS + i]) : xj[NS + i];
                J += 0.5f * (P.r_cost * u[i] * u[i]);
            }
            // defect: q'' = M^{-1} (u - c) of the candidate, one integrator step, against x_{k+1}
            float M[28];
            mass_matrix_lane(t, M);
            float zero[NQ], c[NQ];
#pragma unroll
            for (int i = 0; i < NQ; ++i) zero[i] = 0.f;
            rnea<false>(t, qd, zero, -1, -1, c, nullptr);
            double rhs[NQ], qdd[NQ];
#pragma unroll
            for (int i = 0; i < NQ; ++i) rhs[i] = (double)u[i] - (double)c[i];
            spd7_solve_lane(M, rhs, qdd);
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                const float qn = step ? fmaf(al, dj[NX + i], xj[NX + i]) : xj[NX + i];
                const float qdn = step ? fmaf(al, dj[NX + NQ + i], xj[NX + NQ + i]) : xj[NX + NQ + i];
                float nq, nqd;
                if (P.integrator == 0) {
                    nq = q[i] + P.dt * qd[i];
                    nqd = qd[i] + P.dt * (float)qdd[i];
                } else {
                    nqd = qd[i] + P.dt * (float)qdd[i];
                    nq = q[i] + P.dt * nqd;
                }
                dsum += fabsf(qn - nq) + fabsf(qdn - nqd);
            }
        } else if (step) {
            const int jf = j - k;
#pragma unroll
            for (int i = 0; i < NS; ++i)
                dsum += fabsf(fmaf(al, dz[(size_t)NX * jf + i], xu[(size_t)NX * jf + i]) - xs[(size_t)NS * b + i]);
        }
        float p[3];
        fk_lane<false>(t, p, nullptr);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float e = p[d] - goal[(size_t)6 * j + d];
            J += 0.5f * P.q_ee * e * e;
        }
        knot_merit[(size_t)NUM_ALPHAS * j + a] = J + P.mu * dsum;
    }
}

cudaError_t launch_merit(const BatchView &bv, const ProblemParams &P, int n_alpha, const float *xu, const float *dz,
                         const float *goal, const float *xs, float *knot_merit, int num_sms, cudaStream_t s,
                         int ctas_per_sm)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    const int kpw = n_alpha > 1 ? 32 / NUM_ALPHAS : 32;
    const int warps = (bv.total_knots + kpw - 1) / kpw;
    int blocks = (warps + MERIT_WARPS - 1) / MERIT_WARPS;
    if (blocks > num_sms * ctas_per_sm) blocks = num_sms * ctas_per_sm;
    merit_kernel<<<blocks, 32 * MERIT_WARPS, 0, s>>>(bv, P, n_alpha, xu, dz, goal, xs, knot_merit);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// merit reduction + accept
// ------------------------------------------------------------------------

constexpr int ACC_THREADS = 256;

// Fixed-order sum of knot_merit[8 (kb + k) + a] over k for a < NA; result in out[a] (all threads).  A
// thread loads its knots' NA merits together (two 16-byte loads for the 8 step sizes) and keeps NA
// running sums; each sum adds the knots in the same order as a pass per step size would.
template <int NA>
__device__ __forceinline__ void merit_sums(const float *km, int kb, int N, float (&out)[NA], double *scratch)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = ACC_THREADS / 32;
    double v[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) v[a] = 0.0;
    for (int k = tid; k < N; k += ACC_THREADS) {
        const float *row = km + (size_t)NUM_ALPHAS * (kb + k);
        if constexpr (NA == NUM_ALPHAS) {
            const float4 lo = *reinterpret_cast<const float4 *>(row), hi = *reinterpret_cast<const float4 *>(row + 4);
            const float e[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
            for (int a = 0; a < NA; ++a) v[a] += (double)e[a];
        } else {
#pragma unroll
            for (int a = 0; a < NA; ++a) v[a] += (double)row[a];
        }
    }
#pragma unroll
    for (int a = 0; a < NA; ++a) {
        const double w = warp_sum(v[a]);
        if (lane == 0) scratch[a * NW + warp] = w;
    }
    __syncthreads();
    if (tid < NA) {
        double t = 0.0;
        for (int w = 0; w < NW; ++w) t += scratch[tid * NW + w];
        scratch[NUM_ALPHAS * NW + tid] = t;
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; ++a) out[a] = (float)scratch[NUM_ALPHAS * NW + a];
    __syncthreads();
}

// mode 0: initial merit of the iterate (merit0, toplevel.cuh:235-244)
// mode 1: line-search decision and step (toplevel.cuh:384-444)
__global__ void __launch_bounds__(ACC_THREADS)
    accept_kernel(BatchView bv, int mode, SolverParams SP, const float *__restrict__ knot_merit,
                  const float *__restrict__ dz, float *__restrict__ xu, float *__restrict__ merits_out,
                  uint32_t *__restrict__ active_count)
{
    __shared__ double scratch[NUM_ALPHAS * (ACC_THREADS / 32) + NUM_ALPHAS];
    __shared__ float s_alpha;
    for (int b = bv.b0 + blockIdx.x; b < bv.b0 + bv.B; b += gridDim.x) {
        if (!bv.active(b)) continue;
        const int N = bv.N(b), kb = bv.off(b);
        float m[NUM_ALPHAS];
        if (mode == 0) {
            float m0[1];
            merit_sums<1>(knot_merit, kb, N, m0, scratch);
#pragma unroll
            for (int a = 0; a < NUM_ALPHAS; ++a) m[a] = m0[0];
        } else {
            merit_sums<NUM_ALPHAS>(knot_merit, kb, N, m, scratch);
        }
        if (threadIdx.x == 0) {
            float alpha = 0.f;
            if (merits_out) {
#pragma unroll
                for (int a = 0; a < NUM_ALPHAS; ++a)
                    if (mode != 0 || a == 0) merits_out[NUM_ALPHAS * b + a] = m[a];
            }
            if (bv.st) {
                InstState &s = bv.st[b];
                if (mode == 0) {
                    s.merit0 = m[0];
                    s.merit_init = m[0];
                    if (!isfinite(m[0])) { s.exit_flags |= 4u; s.active = 0; }
                } else {
                    float minm = s.merit0;
                    int best = 0;
                    for (int a = 0; a < NUM_ALPHAS; ++a)
                        if (m[a] < minm) { minm = m[a]; best = a; }
                    const float f = SP.rho_factor;
                    if (minm == s.merit0) {
                        s.drho = fmaxf(s.drho * f, f);
                        s.rho = fmaxf(s.rho * s.drho, SP.rho_min);
                        s.sqp_iters++;
                        s.ls_fail_count++;
                        if (s.rho > SP.rho_max) {
                            s.exit_flags |= 1u;
                            s.rho = s.rho_reset;
                            s.active = 0;
                        }
                    } else {
                        alpha = -1.f / (float)(1 << best);
                        s.drho = fminf(s.drho / f, 1.f / f);
                        s.rho = fmaxf(s.rho * s.drho, SP.rho_min);
                        s.sqp_iters++;
                        s.merit0 = minm;
                    }
                    if (s.active && s.sqp_iters >= SP.sqp_max_iter) {
                        s.active = 0;
                        s.exit_flags |= 8u;
                    }
                    // a failed factorisation or a non-finite reduction leaves no usable iterate
                    if (s.exit_flags & (GPT_EXIT_NONFINITE | GPT_EXIT_FACTOR)) s.active = 0;
                }
                if (active_count && s.active) atomicAdd(active_count, 1u);
            }
            s_alpha = alpha;
        }
        __syncthreads();
        const float alpha = s_alpha;
        if (alpha != 0.f) {
            const int len = NX * N - NC;
            float *xb = xu + (size_t)NX * kb;
            const float *db = dz + (size_t)NX * kb;
            for (int i = threadIdx.x; i < len; i += ACC_THREADS) xb[i] = fmaf(alpha, db[i], xb[i]);
        }
        __syncthreads();
    }
}

cudaError_t launch_accept(const BatchView &bv, int mode, const SolverParams &SP, const float *knot_merit,
                          const float *dz, float *xu, float *merits_out, uint32_t *active_count, int num_sms,
                          cudaStream_t s)
{
    if (bv.B <= 0) return cudaSuccess;
    int blocks = bv.B;
    if (blocks > num_sms * 8) blocks = num_sms * 8;
    accept_kernel<<<blocks, ACC_THREADS, 0, s>>>(bv, mode, SP, knot_merit, dz, xu, merits_out, active_count);
    return cudaGetLastError();
}

// Per-instance start of a solve: x_s = x_0 (toplevel.cuh:110), state from the host image.
__global__ void trace_record_kernel(BatchView bv, int phase, const float *__restrict__ merits,
                                    gpt_iterate_record *__restrict__ rec)
{
    for (int b = bv.b0 + blockIdx.x * blockDim.x + threadIdx.x; b < bv.b0 + bv.B; b += gridDim.x * blockDim.x) {
        const InstState &s = bv.st[b];
        gpt_iterate_record &r = rec[b];
        if (phase == 0) {
            r.rho = s.rho;
            r.merit_prev = s.merit0;
            r.active = s.active;
            r.rho_next = s.rho;
            r.alpha = 0.f;
            r.pcg_iters = 0;
            for (int a = 0; a < NUM_ALPHAS; ++a) r.merits[a] = 0.f;
            continue;
        }
        if (!r.active) continue;
        // the accept kernel's decision, same comparisons in the same order
        float minm = r.merit_prev;
        int best = 0;
        for (int a = 0; a < NUM_ALPHAS; ++a) {
            const float m = merits[NUM_ALPHAS * b + a];
            r.merits[a] = m;
            if (m < minm) {
                minm = m;
                best = a;
            }
        }
        r.alpha = (minm == r.merit_prev) ? 0.f : -1.f / (float)(1 << best);
        r.rho_next = s.rho;
        r.pcg_iters = s.last_pcg_iters;
    }
}

cudaError_t launch_trace_record(const BatchView &bv, int phase, const float *merits, gpt_iterate_record *rec,
                                int num_sms, cudaStream_t s)
{
    if (bv.B <= 0) return cudaSuccess;
    if (!bv.st || !rec || (phase == 1 && !merits)) return cudaErrorInvalidValue;
    int blocks = (bv.B + 127) / 128;
    if (blocks > num_sms) blocks = num_sms;
    trace_record_kernel<<<blocks, 128, 0, s>>>(bv, phase, merits, rec);
    return cudaGetLastError();
}

__global__ void init_kernel(BatchView bv, const float *__restrict__ xu, float *__restrict__ xs)
{
    for (int b = bv.b0 + blockIdx.x; b < bv.b0 + bv.B; b += gridDim.x) {
        const int kb = bv.off(b);
        if (threadIdx.x < NS) xs[(size_t)NS * b + threadIdx.x] = xu[(size_t)NX * kb + threadIdx.x];
    }
}

cudaError_t launch_init(const BatchView &bv, const float *xu, float *xs, int num_sms, cudaStream_t s)
{
    if (bv.B <= 0) return cudaSuccess;
    int blocks = bv.B;
    if (blocks > num_sms * 8) blocks = num_sms * 8;
    init_kernel<<<blocks, 32, 0, s>>>(bv, xu, xs);
    return cudaGetLastError();
}

}  // namespace gpt
