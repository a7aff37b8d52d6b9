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
struct DzWarpSmem {
    double gi[G_STRIDE];  // (Q + rho I)^{-1}, (R + rho I)^{-1}
    double lv[2 * NS];    // lambda_k, lambda_{k+1}
    double s[NX];
    float cm[C_STRIDE];   // -A_k, -B_k
    float gv[NX];
};

__global__ void __launch_bounds__(32 * DZ_WARPS)
    dz_kernel(BatchView bv, const float *__restrict__ Ginv, const double *__restrict__ Ginv64,
              const float *__restrict__ Cm, const float *__restrict__ g, const float *__restrict__ lambda,
              const double *__restrict__ lambda64, float *__restrict__ dz)
{
    __shared__ DzWarpSmem sm_all[DZ_WARPS];
    const int lane = threadIdx.x & 31;
    DzWarpSmem &sm = sm_all[threadIdx.x >> 5];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = bv.j0 + gw; j < bv.j0 + bv.total_knots; j += nw) {
        const int b = bv.inst(j);
        if (!bv.active(b)) continue;
        const int N = bv.N(b), k = j - bv.off(b);
        const bool last = (k == N - 1);
        const float *Cj = Cm + (size_t)C_STRIDE * j;
        const int nl = last ? NS : 2 * NS;
        // ---- all loads of the knot, then the shared-memory stores
        constexpr int NGI = (G_STRIDE + 31) / 32, NCM = (C_STRIDE + 31) / 32;
        const int ngi = last ? SS : G_STRIDE;  // the last knot's block has no R part (buffers of 245N - 49)
        double gi[NGI];
        float cm[NCM];
#pragma unroll
        for (int i = 0; i < NGI; ++i) {
            const int e = lane + 32 * i;
            gi[i] = 0.0;
            if (e < ngi) gi[i] = Ginv64 ? Ginv64[(size_t)G_STRIDE * j + e] : (double)Ginv[(size_t)G_STRIDE * j + e];
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
            if (e < G_STRIDE) sm.gi[e] = gi[i];
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
        if (lane < NS) {
            double a = 0.0;
#pragma unroll
            for (int t = 0; t < NS; ++t) a = fma(sm.gi[lane + NS * t], sm.s[t], a);
            dz[(size_t)NX * j + lane] = (float)a;
        } else if (lane < NX && !last) {
            const int i = lane - NS;
            double a = 0.0;
#pragma unroll
            for (int t = 0; t < NC; ++t) a = fma(sm.gi[SS + i + NC * t], sm.s[NS + t], a);
            dz[(size_t)NX * j + lane] = (float)a;
        }
        __syncwarp();
    }
}

cudaError_t launch_dz(const BatchView &bv, const float *Ginv, const double *Ginv64, const float *C, const float *g,
                      const float *lambda, const double *lambda64, float *dz, int num_sms, cudaStream_t s,
                      int ctas_per_sm)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    int blocks = (bv.total_knots + DZ_WARPS - 1) / DZ_WARPS;
    if (blocks > num_sms * ctas_per_sm) blocks = num_sms * ctas_per_sm;
    dz_kernel<<<blocks, 32 * DZ_WARPS, 0, s>>>(bv, Ginv, Ginv64, C, g, lambda, lambda64, dz);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// merit
// ------------------------------------------------------------------------

struct MeritWarpSmem {
    float x[NX + NS];    // x_k, u_k, x_{k+1}
    float d[NX + NS];    // dz_k, dz_{k+1}
    float goal[3];
    float M[NUM_ALPHAS][CC];
    float cb[NUM_ALPHAS][NQ];
    double qdd[NUM_ALPHAS][NQ];
    JointTrig trig[NUM_ALPHAS];  // sin, cos of q + alpha dq per step size
    float defect[NUM_ALPHAS];
    float cost[NUM_ALPHAS];
};

constexpr int MERIT_WARPS = 4;

__device__ __forceinline__ float alpha_of(int a, int n_alpha)
{
    return n_alpha == 1 ? 0.f : -1.f / (float)(1 << a);  // toplevel.cuh:409, merit.cuh:47
}

// n_alpha = 8: line search (last knot adds ||x_0 + alpha dz_0 - x_s||_1);
// n_alpha = 1: merit at the current iterate (last knot defect 0).
__global__ void __launch_bounds__(32 * MERIT_WARPS)
    merit_kernel(BatchView bv, ProblemParams P, int n_alpha, const float *__restrict__ xu,
                 const float *__restrict__ dz, const float *__restrict__ goal, const float *__restrict__ xs,
                 float *__restrict__ knot_merit)
{
    __shared__ MeritWarpSmem smem_all[MERIT_WARPS];
    const int lane = threadIdx.x & 31;
    MeritWarpSmem &sm = smem_all[threadIdx.x >> 5];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = bv.j0 + gw; j < bv.j0 + bv.total_knots; j += nw) {
        const int b = bv.inst(j);
        if (!bv.active(b)) continue;
        const int N = bv.N(b), k = j - bv.off(b);
        const bool last = (k == N - 1);
        const int len = last ? NS : NX + NS;
        for (int i = lane; i < len; i += 32) {
            sm.x[i] = xu[(size_t)NX * j + i];
            sm.d[i] = (n_alpha > 1) ? dz[(size_t)NX * j + i] : 0.f;
        }
        if (lane < 3) sm.goal[lane] = goal[(size_t)6 * j + lane];
        __syncwarp();
        // sin, cos of every joint at every step size, once (lane = (step size, joint))
        for (int t = lane; t < n_alpha * NQ; t += 32) {
            const int a = t / NQ, i = t - NQ * a;
            sincosf(fmaf(alpha_of(a, n_alpha), sm.d[i], sm.x[i]), &sm.trig[a].s[i], &sm.trig[a].c[i]);
        }
        __syncwarp();

        if (!last) {
            // mass-matrix columns (m < 7) and bias force (m == 7) per step size
            const int rounds = (n_alpha * 8 + 31) / 32;
            for (int rd = 0; rd < rounds; ++rd) {
                const int a = 4 * rd + (lane >> 3), m = lane & 7;
                const int aa = (a < n_alpha) ? a : 0;
                const float al = alpha_of(aa, n_alpha);
                float qd[NQ], qdd[NQ], tau[NQ];
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    qd[i] = (m == 7) ? fmaf(al, sm.d[NQ + i], sm.x[NQ + i]) : 0.f;
                    qdd[i] = (m == i) ? 1.f : 0.f;
                }
                const JointTrig t = sm.trig[aa];
                rnea<false>(t, qd, qdd, -1, -1, tau, nullptr);
                if (a < n_alpha) {
                    if (m < 7) {
#pragma unroll
                        for (int r = 0; r < NQ; ++r) sm.M[a][NQ * m + r] = tau[r];
                    } else {
#pragma unroll
                        for (int r = 0; r < NQ; ++r) sm.cb[a][r] = tau[r];
                    }
                }
            }
            __syncwarp();
            // qdd_a = M_a^{-1} (u_a - c_a): Gauss-Jordan on [M_a | u_a - c_a] by lane groups of 8
            // (lane 8 g + i holds column i), four step sizes per round
            for (int rd = 0; rd < rounds; ++rd) {
                const int a = 4 * rd + (lane >> 3), m = lane & 7;
                const int aa = (a < n_alpha) ? a : 0;
                const float al = alpha_of(aa, n_alpha);
                double col[NQ];
#pragma unroll
                for (int r = 0; r < NQ; ++r)
                    col[r] = (m < NQ) ? 0.5 * ((double)sm.M[aa][NQ * m + r] + (double)sm.M[aa][NQ * r + m])
                                      : (double)fmaf(al, sm.d[NS + r], sm.x[NS + r]) - (double)sm.cb[aa][r];
                gj7_group(col, lane & ~7);
                if (m == NQ && a < n_alpha) {
#pragma unroll
                    for (int r = 0; r < NQ; ++r) sm.qdd[a][r] = col[r];
                }
            }
            __syncwarp();
        }
        if (lane < n_alpha) {
            // defect ||x_{k+1} - f(x_k, u_k)||_1 at xu + alpha dz (integrator.cuh:187-219)
            const int a = lane;
            const float al = alpha_of(a, n_alpha);
            float dsum = 0.f;
            if (!last) {
                const double *qdd = sm.qdd[a];
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    const float q = fmaf(al, sm.d[i], sm.x[i]), qd = fmaf(al, sm.d[NQ + i], sm.x[NQ + i]);
                    const float qn = fmaf(al, sm.d[NX + i], sm.x[NX + i]);
                    const float qdn = fmaf(al, sm.d[NX + NQ + i], sm.x[NX + NQ + i]);
                    float nq, nqd;
                    if (P.integrator == 0) {
                        nq = q + P.dt * qd;
                        nqd = qd + P.dt * (float)qdd[i];
                    } else {
                        nqd = qd + P.dt * (float)qdd[i];
                        nq = q + P.dt * nqd;
                    }
                    dsum += fabsf(qn - nq) + fabsf(qdn - nqd);
                }
            } else if (n_alpha > 1) {
                const int j0 = j - k;
#pragma unroll
                for (int i = 0; i < NS; ++i)
                    dsum += fabsf(fmaf(al, dz[(size_t)NX * j0 + i], xu[(size_t)NX * j0 + i]) - xs[(size_t)NS * b + i]);
            }
            sm.defect[a] = dsum;
        } else if (lane >= 16 && lane < 16 + n_alpha) {
            // tracking cost (iiwa_eepos_plant.cuh:240-290)
            const int a = lane - 16;
            const float al = alpha_of(a, n_alpha);
            float p[3];
            float J = 0.f;
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                const float qd = fmaf(al, sm.d[NQ + i], sm.x[NQ + i]);
                J += 0.5f * (P.qd_cost * qd * qd);
            }
            if (!last) {
#pragma unroll
                for (int i = 0; i < NC; ++i) {
                    const float u = fmaf(al, sm.d[NS + i], sm.x[NS + i]);
                    J += 0.5f * (P.r_cost * u * u);
                }
            }
            const JointTrig t = sm.trig[a];
            fk_lane<false>(t, p, nullptr);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float e = p[d] - sm.goal[d];
                J += 0.5f * P.q_ee * e * e;
            }
            sm.cost[a] = J;
        }
        __syncwarp();
        if (lane < n_alpha) knot_merit[(size_t)NUM_ALPHAS * j + lane] = sm.cost[lane] + P.mu * sm.defect[lane];
        __syncwarp();
    }
}

cudaError_t launch_merit(const BatchView &bv, const ProblemParams &P, int n_alpha, const float *xu, const float *dz,
                         const float *goal, const float *xs, float *knot_merit, int num_sms, cudaStream_t s,
                         int ctas_per_sm)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    int blocks = (bv.total_knots + MERIT_WARPS - 1) / MERIT_WARPS;
    if (blocks > num_sms * ctas_per_sm) blocks = num_sms * ctas_per_sm;
    merit_kernel<<<blocks, 32 * MERIT_WARPS, 0, s>>>(bv, P, n_alpha, xu, dz, goal, xs, knot_merit);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// merit reduction + accept
// ------------------------------------------------------------------------

constexpr int ACC_THREADS = 256;

// Fixed-order sum of knot_merit[8 (kb + k) + a] over k for all a; result in out[a] (all threads).
__device__ void merit_sums(const float *km, int kb, int N, int n_alpha, float *out, double *scratch)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = ACC_THREADS / 32;
    for (int a = 0; a < n_alpha; ++a) {
        double v = 0.0;
        for (int k = tid; k < N; k += ACC_THREADS) v += (double)km[(size_t)NUM_ALPHAS * (kb + k) + a];
        v = warp_sum(v);
        if (lane == 0) scratch[a * NW + warp] = v;
    }
    __syncthreads();
    if (tid < n_alpha) {
        double t = 0.0;
        for (int w = 0; w < NW; ++w) t += scratch[tid * NW + w];
        scratch[NUM_ALPHAS * NW + tid] = t;
    }
    __syncthreads();
    for (int a = 0; a < n_alpha; ++a) out[a] = (float)scratch[NUM_ALPHAS * NW + a];
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
        merit_sums(knot_merit, kb, N, mode == 0 ? 1 : NUM_ALPHAS, m, scratch);
        if (threadIdx.x == 0) {
            float alpha = 0.f;
            if (merits_out) {
                for (int a = 0; a < (mode == 0 ? 1 : NUM_ALPHAS); ++a) merits_out[NUM_ALPHAS * b + a] = m[a];
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
