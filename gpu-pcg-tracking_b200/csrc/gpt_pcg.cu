// gpt_pcg.cu -- preconditioned conjugate gradient on the block-tridiagonal
// Schur system, one thread block per instance.
//
// Replaces the GPU-PCG cooperative kernel the reference launches at
// toplevel.cuh:135-157,292-294 (pcg<T, STATE_SIZE, KNOT_POINTS>; its source
// is a submodule absent from the reference tree).  Solves S lambda = gamma,
// warm-started from lambda, with the block-Jacobi preconditioner Pinv (the
// only Pinv blocks the reference fills, oldschur.cuh:926-933).  One block owns
// one instance: the search direction and residual live in shared memory, the
// block-tridiagonal product reads S from L2/HBM, and all dot products (rho,
// alpha in the classical notation) are reduced in FP64 with a fixed order.
// No grid-wide synchronisation: instances never wait on each other.
//
// Exit test: mode 0 ||r||_2 <= tol ||gamma||_2 (relative residual);
//            mode 1 |r^T Pinv r| < tol.
#include "gpt_common.cuh"
#include "gpt_internal.h"

namespace gpt {

constexpr int PCG_THREADS = 512;
constexpr int PCG_RPT = (NS * MAX_PCG_KNOTS + PCG_THREADS - 1) / PCG_THREADS;  // rows per thread

// Sums NV doubles over the block in a fixed order; every thread gets the result.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NWARP = PCG_THREADS / 32;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) scratch[q * NWARP + warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double t = (lane < NWARP) ? scratch[q * NWARP + lane] : 0.0;
            t = warp_sum(t);
            if (lane == 0) scratch[NV * NWARP + q] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = scratch[NV * NWARP + q];
    __syncthreads();
}

__global__ void __launch_bounds__(PCG_THREADS)
    pcg_kernel(BatchView bv, const float *__restrict__ S, const float *__restrict__ Pinv, int pinv_stride,
               int pinv_off, const float *__restrict__ gamma, float *__restrict__ lambda, int max_iter, float tol,
               int exit_mode, uint32_t *__restrict__ out_iters, uint32_t *__restrict__ pcg_log, int log_stride)
{
    extern __shared__ float pcg_smem[];
    double *scratch = reinterpret_cast<double *>(pcg_smem);  // 3*NWARP + 3 doubles
    float *sp = pcg_smem + 2 * (3 * (PCG_THREADS / 32) + 4);
    const int tid = threadIdx.x;

    for (int b = blockIdx.x; b < bv.B; b += gridDim.x) {
        if (!bv.active(b)) continue;
        const int N = bv.N(b), kb = bv.off(b), n = NS * N;
        float *p = sp;        // [n] search direction
        float *rs = sp + n;   // [n] residual (for the block-diagonal preconditioner)
        const float *Sb = S + (size_t)S_STRIDE * kb;
        const float *Pb = Pinv + (size_t)pinv_stride * kb + pinv_off;
        const float *gb = gamma + (size_t)NS * kb;
        float *lb = lambda + (size_t)NS * kb;

        float lam[PCG_RPT], r[PCG_RPT], pv[PCG_RPT], z[PCG_RPT];

        // r = gamma - S lambda
        for (int i = tid; i < n; i += PCG_THREADS) p[i] = lb[i];
        __syncthreads();
        double acc3[3] = {0.0, 0.0, 0.0};  // gamma^T gamma, r^T z, r^T r
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < n) {
                const int k = i / NS, rr = i - NS * k;
                const float *row = Sb + (size_t)S_STRIDE * k + rr;
                float a = 0.f;
                if (k > 0) {
#pragma unroll
                    for (int cc = 0; cc < NS; ++cc) a = fmaf(row[NS * cc], p[NS * (k - 1) + cc], a);
                }
#pragma unroll
                for (int cc = 0; cc < NS; ++cc) a = fmaf(row[SS + NS * cc], p[NS * k + cc], a);
                if (k < N - 1) {
#pragma unroll
                    for (int cc = 0; cc < NS; ++cc) a = fmaf(row[2 * SS + NS * cc], p[NS * (k + 1) + cc], a);
                }
                const float gi = gb[i];
                lam[q] = lb[i];
                r[q] = gi - a;
                acc3[0] += (double)gi * gi;
            }
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < n) rs[i] = r[q];
        }
        __syncthreads();
        // z = Pinv r, p = z
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < n) {
                const int k = i / NS, rr = i - NS * k;
                const float *prow = Pb + (size_t)pinv_stride * k + rr;
                float a = 0.f;
#pragma unroll
                for (int cc = 0; cc < NS; ++cc) a = fmaf(prow[NS * cc], rs[NS * k + cc], a);
                z[q] = a;
                pv[q] = a;
                p[i] = a;
                acc3[1] += (double)r[q] * a;
                acc3[2] += (double)r[q] * r[q];
            }
        }
        block_sum<3>(acc3, scratch);
        const double gg = acc3[0];
        double eta = acc3[1], rr2 = acc3[2];
        auto converged = [&](double e, double r2) {
            return exit_mode == 0 ? (r2 <= (double)tol * (double)tol * gg) : (fabs(e) < (double)tol);
        };
        int it = 0;
        bool conv = converged(eta, rr2);
        bool bad = false;
        while (!conv && it < max_iter) {
            // v = S p
            double d1[1] = {0.0};
            float v[PCG_RPT];
#pragma unroll
            for (int q = 0; q < PCG_RPT; ++q) {
                const int i = tid + q * PCG_THREADS;
                v[q] = 0.f;
                if (i < n) {
                    const int k = i / NS, rr = i - NS * k;
                    const float *row = Sb + (size_t)S_STRIDE * k + rr;
                    float a = 0.f;
                    if (k > 0) {
#pragma unroll
                        for (int cc = 0; cc < NS; ++cc) a = fmaf(row[NS * cc], p[NS * (k - 1) + cc], a);
                    }
#pragma unroll
                    for (int cc = 0; cc < NS; ++cc) a = fmaf(row[SS + NS * cc], p[NS * k + cc], a);
                    if (k < N - 1) {
#pragma unroll
                        for (int cc = 0; cc < NS; ++cc) a = fmaf(row[2 * SS + NS * cc], p[NS * (k + 1) + cc], a);
                    }
                    v[q] = a;
                    d1[0] += (double)pv[q] * a;
                }
            }
            block_sum<1>(d1, scratch);
            const double alpha_d = eta / d1[0];
            if (!isfinite(alpha_d)) { bad = true; break; }
            const float alpha = (float)alpha_d;
#pragma unroll
            for (int q = 0; q < PCG_RPT; ++q) {
                const int i = tid + q * PCG_THREADS;
                if (i < n) {
                    lam[q] = fmaf(alpha, pv[q], lam[q]);
                    r[q] = fmaf(-alpha, v[q], r[q]);
                    rs[i] = r[q];
                }
            }
            __syncthreads();
            double d2[2] = {0.0, 0.0};
#pragma unroll
            for (int q = 0; q < PCG_RPT; ++q) {
                const int i = tid + q * PCG_THREADS;
                if (i < n) {
                    const int k = i / NS, rr = i - NS * k;
                    const float *prow = Pb + (size_t)pinv_stride * k + rr;
                    float a = 0.f;
#pragma unroll
                    for (int cc = 0; cc < NS; ++cc) a = fmaf(prow[NS * cc], rs[NS * k + cc], a);
                    z[q] = a;
                    d2[0] += (double)r[q] * a;
                    d2[1] += (double)r[q] * r[q];
                }
            }
            block_sum<2>(d2, scratch);
            ++it;
            if (!isfinite(d2[0])) { bad = true; break; }
            conv = converged(d2[0], d2[1]);
            if (conv) break;
            const float beta = (float)(d2[0] / eta);
            eta = d2[0];
#pragma unroll
            for (int q = 0; q < PCG_RPT; ++q) {
                const int i = tid + q * PCG_THREADS;
                if (i < n) {
                    pv[q] = fmaf(beta, pv[q], z[q]);
                    p[i] = pv[q];
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < n) lb[i] = lam[q];
        }
        if (tid == 0) {
            const uint32_t maxit = conv ? 0u : 1u;
            if (out_iters) {
                out_iters[2 * b] = (uint32_t)it;
                out_iters[2 * b + 1] = maxit | (bad ? 2u : 0u);
            }
            if (bv.st) {
                InstState &s = bv.st[b];
                s.last_pcg_iters = it;
                s.last_pcg_exit = maxit;
                s.pcg_iters_total += it;
                s.pcg_maxiter_count += maxit;
                if (bad) s.exit_flags |= 4u;
                if (pcg_log && s.sqp_iters < (uint32_t)log_stride)
                    pcg_log[(size_t)b * log_stride + s.sqp_iters] = (uint32_t)it | (maxit << 31);
            }
        }
        __syncthreads();
    }
}

size_t pcg_smem_bytes(int max_n_knots)
{
    return sizeof(double) * (3 * (PCG_THREADS / 32) + 4) + sizeof(float) * 2 * NS * (size_t)max_n_knots;
}

cudaError_t launch_pcg(const BatchView &bv, int max_n_knots, const float *S, const float *Pinv, int pinv_stride,
                       int pinv_off, const float *gamma, float *lambda, int max_iter, float tol, int exit_mode,
                       uint32_t *out_iters, uint32_t *pcg_log, int log_stride, int num_sms, cudaStream_t s)
{
    if (bv.B <= 0) return cudaSuccess;
    if (max_n_knots > MAX_PCG_KNOTS) return cudaErrorInvalidValue;
    const size_t smem = pcg_smem_bytes(max_n_knots);
    static size_t attr_set = 0;
    if (smem > 48 * 1024 && smem > attr_set) {
        cudaFuncSetAttribute(pcg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = smem;
    }
    int blocks = bv.B;
    const int cap = num_sms * 2;
    if (blocks > cap) blocks = cap;
    pcg_kernel<<<blocks, PCG_THREADS, smem, s>>>(bv, S, Pinv, pinv_stride, pinv_off, gamma, lambda, max_iter, tol,
                                                 exit_mode, out_iters, pcg_log, log_stride);
    return cudaGetLastError();
}

}  // namespace gpt
