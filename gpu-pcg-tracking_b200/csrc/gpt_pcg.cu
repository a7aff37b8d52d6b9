// gpt_pcg.cu -- preconditioned conjugate gradient on the block-tridiagonal
// Schur system, one thread-block cluster per instance, everything on chip.
//
// Replaces the GPU-PCG cooperative kernel the reference launches at
// toplevel.cuh:135-157,292-294 (pcg<T, STATE_SIZE, KNOT_POINTS>; its source
// is a git submodule absent from the reference tree).  Solves S lambda = gamma,
// warm-started from lambda, with the block-Jacobi preconditioner Pinv (the
// only Pinv blocks the reference fills, oldschur.cuh:926-933).
//
// Layout: an instance's N knots are split into CS contiguous chunks, one per
// CTA of a cluster (CS = 1..16).  Each CTA copies its chunk of the packed
// Schur matrix (per knot: left block 196, lower triangle of the diagonal
// block 105, lower triangle of the Pinv block 105, pad 2 = 408 floats) into
// shared memory once and iterates on it: no global traffic inside the loop.
// The right block of row k is the transpose of the left block of row k+1 (the
// reference stores exactly that, oldschur.cuh:945-958), so only left blocks
// are kept.  Neighbouring chunks exchange one knot of the search direction
// through distributed shared memory; the two dot products per iteration are
// reduced in FP64, in a fixed order, across the cluster with one cluster
// barrier each.  No grid-wide synchronisation: clusters never wait on each
// other.
//
// Precision: S, Pinv, the search direction p and z = Pinv r are FP32; the
// iterate lambda, the residual r, the products S p and every dot product are
// FP64.  Exit test: mode 0 ||r||_2 <= tol ||gamma||_2 on the true residual
// (recomputed with FP64 accumulation when the recursive residual passes; up
// to two residual-replacement restarts); mode 1 |r^T Pinv r| < tol.
#include <cooperative_groups.h>

#include "gpt_common.cuh"
#include "gpt_internal.h"

namespace cg = cooperative_groups;

namespace gpt {

constexpr int PK_LEFT = 0, PK_DIAG = SS, PK_PINV = SS + 105;
constexpr int PCG_THREADS = 512;
constexpr int PCG_NWARP = PCG_THREADS / 32;
constexpr int PCG_RPT = 4;  // rows per thread: 14 * PCG_KPC_MAX <= 512 * 4
constexpr int PCG_MAX_RESTARTS = 2;
constexpr int SLOT_CS = 16;

__device__ __forceinline__ int tri_idx(int r, int c)
{
    return r >= c ? ((r * (r + 1)) >> 1) + c : ((c * (c + 1)) >> 1) + r;
}

size_t pcg_cluster_smem_bytes(int kpc)
{
    return sizeof(float) * ((size_t)kpc * PK + SS + (size_t)NS * kpc + (size_t)NS * (kpc + 2) + 2 * NS + 2 * NS) +
           sizeof(double) * (2 * SLOT_CS * 4 + PCG_NWARP * 4) + 16;
}

template <int CS>
struct PcgCtx {
    float *Sp, *left_next, *rv, *pv, *zh_l, *zh_r, *lh_l, *lh_r;
    double *slots, *red;
};

// Fixed-order reduction of NV doubles over the cluster; every thread gets the totals.
template <int CS, int NV>
__device__ __forceinline__ void cluster_sum(double (&v)[NV], const PcgCtx<CS> &c, int set)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) c.red[warp * 4 + q] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
        double t[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            t[q] = (lane < PCG_NWARP) ? c.red[lane * 4 + q] : 0.0;
            t[q] = warp_sum(t[q]);
        }
        if constexpr (CS == 1) {
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < NV; ++q) c.slots[(set * SLOT_CS) * 4 + q] = t[q];
            }
        } else {
            cg::cluster_group cl = cg::this_cluster();
            const int me = (int)cl.block_rank();
            if (lane < CS) {
                double *dst = cl.map_shared_rank(c.slots, lane);
#pragma unroll
                for (int q = 0; q < NV; ++q) dst[(set * SLOT_CS + me) * 4 + q] = t[q];
            }
        }
    }
    if constexpr (CS == 1) {
        __syncthreads();
    } else {
        cg::this_cluster().sync();
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0.0;
#pragma unroll
        for (int src = 0; src < CS; ++src) s += c.slots[(set * SLOT_CS + src) * 4 + q];
        v[q] = s;
    }
}

// One row of S x with x in pv (halo knot at local index 0 and kpc+1); FP32 or FP64 accumulation.
template <typename ACC>
__device__ __forceinline__ ACC schur_row(const float *Sp, const float *left_next, const float *x, int kl, int r, int k,
                                         int N, int kpc)
{
    const float *blk = Sp + (size_t)kl * PK;
    ACC a = 0;
    if (k > 0) {
        const float *xp = x + kl * NS;
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) a += (ACC)blk[PK_LEFT + r + NS * cc] * (ACC)xp[cc];
    }
    {
        const float *xk = x + (kl + 1) * NS;
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) a += (ACC)blk[PK_DIAG + tri_idx(r, cc)] * (ACC)xk[cc];
    }
    if (k < N - 1) {
        const float *ln = (kl + 1 < kpc) ? blk + PK : left_next;
        const float *xn = x + (kl + 2) * NS;
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) a += (ACC)ln[PK_LEFT + cc + NS * r] * (ACC)xn[cc];
    }
    return a;
}

__device__ __forceinline__ float pinv_row(const float *Sp, const float *rv, int kl, int r)
{
    const float *blk = Sp + (size_t)kl * PK + PK_PINV;
    const float *x = rv + kl * NS;
    float a = 0.f;
#pragma unroll
    for (int cc = 0; cc < NS; ++cc) a = fmaf(blk[tri_idx(r, cc)], x[cc], a);
    return a;
}

// FMT 0: S, Pinv in the reference's 3-block layout (588 floats per knot, Pinv diag at +196)
// FMT 1: packed 408 floats per knot (written by the Schur kernel of the SQP loop)
template <int CS, int FMT>
__global__ void __launch_bounds__(PCG_THREADS, 1)
    pcg_cluster_kernel(BatchView bv, int kpc_max, const float *__restrict__ S, const float *__restrict__ Pinv,
                       const float *__restrict__ gamma, float *__restrict__ lambda, double *__restrict__ lambda64,
                       int max_iter, float tol, int exit_mode, uint32_t *__restrict__ out_iters,
                       uint32_t *__restrict__ pcg_log, int log_stride)
{
    extern __shared__ float4 pcg_dyn_smem[];
    float *base = reinterpret_cast<float *>(pcg_dyn_smem);
    PcgCtx<CS> c;
    c.Sp = base;
    c.left_next = c.Sp + (size_t)kpc_max * PK;
    c.rv = c.left_next + SS;
    c.pv = c.rv + NS * kpc_max;
    c.zh_l = c.pv + NS * (kpc_max + 2);
    c.zh_r = c.zh_l + NS;
    c.lh_l = c.zh_r + NS;
    c.lh_r = c.lh_l + NS;
    c.slots = reinterpret_cast<double *>(c.lh_r + NS + ((size_t)(c.lh_r + NS - base) & 1));
    c.red = c.slots + 2 * SLOT_CS * 4;

    const int tid = threadIdx.x;
    const int b = blockIdx.x / CS;
    int rank = 0;
    if constexpr (CS > 1) rank = (int)cg::this_cluster().block_rank();
    if (b >= bv.B || !bv.active(b)) return;  // uniform over the cluster
    const int N = bv.N(b), kb = bv.off(b);
    const int k0 = (rank * N) / CS, k1 = ((rank + 1) * N) / CS, kpc = k1 - k0, nloc = NS * kpc;

    // ---- stage the chunk of S / Pinv (packed) and left block of knot k1
    if (FMT == 1) {
        const float4 *src = reinterpret_cast<const float4 *>(S + (size_t)(kb + k0) * PK);
        float4 *dst = reinterpret_cast<float4 *>(c.Sp);
        for (int i = tid; i < kpc * (PK / 4); i += PCG_THREADS) dst[i] = src[i];
        for (int i = tid; i < SS; i += PCG_THREADS)
            c.left_next[i] = (k1 < N) ? S[(size_t)(kb + k1) * PK + i] : 0.f;
    } else {
        for (int e = tid; e < kpc * SS; e += PCG_THREADS) {
            const int kl = e / SS, w = e - SS * kl, r = w % NS, cc = w / NS;
            const size_t g = (size_t)S_STRIDE * (kb + k0 + kl);
            c.Sp[kl * PK + PK_LEFT + w] = S[g + w];
            if (r >= cc) {
                c.Sp[kl * PK + PK_DIAG + tri_idx(r, cc)] = S[g + SS + w];
                c.Sp[kl * PK + PK_PINV + tri_idx(r, cc)] = Pinv[g + SS + w];
            }
        }
        for (int i = tid; i < SS; i += PCG_THREADS)
            c.left_next[i] = (k1 < N) ? S[(size_t)S_STRIDE * (kb + k1) + i] : 0.f;
    }
    const float *gb = gamma + (size_t)NS * (kb + k0);
    float *lb = lambda + (size_t)NS * (kb + k0);
    // lambda (warm start) with halos from global memory
    for (int i = tid; i < nloc; i += PCG_THREADS) c.pv[NS + i] = lb[i];
    if (tid < NS) {
        c.pv[tid] = (k0 > 0) ? lambda[(size_t)NS * (kb + k0 - 1) + tid] : 0.f;
        c.pv[NS * (kpc + 1) + tid] = (k1 < N) ? lambda[(size_t)NS * (kb + k1) + tid] : 0.f;
    }
    __syncthreads();

    // lambda and the residual in FP64 (an FP32 lambda cannot represent a solution whose relative
    // residual is below ~eps32 ||S|| ||lambda|| / ||gamma||, which exceeds 1e-5 at N = 128); the
    // matrix, the preconditioned residual z and the search direction p stay FP32.
    double lam[PCG_RPT], rr_[PCG_RPT];
    float zz[PCG_RPT], pp[PCG_RPT], gv[PCG_RPT];
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < PCG_RPT; ++q) {
        const int i = tid + q * PCG_THREADS;
        lam[q] = rr_[q] = 0.0;
        zz[q] = pp[q] = gv[q] = 0.f;
        if (i < nloc) {
            const int kl = i / NS, r = i - NS * kl;
            gv[q] = gb[i];
            lam[q] = c.pv[NS + i];
            rr_[q] = (double)gv[q] - schur_row<double>(c.Sp, c.left_next, c.pv, kl, r, k0 + kl, N, kpc);
            acc[0] += (double)gv[q] * gv[q];
        }
    }
    int set = 1;
    double gg = 0.0, eta = 0.0, rr2 = 0.0;
    int restarts = 0;

    // r -> rv, z = Pinv r, p = z (+ halo exchange of z), eta/rr partials, cluster reduce
    auto restart_direction = [&](bool with_gg) {
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < nloc) c.rv[i] = (float)rr_[q];
        }
        __syncthreads();
        double a3[3] = {with_gg ? acc[0] : 0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < nloc) {
                const int kl = i / NS, r = i - NS * kl;
                zz[q] = pinv_row(c.Sp, c.rv, kl, r);
                pp[q] = zz[q];
                c.pv[NS + i] = pp[q];
                a3[1] += rr_[q] * (double)zz[q];
                a3[2] += rr_[q] * rr_[q];
                if constexpr (CS > 1) {
                    cg::cluster_group cl = cg::this_cluster();
                    if (kl == 0 && rank > 0) cl.map_shared_rank(c.zh_r, rank - 1)[r] = zz[q];
                    if (kl == kpc - 1 && rank < CS - 1) cl.map_shared_rank(c.zh_l, rank + 1)[r] = zz[q];
                }
            }
        }
        cluster_sum<CS, 3>(a3, c, set);
        set ^= 1;
        if (with_gg) gg = a3[0];
        eta = a3[1];
        rr2 = a3[2];
        // p halos = z halos (zero outside the horizon)
        if (tid < NS) {
            c.pv[tid] = (k0 > 0) ? c.zh_l[tid] : 0.f;
            c.pv[NS * (kpc + 1) + tid] = (k1 < N) ? c.zh_r[tid] : 0.f;
        }
        __syncthreads();
    };
    restart_direction(true);

    auto converged = [&](double e, double r2) {
        return exit_mode == 0 ? (r2 <= (double)tol * (double)tol * gg) : (fabs(e) < (double)tol);
    };
    int it = 0;
    bool conv = converged(eta, rr2), bad = false, checked = false;
    while (true) {
        if (conv && exit_mode == 0 && !checked) {
            // true residual gamma - S lambda, FP64 accumulation; lambda (FP64) enters as hi + lo floats
            double t1[1] = {0.0};
            double sl[PCG_RPT];
#pragma unroll
            for (int q = 0; q < PCG_RPT; ++q) sl[q] = 0.0;
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                __syncthreads();
#pragma unroll
                for (int q = 0; q < PCG_RPT; ++q) {
                    const int i = tid + q * PCG_THREADS;
                    if (i < nloc) {
                        const float hi = (float)lam[q];
                        c.pv[NS + i] = part == 0 ? hi : (float)(lam[q] - (double)hi);
                    }
                }
                if constexpr (CS > 1) {
                    cg::cluster_group cl = cg::this_cluster();
#pragma unroll
                    for (int q = 0; q < PCG_RPT; ++q) {
                        const int i = tid + q * PCG_THREADS;
                        if (i < nloc) {
                            const int kl = i / NS, r = i - NS * kl;
                            const float hi = (float)lam[q];
                            const float v = part == 0 ? hi : (float)(lam[q] - (double)hi);
                            if (kl == 0 && rank > 0) cl.map_shared_rank(c.lh_r, rank - 1)[r] = v;
                            if (kl == kpc - 1 && rank < CS - 1) cl.map_shared_rank(c.lh_l, rank + 1)[r] = v;
                        }
                    }
                    cl.sync();
                } else {
                    __syncthreads();
                }
                if (tid < NS) {
                    c.pv[tid] = (k0 > 0) ? (CS > 1 ? c.lh_l[tid] : 0.f) : 0.f;
                    c.pv[NS * (kpc + 1) + tid] = (k1 < N) ? (CS > 1 ? c.lh_r[tid] : 0.f) : 0.f;
                }
                __syncthreads();
#pragma unroll
                for (int q = 0; q < PCG_RPT; ++q) {
                    const int i = tid + q * PCG_THREADS;
                    if (i < nloc) {
                        const int kl = i / NS, r = i - NS * kl;
                        sl[q] += schur_row<double>(c.Sp, c.left_next, c.pv, kl, r, k0 + kl, N, kpc);
                    }
                }
                if constexpr (CS > 1) cg::this_cluster().sync();  // halos are rewritten by the next part
            }
#pragma unroll
            for (int q = 0; q < PCG_RPT; ++q) {
                const int i = tid + q * PCG_THREADS;
                if (i < nloc) {
                    const double tr = (double)gv[q] - sl[q];
                    rr_[q] = tr;
                    t1[0] += tr * tr;
                }
            }
            cluster_sum<CS, 1>(t1, c, set);
            set ^= 1;
            if (t1[0] <= (double)tol * (double)tol * gg) break;  // converged on the true residual
            if (restarts >= PCG_MAX_RESTARTS || it >= max_iter) {
                conv = false;
                break;
            }
            ++restarts;
            restart_direction(false);
            conv = converged(eta, rr2);
            checked = conv;  // a restart that is already below tol on the true residual stops next round
            if (conv) break;
            continue;
        }
        if (conv || it >= max_iter) break;
        // v = S p
        double d1[1] = {0.0};
        double vv[PCG_RPT];
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            vv[q] = 0.0;
            if (i < nloc) {
                const int kl = i / NS, r = i - NS * kl;
                vv[q] = schur_row<double>(c.Sp, c.left_next, c.pv, kl, r, k0 + kl, N, kpc);
                d1[0] += (double)pp[q] * vv[q];
            }
        }
        cluster_sum<CS, 1>(d1, c, set);
        set ^= 1;
        const double alpha_d = eta / d1[0];
        if (!isfinite(alpha_d)) {
            bad = true;
            conv = false;
            break;
        }
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < nloc) {
                lam[q] = fma(alpha_d, (double)pp[q], lam[q]);
                rr_[q] = fma(-alpha_d, vv[q], rr_[q]);
                c.rv[i] = (float)rr_[q];
            }
        }
        __syncthreads();
        double d2[2] = {0.0, 0.0};
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < nloc) {
                const int kl = i / NS, r = i - NS * kl;
                zz[q] = pinv_row(c.Sp, c.rv, kl, r);
                d2[0] += rr_[q] * (double)zz[q];
                d2[1] += rr_[q] * rr_[q];
                if constexpr (CS > 1) {
                    cg::cluster_group cl = cg::this_cluster();
                    if (kl == 0 && rank > 0) cl.map_shared_rank(c.zh_r, rank - 1)[r] = zz[q];
                    if (kl == kpc - 1 && rank < CS - 1) cl.map_shared_rank(c.zh_l, rank + 1)[r] = zz[q];
                }
            }
        }
        cluster_sum<CS, 2>(d2, c, set);
        set ^= 1;
        ++it;
        if (!isfinite(d2[0])) {
            bad = true;
            conv = false;
            break;
        }
        conv = converged(d2[0], d2[1]);
        checked = false;
        if (conv) continue;  // true-residual check at the top of the loop
        const float beta = (float)(d2[0] / eta);
        eta = d2[0];
#pragma unroll
        for (int q = 0; q < PCG_RPT; ++q) {
            const int i = tid + q * PCG_THREADS;
            if (i < nloc) {
                pp[q] = fmaf(beta, pp[q], zz[q]);
                c.pv[NS + i] = pp[q];
            }
        }
        if (tid < NS) {
            // halo p = z_halo + beta p_halo (the neighbour's own update, done locally)
            c.pv[tid] = (k0 > 0) ? fmaf(beta, c.pv[tid], c.zh_l[tid]) : 0.f;
            c.pv[NS * (kpc + 1) + tid] = (k1 < N) ? fmaf(beta, c.pv[NS * (kpc + 1) + tid], c.zh_r[tid]) : 0.f;
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < PCG_RPT; ++q) {
        const int i = tid + q * PCG_THREADS;
        if (i < nloc) {
            lb[i] = (float)lam[q];
            if (lambda64) lambda64[(size_t)NS * (kb + k0) + i] = lam[q];
        }
    }
    if (tid == 0 && rank == 0) {
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
    // no CTA may exit while a neighbour can still write into its shared memory
    if constexpr (CS > 1) cg::this_cluster().sync();
}

// ---------------------------------------------------------------------------

int pcg_pick_cluster(int maxN, int B, int num_sms, int requested)
{
    if (requested > 0) return requested;
    int cs = 1;
    while ((maxN + cs - 1) / cs > PCG_KPC_MAX) cs *= 2;
    // a lone instance (plain path) spreads over more SMs to cut per-iteration latency
    if (B == 1) {
        while (cs < 8 && (maxN + 2 * cs - 1) / (2 * cs) >= 16) cs *= 2;
    }
    (void)num_sms;
    return cs;
}

template <int CS, int FMT>
static cudaError_t launch_pcg_cs(const BatchView &bv, int kpc_max, const float *S, const float *Pinv,
                                 const float *gamma, float *lambda, double *lambda64, int max_iter, float tol,
                                 int exit_mode, uint32_t *out_iters, uint32_t *pcg_log, int log_stride, cudaStream_t s)
{
    auto kern = pcg_cluster_kernel<CS, FMT>;
    const size_t smem = pcg_cluster_smem_bytes(kpc_max);
    static size_t attr_smem = 0;
    if (smem > attr_smem) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        if (CS > 8) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
        }
        attr_smem = smem;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(bv.B * CS), 1, 1);
    cfg.blockDim = dim3(PCG_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, bv, kpc_max, S, Pinv, gamma, lambda, lambda64, max_iter, tol, exit_mode,
                              out_iters, pcg_log, log_stride);
}

cudaError_t launch_pcg(const BatchView &bv, int max_n_knots, int min_n_knots, int fmt, const float *S,
                       const float *Pinv, const float *gamma, float *lambda, double *lambda64, int max_iter,
                       float tol, int exit_mode, uint32_t *out_iters, uint32_t *pcg_log, int log_stride,
                       int cluster_size, int num_sms, cudaStream_t s)
{
    if (bv.B <= 0) return cudaSuccess;
    if (max_n_knots > MAX_PCG_KNOTS) return cudaErrorInvalidValue;
    int cs = pcg_pick_cluster(max_n_knots, bv.B, num_sms, cluster_size);
    while (cs > 1 && cs > min_n_knots) cs /= 2;  // every CTA owns at least one knot
    const int kpc_max = (max_n_knots + cs - 1) / cs;
    if (kpc_max > PCG_KPC_MAX) return cudaErrorInvalidValue;
#define GPT_PCG_CASE(CSV)                                                                                      \
    case CSV:                                                                                                  \
        return fmt ? launch_pcg_cs<CSV, 1>(bv, kpc_max, S, Pinv, gamma, lambda, lambda64, max_iter, tol,       \
                                           exit_mode, out_iters, pcg_log, log_stride, s)                       \
                   : launch_pcg_cs<CSV, 0>(bv, kpc_max, S, Pinv, gamma, lambda, lambda64, max_iter, tol,       \
                                           exit_mode, out_iters, pcg_log, log_stride, s);
    switch (cs) {
        GPT_PCG_CASE(1)
        GPT_PCG_CASE(2)
        GPT_PCG_CASE(4)
        GPT_PCG_CASE(8)
        GPT_PCG_CASE(16)
    default:
        return cudaErrorInvalidValue;
    }
#undef GPT_PCG_CASE
}

}  // namespace gpt
