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
// Schur matrix (per knot: left block 196 column-major, lower triangle of the
// diagonal block 105, lower triangle of the Pinv block 105, pad 2 = 408
// floats) into shared memory once and iterates on it: no global traffic
// inside the loop.  The right block of row k is the transpose of the left
// block of row k+1 (the reference stores exactly that, oldschur.cuh:945-958),
// so only left blocks are kept.  Thread (r, g) owns row r of knots g, g+TK,
// g+2TK, g+3TK, so its triangle offsets are computed once and its rows give
// independent accumulation chains.  Neighbouring chunks exchange one knot of
// the search direction through distributed shared memory; the dot products
// are reduced in FP64, in a fixed order, across the cluster with one cluster
// barrier per reduction.  Clusters never wait on each other.
//
// Precision: S, Pinv, the search direction p, z = Pinv r and the product S p
// are FP32; the iterate lambda, the residual r and every dot product are
// FP64.  Every RR_PERIOD iterations, and whenever the recursive residual
// passes the exit test, r is replaced by the true residual gamma - S lambda
// evaluated with FP64 accumulation (lambda split into two floats), so the
// exit test always holds for the true residual.
// Exit test: mode 0 ||r||_2 <= tol ||gamma||_2; mode 1 |r^T Pinv r| < tol.
#include <cooperative_groups.h>
#include <type_traits>

#include "gpt_common.cuh"
#include "gpt_internal.h"
#include "gpt_layout.h"

namespace cg = cooperative_groups;

namespace gpt {

constexpr int PK_LEFT = 0, PK_DIAG = SS, PK_PINV = SS + 105;
constexpr int PCG_TK = 36;                       // knot groups per CTA
constexpr int PCG_THREADS = 512;                 // 14 * 36 = 504 workers
constexpr int PCG_WORKERS = NS * PCG_TK;
constexpr int PCG_NWARP = PCG_THREADS / 32;
constexpr int PCG_KPT = (PCG_KPC_MAX + PCG_TK - 1) / PCG_TK;  // knots per thread (4)
constexpr int RR_PERIOD = 32;
constexpr int SLOT_CS = 16;

// stair: the stair preconditioner's left blocks of Pinv, per knot of the chunk and for the next
// chunk's first knot ((kpc + 1) x 196 floats)
size_t pcg_cluster_smem_bytes(int kpc, bool stair)
{
    return sizeof(float) * ((size_t)kpc * PK + SS + 2 * (size_t)NS * (kpc + 2) + 2 * NS) +
           sizeof(double) * (2 * SLOT_CS * 4 + PCG_NWARP * 4) + 16 +
           (stair ? sizeof(float) * (size_t)(kpc + 1) * SS : 0);
}
size_t pcg_cluster_smem_bytes(int kpc) { return pcg_cluster_smem_bytes(kpc, false); }

struct PcgCtx {
    float *Sp, *left_next, *rv, *pv, *zh_l, *zh_r;
    double *slots, *red;
    float *Pl;  // stair preconditioner: Pinv left blocks (kpc_max + 1 blocks; the last one is the next chunk's)
};

// Fixed-order reduction of NV doubles over the cluster; every thread gets the totals.
template <int CS, int NV>
__device__ __forceinline__ void cluster_sum_raw(double (&v)[NV], double *slots, double *red, int set)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) red[warp * 4 + q] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
        double t[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            t[q] = (lane < PCG_NWARP) ? red[lane * 4 + q] : 0.0;
            t[q] = warp_sum(t[q]);
        }
        if constexpr (CS == 1) {
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < NV; ++q) slots[(set * SLOT_CS) * 4 + q] = t[q];
            }
        } else {
            cg::cluster_group cl = cg::this_cluster();
            const int me = (int)cl.block_rank();
            if (lane < CS) {
                double *dst = cl.map_shared_rank(slots, lane);
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
        for (int src = 0; src < CS; ++src) s += slots[(set * SLOT_CS + src) * 4 + q];
        v[q] = s;
    }
}

template <int CS, int NV>
__device__ __forceinline__ void cluster_sum(double (&v)[NV], const PcgCtx &c, int set)
{
    cluster_sum_raw<CS, NV>(v, c.slots, c.red, set);
}

// Triangle offsets of row r: element (r, c) of a packed lower triangle.
struct RowOffsets {
    int o[NS];
    __device__ __forceinline__ explicit RowOffsets(int r)
    {
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) o[cc] = (cc <= r) ? ((r * (r + 1)) >> 1) + cc : ((cc * (cc + 1)) >> 1) + r;
    }
};

__device__ __forceinline__ float2 lds2(const float *p) { return *reinterpret_cast<const float2 *>(p); }

// Row r of (S x)_k, FP32; x points at knot k-1's block of a halo-padded vector.
__device__ __forceinline__ float schur_row_f32(const float *blk, const float *ln, const float *x, const RowOffsets &ro,
                                               int r, bool has_left, bool has_right)
{
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    if (has_left) {
#pragma unroll
        for (int m = 0; m < NS / 2; ++m) {
            const float2 xv = lds2(x + 2 * m);
            a0 = fmaf(blk[PK_LEFT + r + NS * (2 * m)], xv.x, a0);
            a0 = fmaf(blk[PK_LEFT + r + NS * (2 * m + 1)], xv.y, a0);
        }
    }
#pragma unroll
    for (int m = 0; m < NS / 2; ++m) {
        const float2 xv = lds2(x + NS + 2 * m);
        a1 = fmaf(blk[PK_DIAG + ro.o[2 * m]], xv.x, a1);
        a1 = fmaf(blk[PK_DIAG + ro.o[2 * m + 1]], xv.y, a1);
    }
    if (has_right) {
#pragma unroll
        for (int m = 0; m < NS / 2; ++m) {
            const float2 xv = lds2(x + 2 * NS + 2 * m);
            const float2 lv = lds2(ln + PK_LEFT + NS * r + 2 * m);
            a2 = fmaf(lv.x, xv.x, a2);
            a2 = fmaf(lv.y, xv.y, a2);
        }
    }
    return (a0 + a1) + a2;
}

// Same row with FP64 accumulation (used for the true residual).
__device__ __forceinline__ double schur_row_f64(const float *blk, const float *ln, const float *x, const RowOffsets &ro,
                                                int r, bool has_left, bool has_right)
{
    double a = 0.0;
    if (has_left) {
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) a = fma((double)blk[PK_LEFT + r + NS * cc], (double)x[cc], a);
    }
#pragma unroll
    for (int cc = 0; cc < NS; ++cc) a = fma((double)blk[PK_DIAG + ro.o[cc]], (double)x[NS + cc], a);
    if (has_right) {
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) a = fma((double)ln[PK_LEFT + NS * r + cc], (double)x[2 * NS + cc], a);
    }
    return a;
}

__device__ __forceinline__ float pinv_row(const float *blk, const float *x, const RowOffsets &ro)
{
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int m = 0; m < NS / 2; ++m) {
        const float2 xv = lds2(x + 2 * m);
        a0 = fmaf(blk[PK_PINV + ro.o[2 * m]], xv.x, a0);
        a1 = fmaf(blk[PK_PINV + ro.o[2 * m + 1]], xv.y, a1);
    }
    return a0 + a1;
}

// FMT 0: S, Pinv in the reference's 3-block layout (588 floats per knot, Pinv diag at +196)
// FMT 1: packed 408 floats per knot (written by the Schur kernel of the SQP loop)
// PRE 0: block-Jacobi (Pinv's diagonal blocks); PRE 2: the stair preconditioner of gato_form_ss
// (oldschur.cuh:334-494; FMT 0 only), z_k = Pinv[k].left r_{k-1} + Pinv[k].diag r_k + Pinv[k].right r_{k+1}
// with Pinv[k].right = Pinv[k+1].left^T (both are -theta^{-1} L theta^{-1} products of the symmetric
// theta^{-1}), so only the left blocks are staged; the residual's neighbouring knots come through
// the halo slots of the residual copy, exchanged through distributed shared memory like p's.
template <int CS, int FMT, int PRE>
__global__ void __launch_bounds__(PCG_THREADS, 1)
    pcg_cluster_kernel(BatchView bv, int kpc_max, const float *__restrict__ S, const float *__restrict__ Pinv,
                       const float *__restrict__ gamma, float *__restrict__ lambda, double *__restrict__ lambda64,
                       int max_iter, float tol, int exit_mode, uint32_t *__restrict__ out_iters,
                       uint32_t *__restrict__ pcg_log, int log_stride)
{
    extern __shared__ float4 pcg_dyn_smem[];
    float *base = reinterpret_cast<float *>(pcg_dyn_smem);
    PcgCtx c;
    c.Sp = base;
    c.left_next = c.Sp + (size_t)kpc_max * PK;
    c.rv = c.left_next + SS;           // (kpc+2) x 14: residual copy / lambda parts, halo slots at both ends
    c.pv = c.rv + NS * (kpc_max + 2);  // (kpc+2) x 14: search direction with halos
    c.zh_l = c.pv + NS * (kpc_max + 2);
    c.zh_r = c.zh_l + NS;
    {
        const size_t used = (size_t)(c.zh_r + NS - base);
        c.slots = reinterpret_cast<double *>(base + used + (used & 1));
    }
    c.red = c.slots + 2 * SLOT_CS * 4;
    c.Pl = reinterpret_cast<float *>(c.red + PCG_NWARP * 4);
    static_assert(PRE == 0 || FMT == 0, "the stair preconditioner reads the reference's 3-block Pinv");

    const int tid = threadIdx.x;
    const int b = bv.b0 + (int)blockIdx.x / CS;
    int rank = 0;
    if constexpr (CS > 1) rank = (int)cg::this_cluster().block_rank();
    if (b >= bv.b0 + bv.B || !bv.active(b)) return;  // uniform over the cluster
    const int N = bv.N(b), kb = bv.off(b);
    const int k0 = (rank * N) / CS, k1 = ((rank + 1) * N) / CS, kpc = k1 - k0;
    // chunk size of the left neighbour (its right halo slot is kpc_left + 1)
    const int kpc_left = (rank > 0) ? k0 - ((rank - 1) * N) / CS : 0;

    // ---- stage the chunk of S / Pinv (packed) and the left block of knot k1
    if (FMT == 1) {
        const float4 *src = reinterpret_cast<const float4 *>(S + (size_t)(kb + k0) * PK);
        float4 *dst = reinterpret_cast<float4 *>(c.Sp);
        for (int i = tid; i < kpc * (PK / 4); i += PCG_THREADS) dst[i] = src[i];
        for (int i = tid; i < SS; i += PCG_THREADS) c.left_next[i] = (k1 < N) ? S[(size_t)(kb + k1) * PK + i] : 0.f;
    } else {
        for (int e = tid; e < kpc * SS; e += PCG_THREADS) {
            const int kl = e / SS, w = e - SS * kl, r = w % NS, cc = w / NS;
            const size_t g = (size_t)S_STRIDE * (kb + k0 + kl);
            c.Sp[kl * PK + PK_LEFT + w] = S[g + w];
            if (r >= cc) {
                const int t = ((r * (r + 1)) >> 1) + cc;
                c.Sp[kl * PK + PK_DIAG + t] = S[g + SS + w];
                c.Sp[kl * PK + PK_PINV + t] = Pinv[g + SS + w];
            }
            if (PRE == 2) c.Pl[kl * SS + w] = Pinv[g + w];
        }
        for (int i = tid; i < SS; i += PCG_THREADS) {
            c.left_next[i] = (k1 < N) ? S[(size_t)S_STRIDE * (kb + k1) + i] : 0.f;
            if (PRE == 2) c.Pl[kpc_max * SS + i] = (k1 < N) ? Pinv[(size_t)S_STRIDE * (kb + k1) + i] : 0.f;
        }
    }
    const float *gb = gamma + (size_t)NS * (kb + k0);
    float *lb = lambda + (size_t)NS * (kb + k0);
    // warm start (FP32) with halos from global memory into rv
    for (int i = tid; i < NS * kpc; i += PCG_THREADS) c.rv[NS + i] = lb[i];
    if (tid < NS) {
        c.rv[tid] = (k0 > 0) ? lambda[(size_t)NS * (kb + k0 - 1) + tid] : 0.f;
        c.rv[NS * (kpc + 1) + tid] = (k1 < N) ? lambda[(size_t)NS * (kb + k1) + tid] : 0.f;
    }
    __syncthreads();

    // ---- per-thread rows: row r of local knots g0 + PCG_TK * j
    const bool worker = tid < PCG_WORKERS;
    const int r = worker ? tid % NS : 0, g0 = worker ? tid / NS : 0;
    const RowOffsets ro(r);
    double lam[PCG_KPT], res[PCG_KPT];
    float pp[PCG_KPT], zz[PCG_KPT], gv[PCG_KPT];
    bool own[PCG_KPT];
#pragma unroll
    for (int j = 0; j < PCG_KPT; ++j) {
        const int kl = g0 + PCG_TK * j;
        own[j] = worker && kl < kpc;
        lam[j] = res[j] = 0.0;
        pp[j] = zz[j] = gv[j] = 0.f;
        if (own[j]) {
            gv[j] = gb[NS * kl + r];
            lam[j] = (double)c.rv[NS * (kl + 1) + r];
        }
    }
    auto row_f64 = [&](int j, const float *x) -> double {
        const int kl = g0 + PCG_TK * j, k = k0 + kl;
        const float *blk = c.Sp + (size_t)kl * PK;
        const float *ln = (kl + 1 < kpc) ? blk + PK : c.left_next;
        return schur_row_f64(blk, ln, x + NS * kl, ro, r, k > 0, k < N - 1);
    };
    // initial residual gamma - S lambda (lambda is FP32 here: one FP64 pass is exact to rounding)
    double acc3[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < PCG_KPT; ++j) {
        if (own[j]) {
            res[j] = (double)gv[j] - row_f64(j, c.rv);
            acc3[0] += (double)gv[j] * gv[j];
        }
    }
    int set = 1;

    // true residual r = gamma - S lambda with lambda (FP64) split into hi + lo floats
    auto replace_residual = [&]() {
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) res[j] = own[j] ? (double)gv[j] : 0.0;
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            __syncthreads();
#pragma unroll
            for (int j = 0; j < PCG_KPT; ++j) {
                if (own[j]) {
                    const int kl = g0 + PCG_TK * j;
                    const float hi = (float)lam[j];
                    const float v = part == 0 ? hi : (float)(lam[j] - (double)hi);
                    c.rv[NS * (kl + 1) + r] = v;
                    if constexpr (CS > 1) {
                        // neighbours keep this CTA's boundary knots in their halo slots
                        cg::cluster_group cl = cg::this_cluster();
                        if (kl == 0 && rank > 0) cl.map_shared_rank(c.rv, rank - 1)[NS * (kpc_left + 1) + r] = v;
                        if (kl == kpc - 1 && rank < CS - 1) cl.map_shared_rank(c.rv, rank + 1)[r] = v;
                    }
                }
            }
            if constexpr (CS > 1) {
                cg::this_cluster().sync();
            } else {
                __syncthreads();
            }
#pragma unroll
            for (int j = 0; j < PCG_KPT; ++j)
                if (own[j]) res[j] -= row_f64(j, c.rv);
            if constexpr (CS > 1) cg::this_cluster().sync();  // halos are rewritten by the next part
        }
    };

    // z = Pinv r from the FP32 copy of r; halo exchange of z; partial dot products
    auto precond = [&](double (&d)[3]) {
        // with the stair preconditioner the neighbours' halo slots of rv are written below: every CTA
        // of the cluster must be done reading its rv (the initial residual reads the warm start's halos)
        if constexpr (PRE == 2 && CS > 1) {
            cg::this_cluster().sync();
        } else {
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j)
            if (own[j]) c.rv[NS * (g0 + PCG_TK * j + 1) + r] = (float)res[j];
        if constexpr (PRE == 2) {
            // the neighbouring chunks' boundary residuals into the halo slots (zero at the horizon's ends)
            if (tid < NS) {
                if (k0 == 0) c.rv[tid] = 0.f;
                if (k1 == N) c.rv[NS * (kpc + 1) + tid] = 0.f;
            }
            if constexpr (CS > 1) {
                cg::cluster_group cl = cg::this_cluster();
#pragma unroll
                for (int j = 0; j < PCG_KPT; ++j) {
                    if (own[j]) {
                        const int kl = g0 + PCG_TK * j;
                        if (kl == 0 && rank > 0) cl.map_shared_rank(c.rv, rank - 1)[NS * (kpc_left + 1) + r] = (float)res[j];
                        if (kl == kpc - 1 && rank < CS - 1) cl.map_shared_rank(c.rv, rank + 1)[r] = (float)res[j];
                    }
                }
                cl.sync();
            } else {
                __syncthreads();
            }
        } else {
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            if (own[j]) {
                const int kl = g0 + PCG_TK * j;
                zz[j] = pinv_row(c.Sp + (size_t)kl * PK, c.rv + NS * (kl + 1), ro);
                if constexpr (PRE == 2) {
                    const int k = k0 + kl;
                    const float *pl = c.Pl + (size_t)kl * SS;                                  // Pinv[k].left
                    const float *pn = c.Pl + (size_t)(kl + 1 < kpc ? kl + 1 : kpc_max) * SS;  // Pinv[k+1].left
                    float a0 = 0.f, a1 = 0.f;
#pragma unroll
                    for (int t = 0; t < NS; ++t) {
                        if (k > 0) a0 = fmaf(pl[r + NS * t], c.rv[NS * kl + t], a0);
                        if (k < N - 1) a1 = fmaf(pn[t + NS * r], c.rv[NS * (kl + 2) + t], a1);
                    }
                    zz[j] += a0 + a1;
                }
                d[1] += res[j] * (double)zz[j];
                d[2] += res[j] * res[j];
                if constexpr (CS > 1) {
                    cg::cluster_group cl = cg::this_cluster();
                    if (kl == 0 && rank > 0) cl.map_shared_rank(c.zh_r, rank - 1)[r] = zz[j];
                    if (kl == kpc - 1 && rank < CS - 1) cl.map_shared_rank(c.zh_l, rank + 1)[r] = zz[j];
                }
            }
        }
    };

    // ---- p = z
    double eta, rr2, gg;
    {
        precond(acc3);
        cluster_sum<CS, 3>(acc3, c, set);
        set ^= 1;
        gg = acc3[0];
        eta = acc3[1];
        rr2 = acc3[2];
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            pp[j] = zz[j];
            if (own[j]) c.pv[NS * (g0 + PCG_TK * j + 1) + r] = pp[j];
        }
        if (tid < NS) {
            c.pv[tid] = (k0 > 0) ? c.zh_l[tid] : 0.f;
            c.pv[NS * (kpc + 1) + tid] = (k1 < N) ? c.zh_r[tid] : 0.f;
        }
        __syncthreads();
    }
    auto converged = [&](double e, double r2) {
        return exit_mode == 0 ? (r2 <= (double)tol * (double)tol * gg) : (fabs(e) < (double)tol);
    };
    bool conv = converged(eta, rr2), bad = false;
    int it = 0;
    while (!conv && it < max_iter) {
        // v = S p (FP32), pAp (FP64)
        double d1[1] = {0.0};
        float vv[PCG_KPT];
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            vv[j] = 0.f;
            if (own[j]) {
                const int kl = g0 + PCG_TK * j, k = k0 + kl;
                const float *blk = c.Sp + (size_t)kl * PK;
                const float *ln = (kl + 1 < kpc) ? blk + PK : c.left_next;
                vv[j] = schur_row_f32(blk, ln, c.pv + NS * kl, ro, r, k > 0, k < N - 1);
                d1[0] += (double)pp[j] * (double)vv[j];
            }
        }
        cluster_sum<CS, 1>(d1, c, set);
        set ^= 1;
        const double alpha = eta / d1[0];
        if (!isfinite(alpha)) {
            bad = true;
            break;
        }
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            lam[j] = fma(alpha, (double)pp[j], lam[j]);
            res[j] = fma(-alpha, (double)vv[j], res[j]);
        }
        ++it;
        bool replaced = false;
        if (it % RR_PERIOD == 0) {
            replace_residual();
            replaced = true;
        }
        double d2[3] = {0.0, 0.0, 0.0};
        precond(d2);
        cluster_sum<CS, 3>(d2, c, set);
        set ^= 1;
        conv = converged(d2[1], d2[2]);
        if (conv && exit_mode == 0 && !replaced) {
            // confirm on the true residual
            replace_residual();
            double d3[3] = {0.0, 0.0, 0.0};
            precond(d3);
            cluster_sum<CS, 3>(d3, c, set);
            set ^= 1;
            d2[1] = d3[1];
            d2[2] = d3[2];
            conv = converged(d2[1], d2[2]);
        }
        if (!isfinite(d2[1])) {
            bad = true;
            conv = false;
            break;
        }
        if (conv) break;
        const float beta = (float)(d2[1] / eta);
        eta = d2[1];
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            pp[j] = fmaf(beta, pp[j], zz[j]);
            if (own[j]) c.pv[NS * (g0 + PCG_TK * j + 1) + r] = pp[j];
        }
        if (tid < NS) {
            // halo p = z_halo + beta p_halo (the neighbour's own update, done locally)
            c.pv[tid] = (k0 > 0) ? fmaf(beta, c.pv[tid], c.zh_l[tid]) : 0.f;
            c.pv[NS * (kpc + 1) + tid] = (k1 < N) ? fmaf(beta, c.pv[NS * (kpc + 1) + tid], c.zh_r[tid]) : 0.f;
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < PCG_KPT; ++j) {
        if (own[j]) {
            const int i = NS * (g0 + PCG_TK * j) + r;
            lb[i] = (float)lam[j];
            if (lambda64) lambda64[(size_t)NS * (kb + k0) + i] = lam[j];
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
// PCG with the chunk block-tridiagonal preconditioner (block cyclic reduction)
// ---------------------------------------------------------------------------
//
// M = -S is symmetric positive definite and block tridiagonal: diagonal
// blocks A_k = -S_kk, couplings M_{k,k-1} = -L_k with L_k = left_k.  The
// preconditioner solves each CTA's chunk of K knots exactly, M_chunk x = y,
// z = S_chunk^{-1} r = -x, by block cyclic reduction (odd-even elimination):
// at level l (h = 2^l) the knots j = h, 3h, 5h, ... are eliminated from the
// system on the multiples of h, which leaves a block-tridiagonal system on the
// multiples of 2h with
//   A_{j-h} -= L_j^T A_j^{-1} L_j,   A_{j+h} -= L_{j+h} A_j^{-1} L_{j+h}^T,
//   L'_{j+h} = L_{j+h} A_j^{-1} L_j   (coupling of j+h to j-h at level l+1),
// until knot 0 is left.  It is Gaussian elimination of an SPD matrix in the
// odd-even order, so every pivot block is SPD and no pivoting is needed; its
// depth is log2 K levels instead of the K steps of a sequential LDL^T, and
// every level's eliminations run in parallel (one warp each).  The factors
// are FP64: A_j^{-1} in shared memory (packed lower triangle), the level >= 1
// couplings in a global workspace (L2-resident, K blocks per chunk).  The
// solve runs the same levels: forward t_j = A_j^{-1} y_j, y_{j-h} += L_j^T t_j,
// y_{j+h} += L_{j+h} t_j; then x_0 = A_0^{-1} y_0 and backward
// x_j = t_j + A_j^{-1} (L_j x_{j-h} + L_{j+h}^T x_{j+h}).  With one CTA per
// instance the preconditioner is the inverse of S up to rounding and the PCG
// stops after one or two iterations; with several CTAs the chunks are coupled
// through the iterations.  S (left and diagonal blocks) is read from global
// memory (L2).

constexpr int CH_SLOTS = 2 * SLOT_CS * 4;
constexpr int CR_WARP_SCRATCH = 2 * SS;  // two couplings per warp during the factorisation

// union region: per-warp coupling scratch during the factorisation; then the
// halo-padded vector rv (14 (K+2)), t (14 K) and s (14 K) of the solve
__host__ __device__ constexpr int cr_union_doubles(int kpc)
{
    return PCG_NWARP * CR_WARP_SCRATCH > NS * (3 * kpc + 2) ? PCG_NWARP * CR_WARP_SCRATCH : NS * (3 * kpc + 2);
}
__host__ __device__ constexpr int chain_double_words(int kpc)
{
    return kpc * 105 + cr_union_doubles(kpc) + CH_SLOTS + PCG_NWARP * 4;
}

size_t pcg_chain_smem_bytes(int kpc) { return sizeof(double) * (size_t)chain_double_words(kpc); }

__device__ __forceinline__ int tri_lo(int r, int c)  // packed lower-triangle index of (r, c), any order
{
    return r >= c ? ((r * (r + 1)) >> 1) + c : ((c * (c + 1)) >> 1) + r;
}

// element (r, c) of knot kg's diagonal Schur block (lower triangle used: exactly symmetric)
template <int FMT>
__device__ __forceinline__ int diag_off(int r, int c)
{
    const int hi = r >= c ? r : c, lo = r >= c ? c : r;
    if (FMT >= 1) return PK_DIAG + ((hi * (hi + 1)) >> 1) + lo;  // packed rows, FP32 (1) or FP64 (2)
    return SS + hi + NS * lo;
}

// In-place inverse of an SPD 14x14 block held as a packed lower triangle
// (FP64), by one warp: Gauss-Jordan on [A | I], lanes 0..13 holding A's
// columns and lanes 14..27 the identity's.  Not inlined: its unrolled body is
// large, and one shared copy stays in the instruction cache across the
// factorisation's calls (single-warp calls late in the factorisation otherwise
// run from cold instruction fetches).
__device__ __noinline__ void warp_spd_inverse_packed(double *Ap, int lane)
{
    double col[NS];
    const bool lft = lane < NS, rgt = lane >= NS && lane < 2 * NS;
#pragma unroll
    for (int r = 0; r < NS; ++r) col[r] = lft ? Ap[tri_lo(r, lane)] : ((rgt && r == lane - NS) ? 1.0 : 0.0);
    __syncwarp();
    // pivot p: the pivot element first, then each row's element of the pivot column is
    // broadcast just before it is used, so only the 14 column entries stay live
#pragma unroll
    for (int p = 0; p < NS; ++p) {
        const double piv = __shfl_sync(0xffffffffu, col[p], p);
        const double prow = col[p] * __drcp_rn(piv);  // correctly rounded reciprocal: ~3x less latency than a divide
#pragma unroll
        for (int r = 0; r < NS; ++r) {
            if (r == p) continue;
            const double pr = __shfl_sync(0xffffffffu, col[r], p);
            col[r] = fma(-pr, prow, col[r]);
        }
        col[p] = prow;
    }
    if (rgt) {
        const int cc = lane - NS;
#pragma unroll
        for (int r = 0; r < NS; ++r)
            if (r >= cc) Ap[((r * (r + 1)) >> 1) + cc] = col[r];
    }
    __syncwarp();
}

// Precision: with an exact preconditioner the search direction must not be
// rounded to FP32 -- the rounding error of p is amplified by cond(S) (up to
// ~4e7 here) -- so p, z, S p, lambda and r are all FP64; S stays FP32 (its
// products are exact in FP64).
template <int CS, int FMT>
__global__ void __launch_bounds__(PCG_THREADS, 1)
    pcg_chain_kernel(BatchView bv, int kpc_max, const void *__restrict__ Sv, const float *__restrict__ gamma,
                     const double *__restrict__ gamma64, float *__restrict__ lambda, double *__restrict__ lambda64,
                     double *__restrict__ cr_ws, int max_iter, float tol, int exit_mode,
                     uint32_t *__restrict__ out_iters, uint32_t *__restrict__ pcg_log, int log_stride)
{
    // FMT 2: packed FP64 rows (PK64 doubles per knot) and FP64 gamma, from schur64_kernel
    using ST = typename std::conditional<FMT == 2, double, float>::type;
    const ST *S = reinterpret_cast<const ST *>(Sv);
    extern __shared__ double chain_dyn_smem[];
    double *Aq = chain_dyn_smem;                    // kpc_max x 105: A_k, then A_k^{-1}
    double *un = Aq + (size_t)kpc_max * 105;         // union region
    double *rv = un;                                 // 14 (kpc_max+2): p / r / lambda / the solve's y, x
    double *tv = rv + NS * (kpc_max + 2);            // 14 kpc_max: t_j
    double *sv = tv + NS * kpc_max;                  // 14 kpc_max: s_j
    double *slots = un + cr_union_doubles(kpc_max);
    double *red = slots + CH_SLOTS;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = bv.b0 + (int)blockIdx.x / CS;
    int rank = 0;
    if constexpr (CS > 1) rank = (int)cg::this_cluster().block_rank();
    if (b >= bv.b0 + bv.B || !bv.active(b)) return;  // uniform over the cluster
    const int N = bv.N(b), kb = bv.off(b);
    const int k0 = (rank * N) / CS, k1 = ((rank + 1) * N) / CS, kpc = k1 - k0;
    const int kpc_left = (rank > 0) ? k0 - ((rank - 1) * N) / CS : 0;
    const size_t kg0 = (size_t)kb + k0;
    const size_t kstride = FMT == 2 ? PK64 : (FMT == 1 ? PK : S_STRIDE);
    int nlev = 0;
    while ((1 << nlev) < kpc) ++nlev;

    // level-l coupling of local knot k (a multiple of 2^l, k >= 2^l) to k - 2^l, column-major:
    // level 0 is the left block of S, levels >= 1 live in the workspace
    auto lev_block = [&](int l, int k) -> double * {
        int o = 0;
        for (int q = 1; q < l; ++q) o += (kpc - 1) >> q;
        return cr_ws + (kg0 + (size_t)o + (size_t)((k >> l) - 1)) * SS;
    };
    // row rr (col_major = false: elements (rr, cc)) or column rr (true: (cc, rr)) of a level-l
    // coupling, all 14 loads issued before use
    auto coupling_line = [&](int l, int k, int rr, bool column, double (&v)[NS]) {
        if (l == 0) {
            const ST *src = S + (kg0 + k) * kstride;
            ST f[NS];
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) f[cc] = __ldg(src + (column ? cc + NS * rr : rr + NS * cc));
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) v[cc] = (double)f[cc];
        } else {
            const double *src = lev_block(l, k);
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) v[cc] = src[column ? cc + NS * rr : rr + NS * cc];
        }
    };

    // ---- A_k = -S_kk (FP64, packed lower triangle); loads issued in groups of 8 before the stores
    {
        constexpr int G = 8;
        for (int i0 = tid; i0 < kpc * 105; i0 += G * PCG_THREADS) {
            ST v[G];
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int i = i0 + q * PCG_THREADS;
                v[q] = 0.f;
                if (i < kpc * 105) {
                    const int kl = i / 105, t = i - kl * 105;
                    if (FMT >= 1) {
                        v[q] = __ldg(S + (kg0 + kl) * kstride + PK_DIAG + t);  // same packed order
                    } else {
                        int rr = 0;
                        while (((rr + 1) * (rr + 2)) / 2 <= t) ++rr;
                        const int cc = t - (rr * (rr + 1)) / 2;
                        v[q] = __ldg(S + (kg0 + kl) * kstride + diag_off<FMT>(rr, cc));
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int i = i0 + q * PCG_THREADS;
                if (i < kpc * 105) Aq[i] = -(double)v[q];
            }
        }
    }
    __syncthreads();

    // ---- factorisation by levels; warp w eliminates knots j = h (2m+1), m = w, w+16, ...
    {
        double *Lw0 = un + (size_t)warp * CR_WARP_SCRATCH, *Lw1 = Lw0 + SS;
        const int c = lane >> 1, hh = lane & 1;
        const bool cval = c < NS;
        const int cq = cval ? c : NS - 1;
        // a coupling into the warp's scratch (FP64); all 7 loads per lane issued before the stores
        auto stage = [&](double *dst, int l, int k) {
            double v[7];
            if (l == 0) {
                const ST *src = S + (kg0 + k) * kstride;
#pragma unroll
                for (int q = 0; q < 7; ++q) v[q] = (lane + 32 * q < SS) ? (double)__ldg(src + lane + 32 * q) : 0.0;
            } else {
                const double *src = lev_block(l, k);
#pragma unroll
                for (int q = 0; q < 7; ++q) v[q] = (lane + 32 * q < SS) ? src[lane + 32 * q] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < 7; ++q)
                if (lane + 32 * q < SS) dst[lane + 32 * q] = v[q];
        };
        // w[q] = (A_j^{-1} X)(7 hh + q, c) for X = Lw (x_cm: X(t, c) = Lw[t + 14 c]) or X = Lw^T
        auto ainv_times = [&](const double *Ai, const double *Lw, bool transpose, double (&w)[7]) {
            double xc[NS];
#pragma unroll
            for (int t = 0; t < NS; ++t) xc[t] = transpose ? Lw[cq + NS * t] : Lw[t + NS * cq];
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                const int rr = 7 * hh + q;
                double a = 0.0;
#pragma unroll
                for (int t = 0; t < NS; ++t) a = fma(Ai[tri_lo(rr, t)], xc[t], a);
                w[q] = a;
            }
        };
        // d[a] = (Y W)(a, c) with Y(a, t) = Lw[a + 14 t] (transpose: Lw[t + 14 a]); both lanes of a pair get the sum
        auto times_w = [&](const double *Lw, bool transpose, const double (&w)[7], double (&d)[NS]) {
#pragma unroll
            for (int a = 0; a < NS; ++a) {
                double acc = 0.0;
#pragma unroll
                for (int q = 0; q < 7; ++q) {
                    const int t = 7 * hh + q;
                    acc = fma(transpose ? Lw[t + NS * a] : Lw[a + NS * t], w[q], acc);
                }
                d[a] = acc + __shfl_xor_sync(0xffffffffu, acc, 1);
            }
        };
        for (int l = 0; l < nlev; ++l) {
            const int h = 1 << l;
            const int ne = (kpc - 1 - h) / (2 * h) + 1;
            // phase A: invert A_j; A_{j-h} -= L_j^T A_j^{-1} L_j
            for (int m = warp; m < ne; m += PCG_NWARP) {
                const int j = h * (2 * m + 1);
                stage(Lw0, l, j);
                double *Ai = Aq + (size_t)j * 105;
                warp_spd_inverse_packed(Ai, lane);
                double w[7], d[NS];
                ainv_times(Ai, Lw0, false, w);
                times_w(Lw0, true, w, d);
                double *Ad = Aq + (size_t)(j - h) * 105;
                if (cval) {
#pragma unroll
                    for (int a = 0; a < NS; ++a)
                        if (a >= c && (a & 1) == hh) Ad[((a * (a + 1)) >> 1) + c] -= d[a];
                }
                __syncwarp();
            }
            __syncthreads();
            // phase B: L'_{j+h} = L_{j+h} A_j^{-1} L_j; A_{j+h} -= L_{j+h} A_j^{-1} L_{j+h}^T
            for (int m = warp; m < ne; m += PCG_NWARP) {
                const int j = h * (2 * m + 1);
                if (j + h >= kpc) continue;
                stage(Lw0, l, j);
                stage(Lw1, l, j + h);
                __syncwarp();
                const double *Ai = Aq + (size_t)j * 105;
                double w[7], d[NS];
                ainv_times(Ai, Lw0, false, w);
                times_w(Lw1, false, w, d);
                double *Ln = lev_block(l + 1, j + h);
                if (cval) {
#pragma unroll
                    for (int a = 0; a < NS; ++a)
                        if ((a & 1) == hh) Ln[a + NS * c] = d[a];
                }
                ainv_times(Ai, Lw1, true, w);
                times_w(Lw1, false, w, d);
                double *Ad = Aq + (size_t)(j + h) * 105;
                if (cval) {
#pragma unroll
                    for (int a = 0; a < NS; ++a)
                        if (a >= c && (a & 1) == hh) Ad[((a * (a + 1)) >> 1) + c] -= d[a];
                }
                __syncwarp();
            }
            __syncthreads();
        }
        if (warp == 0) warp_spd_inverse_packed(Aq, lane);
        __syncthreads();
    }

    // ---- per-thread rows
    const bool worker = tid < PCG_WORKERS;
    const int r = worker ? tid % NS : 0, g0 = worker ? tid / NS : 0;
    int doff[NS];  // offsets of row r of the diagonal block within a knot block
#pragma unroll
    for (int cc = 0; cc < NS; ++cc) doff[cc] = diag_off<FMT>(r, cc);
    const float *gb = (FMT == 2) ? nullptr : gamma + NS * kg0;
    const double *gb64 = (FMT == 2) ? gamma64 + NS * kg0 : nullptr;
    float *lb = lambda + NS * kg0;
    double lam[PCG_KPT], res[PCG_KPT], pp[PCG_KPT], zz[PCG_KPT];
    double gv[PCG_KPT];
    bool own[PCG_KPT];
#pragma unroll
    for (int j = 0; j < PCG_KPT; ++j) {
        const int kl = g0 + PCG_TK * j;
        own[j] = worker && kl < kpc;
        lam[j] = res[j] = pp[j] = zz[j] = 0.0;
        gv[j] = 0.f;
        if (own[j]) {
            gv[j] = (FMT == 2) ? gb64[NS * kl + r] : (double)gb[NS * kl + r];
            lam[j] = (double)lb[NS * kl + r];
        }
    }
    // (S x)_row with FP64 accumulation; x = rv holds 14 (kpc+2) doubles with halo slots
    auto row_f64 = [&](int j) -> double {
        const int kl = g0 + PCG_TK * j, k = k0 + kl;
        const ST *lk = S + (kg0 + kl) * kstride;
        const double *xk = rv + NS * kl;
        ST fl[NS], fd[NS], fr[NS];
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) {
            fl[cc] = (k > 0) ? __ldg(lk + r + NS * cc) : 0.f;
            fd[cc] = __ldg(lk + doff[cc]);
            fr[cc] = (k < N - 1) ? __ldg(lk + kstride + cc + NS * r) : 0.f;
        }
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) {
            a0 = fma((double)fl[cc], xk[cc], a0);
            a1 = fma((double)fd[cc], xk[NS + cc], a1);
            a2 = fma((double)fr[cc], xk[2 * NS + cc], a2);
        }
        return (a0 + a1) + a2;
    };
    // write a per-row vector (FP64) into rv with its halo knots; barrier makes it visible
    auto publish = [&](const double (&v)[PCG_KPT], bool halo_from_global) {
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            if (own[j]) {
                const int kl = g0 + PCG_TK * j;
                rv[NS * (kl + 1) + r] = v[j];
                if constexpr (CS > 1) {
                    if (!halo_from_global) {
                        cg::cluster_group cl = cg::this_cluster();
                        if (kl == 0 && rank > 0) cl.map_shared_rank(rv, rank - 1)[NS * (kpc_left + 1) + r] = v[j];
                        if (kl == kpc - 1 && rank < CS - 1) cl.map_shared_rank(rv, rank + 1)[r] = v[j];
                    }
                }
            }
        }
        if (tid < NS) {
            if (halo_from_global) {
                rv[tid] = (k0 > 0) ? (double)lambda[NS * (kg0 - 1) + tid] : 0.0;
                rv[NS * (kpc + 1) + tid] = (k1 < N) ? (double)lambda[NS * ((size_t)kb + k1) + tid] : 0.0;
            } else {
                if (k0 == 0) rv[tid] = 0.0;
                if (k1 == N) rv[NS * (kpc + 1) + tid] = 0.0;
            }
        }
        if constexpr (CS > 1) {
            cg::this_cluster().sync();
        } else {
            __syncthreads();
        }
    };
    // all reads of rv's halo slots by neighbours done before rv is rewritten
    auto release = [&]() {
        if constexpr (CS > 1) {
            cg::this_cluster().sync();
        } else {
            __syncthreads();
        }
    };
    auto true_residual = [&](bool from_global) {
        publish(lam, from_global);
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j)
            if (own[j]) res[j] = (double)gv[j] - row_f64(j);
        release();
    };
    // exact chunk solve by all threads, in place on rv's interior slots: rv <- M_chunk^{-1} rv
    auto chain_solve = [&]() {
        for (int l = 0; l < nlev; ++l) {
            const int h = 1 << l;
            const int ne = (kpc - 1 - h) / (2 * h) + 1, ns = (kpc - 1) / (2 * h) + 1;
            for (int i = tid; i < ne * NS; i += PCG_THREADS) {
                const int m = i / NS, rr = i - m * NS, j = h * (2 * m + 1);
                const double *Ai = Aq + (size_t)j * 105, *y = rv + NS * (j + 1);
                double a = 0.0;
#pragma unroll
                for (int cc = 0; cc < NS; ++cc) a = fma(Ai[tri_lo(rr, cc)], y[cc], a);
                tv[NS * j + rr] = a;
            }
            __syncthreads();
            for (int i = tid; i < ns * NS; i += PCG_THREADS) {
                const int m = i / NS, rr = i - m * NS, k = 2 * h * m;
                double a = 0.0, cl[NS];
                if (k > 0) {
                    coupling_line(l, k, rr, false, cl);
                    const double *t = tv + NS * (k - h);
#pragma unroll
                    for (int cc = 0; cc < NS; ++cc) a = fma(cl[cc], t[cc], a);
                }
                if (k + h < kpc) {
                    coupling_line(l, k + h, rr, true, cl);
                    const double *t = tv + NS * (k + h);
#pragma unroll
                    for (int cc = 0; cc < NS; ++cc) a = fma(cl[cc], t[cc], a);
                }
                rv[NS * (k + 1) + rr] += a;
            }
            __syncthreads();
        }
        double x0 = 0.0;
        if (tid < NS) {
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) x0 = fma(Aq[tri_lo(tid, cc)], rv[NS + cc], x0);
        }
        __syncthreads();
        if (tid < NS) rv[NS + tid] = x0;
        __syncthreads();
        for (int l = nlev - 1; l >= 0; --l) {
            const int h = 1 << l;
            const int ne = (kpc - 1 - h) / (2 * h) + 1;
            for (int i = tid; i < ne * NS; i += PCG_THREADS) {
                const int m = i / NS, rr = i - m * NS, j = h * (2 * m + 1);
                const double *xl = rv + NS * (j - h + 1);
                double a = 0.0, cl[NS];
                coupling_line(l, j, rr, false, cl);
#pragma unroll
                for (int cc = 0; cc < NS; ++cc) a = fma(cl[cc], xl[cc], a);
                if (j + h < kpc) {
                    coupling_line(l, j + h, rr, true, cl);
                    const double *xr = rv + NS * (j + h + 1);
#pragma unroll
                    for (int cc = 0; cc < NS; ++cc) a = fma(cl[cc], xr[cc], a);
                }
                sv[NS * j + rr] = a;
            }
            __syncthreads();
            for (int i = tid; i < ne * NS; i += PCG_THREADS) {
                const int m = i / NS, rr = i - m * NS, j = h * (2 * m + 1);
                const double *Ai = Aq + (size_t)j * 105, *sj = sv + NS * j;
                double a = tv[NS * j + rr];
#pragma unroll
                for (int cc = 0; cc < NS; ++cc) a = fma(Ai[tri_lo(rr, cc)], sj[cc], a);
                rv[NS * (j + 1) + rr] = a;
            }
            __syncthreads();
        }
    };
    // z = S_chunk^{-1} r, partial dot products
    auto precond = [&](double (&d)[3]) {
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j)
            if (own[j]) rv[NS * (g0 + PCG_TK * j + 1) + r] = res[j];
        __syncthreads();
        chain_solve();
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            if (own[j]) {
                const int kl = g0 + PCG_TK * j;
                zz[j] = -rv[NS * (kl + 1) + r];
                d[1] += res[j] * zz[j];
                d[2] += res[j] * res[j];
            }
        }
    };

    // ---- initial residual (FP64, lambda FP32 from global with halos), z, p = z
    true_residual(true);
    int set = 1;
    double eta, rr2, gg;
    {
        double acc3[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j)
            if (own[j]) acc3[0] += (double)gv[j] * gv[j];
        precond(acc3);
        cluster_sum_raw<CS, 3>(acc3, slots, red, set);
        set ^= 1;
        gg = acc3[0];
        eta = acc3[1];
        rr2 = acc3[2];
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) pp[j] = zz[j];
    }
    auto converged = [&](double e, double r2) {
        return exit_mode == 0 ? (r2 <= (double)tol * (double)tol * gg) : (fabs(e) < (double)tol);
    };
    bool conv = converged(eta, rr2), bad = false;
    int it = 0;
    while (!conv && it < max_iter) {
        publish(pp, false);
        double d1[1] = {0.0};
        double vv[PCG_KPT];
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            vv[j] = 0.0;
            if (own[j]) {
                vv[j] = row_f64(j);
                d1[0] += pp[j] * vv[j];
            }
        }
        cluster_sum_raw<CS, 1>(d1, slots, red, set);  // its barrier also releases rv
        set ^= 1;
        const double alpha = eta / d1[0];
        if (!isfinite(alpha)) {
            bad = true;
            break;
        }
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) {
            lam[j] = fma(alpha, pp[j], lam[j]);
            res[j] = fma(-alpha, vv[j], res[j]);
        }
        ++it;
        bool replaced = false;
        if (it % RR_PERIOD == 0) {
            true_residual(false);
            replaced = true;
        }
        if (exit_mode == 0) {
            // ||r|| <= tol ||gamma||: tested before preconditioning, so the exact chunk solve runs
            // only while the iteration continues, and confirmed on the true residual from the second
            // iteration on.  After the first, r = r0 - alpha S p with r0 the true residual and S p one
            // FP64 product: it equals gamma - S lambda up to FP64 rounding, ~eps64 cond(S) relative
            // (~3e-8 at cond(S) = 2e7), far below any usable tolerance.
            double d0[1] = {0.0};
#pragma unroll
            for (int j = 0; j < PCG_KPT; ++j)
                if (own[j]) d0[0] += res[j] * res[j];
            cluster_sum_raw<CS, 1>(d0, slots, red, set);
            set ^= 1;
            if (!isfinite(d0[0])) {
                bad = true;
                break;
            }
            if (converged(0.0, d0[0]) && !replaced && it > 1) {
                true_residual(false);
                d0[0] = 0.0;
#pragma unroll
                for (int j = 0; j < PCG_KPT; ++j)
                    if (own[j]) d0[0] += res[j] * res[j];
                cluster_sum_raw<CS, 1>(d0, slots, red, set);
                set ^= 1;
            }
            if (converged(0.0, d0[0])) {
                conv = true;
                break;
            }
        }
        double d2[3] = {0.0, 0.0, 0.0};
        precond(d2);
        cluster_sum_raw<CS, 3>(d2, slots, red, set);
        set ^= 1;
        if (exit_mode != 0) conv = converged(d2[1], d2[2]);
        if (!isfinite(d2[1])) {
            bad = true;
            conv = false;
            break;
        }
        if (conv) break;
        const double beta = d2[1] / eta;
        eta = d2[1];
#pragma unroll
        for (int j = 0; j < PCG_KPT; ++j) pp[j] = fma(beta, pp[j], zz[j]);
    }
#pragma unroll
    for (int j = 0; j < PCG_KPT; ++j) {
        if (own[j]) {
            const int i = NS * (g0 + PCG_TK * j) + r;
            lb[i] = (float)lam[j];
            if (lambda64) lambda64[NS * kg0 + i] = lam[j];
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
    if constexpr (CS > 1) cg::this_cluster().sync();
}

// ---------------------------------------------------------------------------
// Warp-pair PCG: one 128-thread CTA per instance (pcg_cluster_size PCG_WARP_PAIR).
//
// The PCG of pcg_chain_kernel with one CTA per instance -- its preconditioner
// is the exact inverse of the instance's S -- with the factorisation done by a
// twisted block LDL^T instead of cyclic reduction.  With M = -S (SPD),
// A_k = -S_kk and E_k = M_{k,k-1} = -L_k (L_k the left block of row k), and
// m = (n-1)/2:
//   warp 0, top-down:   D_0 = A_0,         D_k = A_k - E_k D_{k-1}^{-1} E_k^T,          k = 1..m
//   warp 1, bottom-up:  U_{n-1} = A_{n-1}, U_k = A_k - E_{k+1}^T U_{k+1}^{-1} E_{k+1},  k = n-2..m+1
//   then                T_m = D_m - E_{m+1}^T U_{m+1}^{-1} E_{m+1}
// (the two warps run at the same time; the quadratic forms are sign-free, so
// L is used for E).  M x = y is then solved by
//   forward   t_k = D_k^{-1} y_k, y_{k+1} += L_{k+1} t_k          (k = 0..m-1)
//             t_k = U_k^{-1} y_k, y_{k-1} += L_k^T t_k            (k = n-1..m+1)
//   middle    x_m = T_m^{-1} y_m
//   backward  x_k = t_k + D_k^{-1} L_{k+1}^T x_{k+1}              (k = m-1..0)
//             x_k = t_k + U_k^{-1} L_k x_{k-1}                    (k = m+1..n-1)
// and z = S^{-1} r = -x.  Warps 2-3 form the initial residual gamma - S lambda
// while warps 0-1 factor.  Each elimination step is sequential, but a CTA
// holds ~36 KB of shared memory at n = 128 (4 CTAs per SM), so a batch of up to
// ~600 instances runs in one wave instead of one CTA per SM at a time.
//
// Storage: the inverse factors D_k^{-1}, U_k^{-1}, T_m^{-1} (packed lower
// triangles, FP64) and the PCG vectors lambda, r, p, S p (FP64) live in the
// FP64 workspace (196 doubles per knot); the solve's x and t in shared memory.
// S is read from global memory (FP64 rows of schur64_kernel, or FP32 packed
// rows), the next step's blocks loaded while the current step computes.
constexpr int PAIR_THREADS = 128;
constexpr int PAIR_NWARP = PAIR_THREADS / 32;
constexpr int PW_STRIDE = SS, PW_INV = 0, PW_LAM = 105, PW_RES = 119, PW_P = 133, PW_V = 147;
// per factoring warp: the previous inverse factor as a full symmetric matrix (196), the coupling
// block (196), the diagonal block A_k (packed lower triangle, 105) and the product buffer (196)
constexpr int PAIR_FWARP = 3 * SS + 105;
constexpr int PF_INV = 0, PF_L = SS, PF_A = 2 * SS, PF_W = 2 * SS + 105;

__host__ __device__ constexpr int pair_smem_doubles(int n)
{
    return 2 * NS * n + 2 * PAIR_FWARP + SS + NS + 2 * PAIR_NWARP * 3 + 2;
}
size_t pcg_pair_smem_bytes(int n) { return sizeof(double) * (size_t)pair_smem_doubles(n); }

// In-place Gauss-Jordan inverse of an SPD 14x14 matrix held by lane pairs: lane (c, hh) =
// (lane >> 1, lane & 1), c < 14, holds rows 7 hh .. 7 hh + 6 of column c in a[]; on return the
// same entries of the inverse.  The pivots are the 2x2 diagonal blocks P = {p, p+1} (no pivoting:
// each is a diagonal block of a Schur complement of an SPD matrix, hence SPD), which halves the
// chain of dependent reciprocals against scalar pivots.  Per block, with Pi = A_PP^{-1}:
//   A_Pc <- Pi A_Pc,  A_ic <- A_ic - A_iP (Pi A_Pc)  (i, c outside P),  A_iP <- -A_iP Pi,  A_PP <- Pi,
// done uniformly by treating the pivot columns as the identity's columns e_p, e_{p+1}.  The lane
// needs the pivot block, rows p, p+1 of its column and columns p, p+1 of its rows (shuffles).
__device__ __forceinline__ void pair_gj_inverse(double (&a)[7], int c, int hh)
{
    const int cs = c < NS ? c : NS - 1;
#pragma unroll
    for (int p = 0; p < NS; p += 2) {
        const int h0 = p / 7, q0 = p - 7 * h0, h1 = (p + 1) / 7, q1 = (p + 1) - 7 * h1;
        const double x = __shfl_sync(0xffffffffu, a[q0], 2 * p + h0);        // A_pp
        const double y = __shfl_sync(0xffffffffu, a[q1], 2 * p + h1);        // A_{p+1,p}
        const double z = __shfl_sync(0xffffffffu, a[q1], 2 * (p + 1) + h1);  // A_{p+1,p+1}
        const double v0 = __shfl_sync(0xffffffffu, a[q0], 2 * cs + h0);      // A_pc
        const double v1 = __shfl_sync(0xffffffffu, a[q1], 2 * cs + h1);      // A_{p+1,c}
        double u0[7], u1[7];                                                 // A_ip, A_i,p+1
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            u0[q] = __shfl_sync(0xffffffffu, a[q], 2 * p + hh);
            u1[q] = __shfl_sync(0xffffffffu, a[q], 2 * (p + 1) + hh);
        }
        const double rd = rcp_newton(fma(x, z, -y * y));
        const double i00 = z * rd, i01 = -y * rd, i11 = x * rd;
        const bool c0 = (c == p), c1 = (c == p + 1), cp = c0 || c1;
        const double w0 = cp ? (c0 ? 1.0 : 0.0) : v0, w1 = cp ? (c1 ? 1.0 : 0.0) : v1;
        const double n0 = fma(i00, w0, i01 * w1), n1 = fma(i01, w0, i11 * w1);
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            const int i = 7 * hh + q;
            const double upd = fma(-u0[q], n0, fma(-u1[q], n1, cp ? 0.0 : a[q]));
            a[q] = (i == p) ? n0 : ((i == p + 1) ? n1 : upd);
        }
    }
}
// row r of a 14x14 block times v: lane (r, hh) sums columns 7 hh .. 7 hh + 6, the pair adds up
__device__ __forceinline__ double pair_dot7(const double (&m)[7], const double *v, int hh)
{
    double a = 0.0;
#pragma unroll
    for (int q = 0; q < 7; ++q) a = fma(m[q], v[7 * hh + q], a);
    return a + __shfl_xor_sync(0xffffffffu, a, 1);
}
template <typename ST, int CNT>
__device__ __forceinline__ void warp_fetch(const ST *src, int n, int lane, double (&v)[CNT])
{
#pragma unroll
    for (int i = 0; i < CNT; ++i) {
        const int e = lane + 32 * i;
        v[i] = (e < n) ? (double)__ldg(src + e) : 0.0;
    }
}

template <int FMT>
__global__ void __launch_bounds__(PAIR_THREADS, 4)
    pcg_pair_kernel(BatchView bv, const void *__restrict__ Sv, const float *__restrict__ gamma,
                    const double *__restrict__ gamma64, float *__restrict__ lambda, double *__restrict__ lambda64,
                    double *__restrict__ ws, int max_iter, float tol, int exit_mode, uint32_t *__restrict__ out_iters,
                    uint32_t *__restrict__ pcg_log, int log_stride)
{
    static_assert(FMT == 1 || FMT == 2, "packed rows only");
    using ST = typename std::conditional<FMT == 2, double, float>::type;
    const ST *S = reinterpret_cast<const ST *>(Sv);
    const size_t ks = FMT == 2 ? PK64 : PK;
    const int b = bv.b0 + (int)blockIdx.x;
    if (b >= bv.b0 + bv.B || !bv.active(b)) return;
    const int n = bv.N(b), m = (n - 1) / 2, nv = NS * n;
    const size_t kg0 = (size_t)bv.off(b);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    extern __shared__ double pair_dyn_smem[];
    double *xv = pair_dyn_smem;        // 14 n: the solve's vector (y, then x); lambda_0 during set-up
    double *tv = xv + nv;              // 14 n: t_k of the solve
    double *fw0 = tv + nv;             // warp 0: D_{k-1}^{-1} (full), coupling / scratch, A_k
    double *fw1 = fw0 + PAIR_FWARP;    // warp 1: U_{k+1}^{-1} (full), coupling / scratch, A_k
    double *dmf = fw1 + PAIR_FWARP;    // D_m (full), from warp 0 to the middle step
    double *ubot = dmf + SS;           // 14: L_{m+1}^T t_{m+1} from the bottom sweep
    double *red = ubot + NS;           // 2 sets x 4 warps x 3
    double *ginit = red + 2 * PAIR_NWARP * 3;  // gamma . gamma partials of warps 2, 3

    const ST *Sb = S + kg0 * ks;
    double *wsb = ws + kg0 * PW_STRIDE;
    auto wsv = [&](int slot, int e) -> double & { return wsb[(size_t)(e / NS) * PW_STRIDE + slot + e % NS]; };
    const float *gb = (FMT == 2) ? nullptr : gamma + NS * kg0;
    const double *gb64 = (FMT == 2) ? gamma64 + NS * kg0 : nullptr;
    auto gam = [&](int e) -> double { return (FMT == 2) ? gb64[e] : (double)gb[e]; };
    float *lb = lambda + NS * kg0;

    // (S v)_e with FP64 accumulation (same order as pcg_chain_kernel's rows)
    auto srow = [&](int e, const double *v) -> double {
        const int k = e / NS, r = e - NS * k;
        const ST *row = Sb + (size_t)k * ks;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        ST fd[NS];
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) fd[cc] = __ldg(row + PK_DIAG + tri_lo(r, cc));
        if (k > 0) {
            ST fl[NS];
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) fl[cc] = __ldg(row + r + NS * cc);
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) a0 = fma((double)fl[cc], v[NS * (k - 1) + cc], a0);
        }
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) a1 = fma((double)fd[cc], v[NS * k + cc], a1);
        if (k < n - 1) {
            ST fr[NS];
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) fr[cc] = __ldg(row + ks + cc + NS * r);
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) a2 = fma((double)fr[cc], v[NS * (k + 1) + cc], a2);
        }
        return (a0 + a1) + a2;
    };

    const int c = lane >> 1, hh = lane & 1;
    const bool cval = c < NS;
    const int cq = cval ? c : NS - 1;
    // Wb <- L F L^T (F full symmetric, L column-major, both 14x14 in shared memory) on the FP64 tensor
    // cores: W = F L^T, then L W; every lane of the warp takes part
    auto schur_update = [&](const double *F, const double *L, double *Wb) {
        double cw[2][2][2] = {};
        warp_dmma<2, 2, 4>([&](int i, int k) { return (i < NS && k < NS) ? F[i + NS * k] : 0.0; },
                           [&](int k, int j) { return (k < NS && j < NS) ? L[j + NS * k] : 0.0; }, cw, lane);
        warp_dmma_store(cw, [&](int i, int j, double v) { if (i < NS && j < NS) Wb[i + NS * j] = v; }, lane);
        __syncwarp();
        double cd[2][2][2] = {};
        warp_dmma<2, 2, 4>([&](int i, int k) { return (i < NS && k < NS) ? L[i + NS * k] : 0.0; },
                           [&](int k, int j) { return (k < NS && j < NS) ? Wb[k + NS * j] : 0.0; }, cd, lane);
        __syncwarp();
        warp_dmma_store(cd, [&](int i, int j, double v) { if (i < NS && j < NS) Wb[i + NS * j] = v; }, lane);
        __syncwarp();
    };
    // an inverse factor: full matrix into shared memory (next step's products), packed lower
    // triangle into the workspace (the solve)
    auto keep_inv = [&](double *F, const double (&a)[7], int k) {
        __syncwarp();
        if (cval) {
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                const int i = 7 * hh + q;
                if (F) F[i + NS * c] = a[q];
                if (i >= c) wsb[(size_t)k * PW_STRIDE + PW_INV + ((i * (i + 1)) >> 1) + c] = a[q];
            }
        }
        __syncwarp();
    };

    // ---- factorisation (warps 0, 1) and initial residual (warps 2, 3).  Both factoring warps run
    // one loop body (one copy in the instruction cache): warp 0 walks k = 0 .. m with the coupling
    // L_k, warp 1 walks k = n-1 .. m+1 with L_{k+1} stored transposed, which turns its update
    // L_{k+1}^T U_{k+1}^{-1} L_{k+1} into the same products as warp 0's L_k D_{k-1}^{-1} L_k^T.
    if (warp < 2) {
        const bool top = warp == 0;
        double *fw = top ? fw0 : fw1;
        double *Fi = fw + PF_INV, *Lw = fw + PF_L, *Ap = fw + PF_A;
        const int steps = top ? m + 1 : n - 1 - m;
        const int dir = top ? 1 : -1, k0 = top ? 0 : n - 1, lofs = top ? 0 : 1;
        double pd[4], pl[7];  // diagonal triangle of row k, left block of row k + lofs
        if (steps > 0) {
            warp_fetch<ST, 4>(Sb + (size_t)k0 * ks + PK_DIAG, 105, lane, pd);
            if (top) warp_fetch<ST, 7>(Sb, SS, lane, pl);
        }
        for (int st = 0; st < steps; ++st) {
            const int k = k0 + dir * st;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int e = lane + 32 * i;
                if (e < 105) Ap[e] = -pd[i];
            }
            if (st > 0) {
#pragma unroll
                for (int i = 0; i < 7; ++i) {
                    const int e = lane + 32 * i;
                    if (e < SS) Lw[top ? e : (e / NS) + NS * (e % NS)] = pl[i];
                }
            }
            __syncwarp();
            if (st + 1 < steps) {
                warp_fetch<ST, 4>(Sb + (size_t)(k + dir) * ks + PK_DIAG, 105, lane, pd);
                warp_fetch<ST, 7>(Sb + (size_t)(k + dir + lofs) * ks, SS, lane, pl);
            }
            double *Wb = fw + PF_W;
            if (st > 0) schur_update(Fi, Lw, Wb);
            double a[7];
#pragma unroll
            for (int q = 0; q < 7; ++q)
                a[q] = Ap[tri_lo(7 * hh + q, cq)] - (st > 0 ? Wb[7 * hh + q + NS * cq] : 0.0);
            if (top && k == m) {
                if (cval) {
#pragma unroll
                    for (int q = 0; q < 7; ++q) dmf[7 * hh + q + NS * c] = a[q];
                }
            } else {
                pair_gj_inverse(a, c, hh);
                keep_inv(Fi, a, k);
            }
        }
    } else {
        const int t2 = tid - 64;
        for (int e = t2; e < nv; e += 64) xv[e] = (double)lb[e];
        asm volatile("bar.sync 1, 64;" ::: "memory");
        double g2 = 0.0;
        for (int e = t2; e < nv; e += 64) {
            const double gv = gam(e);
            wsv(PW_RES, e) = gv - srow(e, xv);
            wsv(PW_LAM, e) = xv[e];
            g2 += gv * gv;
        }
        g2 = warp_sum(g2);
        if (lane == 0) ginit[warp - 2] = g2;
    }
    __syncthreads();
    // ---- middle knot: T_m = D_m - L_{m+1}^T U_{m+1}^{-1} L_{m+1}, inverted (warp 1)
    if (warp == 1) {
        double *Wb = fw1 + PF_W;
        const bool upd = m + 1 <= n - 1;
        if (upd) {
            double *Fi = fw1 + PF_INV, *Lw = fw1 + PF_L;
            double pl[7];
            warp_fetch<ST, 7>(Sb + (size_t)(m + 1) * ks, SS, lane, pl);
#pragma unroll
            for (int i = 0; i < 7; ++i) {
                const int e = lane + 32 * i;
                if (e < SS) Lw[(e / NS) + NS * (e % NS)] = pl[i];  // transposed, as in the loop
            }
            __syncwarp();
            schur_update(Fi, Lw, Wb);
        }
        double a[7];
#pragma unroll
        for (int q = 0; q < 7; ++q) a[q] = dmf[7 * hh + q + NS * cq] - (upd ? Wb[7 * hh + q + NS * cq] : 0.0);
        pair_gj_inverse(a, c, hh);
        keep_inv(nullptr, a, m);
    }
    const double gg = ginit[0] + ginit[1];
    __syncthreads();

    // ---- M x = y in place on xv (warps 0, 1; every thread takes the barriers)
    const int r = c;  // sweep lanes: (row r, half hh)
    const bool rv = cval;
    auto ld_inv = [&](int k, double (&v)[7]) {
#pragma unroll
        for (int q = 0; q < 7; ++q) v[q] = rv ? wsb[(size_t)k * PW_STRIDE + PW_INV + tri_lo(r, 7 * hh + q)] : 0.0;
    };
    // row r (TR: column r) of L_k, columns (rows) 7 hh .. 7 hh + 6
    auto ld_left = [&](int k, bool tr, double (&v)[7]) {
        const ST *p = Sb + (size_t)k * ks;
#pragma unroll
        for (int q = 0; q < 7; ++q) v[q] = rv ? (double)__ldg(p + (tr ? 7 * hh + q + NS * r : r + NS * (7 * hh + q))) : 0.0;
    };
    // L2 prefetch of a sweep step's blocks (the packed inverse factor of knot kf, 840 B, and the left
    // block of row kl) PF_AHEAD steps before they are loaded; every address lies inside its block
    constexpr int PF_AHEAD = 4;
    constexpr int LEFT_LINES = (SS * (int)sizeof(ST) + 127) / 128;
    auto l2_prefetch = [&](int kf, int kl) {
        if (lane < 7) {
            if (kf >= 0 && kf < n)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(wsb + (size_t)kf * PW_STRIDE) + 128 * lane));
        } else if (lane < 7 + LEFT_LINES) {
            if (kl >= 1 && kl < n)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(Sb + (size_t)kl * ks) + 128 * (lane - 7)));
        }
    };
    auto solve = [&]() {
        if (warp == 0 && m > 0) {
            double di[7], li[7];
            ld_inv(0, di);
            ld_left(1, false, li);
            for (int k = 0; k < m; ++k) {
                double dc[7], lc[7];
#pragma unroll
                for (int q = 0; q < 7; ++q) {
                    dc[q] = di[q];
                    lc[q] = li[q];
                }
                if (k + 1 < m) {
                    ld_inv(k + 1, di);
                    ld_left(k + 2, false, li);
                }
                l2_prefetch(k + PF_AHEAD < m ? k + PF_AHEAD : -1, k + PF_AHEAD + 1);
                const double a = pair_dot7(dc, xv + NS * k, hh);
                if (hh == 0 && rv) tv[NS * k + r] = a;
                __syncwarp();
                const double u = pair_dot7(lc, tv + NS * k, hh);
                if (hh == 0 && rv) xv[NS * (k + 1) + r] += u;
                __syncwarp();
            }
        } else if (warp == 1) {
            if (n - 1 > m) {
                double di[7], li[7];
                ld_inv(n - 1, di);
                ld_left(n - 1, true, li);
                for (int k = n - 1; k > m; --k) {
                    double dc[7], lc[7];
#pragma unroll
                    for (int q = 0; q < 7; ++q) {
                        dc[q] = di[q];
                        lc[q] = li[q];
                    }
                    if (k - 1 > m) {
                        ld_inv(k - 1, di);
                        ld_left(k - 1, true, li);
                    }
                    l2_prefetch(k - PF_AHEAD > m ? k - PF_AHEAD : -1, k - PF_AHEAD > m ? k - PF_AHEAD : -1);
                    const double a = pair_dot7(dc, xv + NS * k, hh);
                    if (hh == 0 && rv) tv[NS * k + r] = a;
                    __syncwarp();
                    const double u = pair_dot7(lc, tv + NS * k, hh);
                    if (hh == 0 && rv) {
                        if (k - 1 > m) xv[NS * (k - 1) + r] += u;
                        else ubot[r] = u;
                    }
                    __syncwarp();
                }
            } else if (lane < NS) {
                ubot[lane] = 0.0;
            }
        }
        __syncthreads();
        if (warp == 0) {
            double *sc = fw0 + PF_L;
            double di[7];
            ld_inv(m, di);
            if (lane < NS) sc[lane] = xv[NS * m + lane] + ubot[lane];
            __syncwarp();
            const double a = pair_dot7(di, sc, hh);
            if (hh == 0 && rv) xv[NS * m + r] = a;
        }
        __syncthreads();
        if (warp == 0 && m > 0) {
            double *sc = fw0 + PF_L;
            double di[7], li[7];
            ld_inv(m - 1, di);
            ld_left(m, true, li);
            for (int k = m - 1; k >= 0; --k) {
                double dc[7], lc[7];
#pragma unroll
                for (int q = 0; q < 7; ++q) {
                    dc[q] = di[q];
                    lc[q] = li[q];
                }
                if (k > 0) {
                    ld_inv(k - 1, di);
                    ld_left(k, true, li);
                }
                l2_prefetch(k - PF_AHEAD, k - PF_AHEAD + 1);
                const double s = pair_dot7(lc, xv + NS * (k + 1), hh);
                if (hh == 0 && rv) sc[r] = s;
                __syncwarp();
                const double a = pair_dot7(dc, sc, hh);
                if (hh == 0 && rv) xv[NS * k + r] = tv[NS * k + r] + a;
                __syncwarp();
            }
        } else if (warp == 1 && n - 1 > m) {
            double *sc = fw1 + PF_L;
            double di[7], li[7];
            ld_inv(m + 1, di);
            ld_left(m + 1, false, li);
            for (int k = m + 1; k < n; ++k) {
                double dc[7], lc[7];
#pragma unroll
                for (int q = 0; q < 7; ++q) {
                    dc[q] = di[q];
                    lc[q] = li[q];
                }
                if (k + 1 < n) {
                    ld_inv(k + 1, di);
                    ld_left(k + 1, false, li);
                }
                l2_prefetch(k + PF_AHEAD, k + PF_AHEAD);
                const double s = pair_dot7(lc, xv + NS * (k - 1), hh);
                if (hh == 0 && rv) sc[r] = s;
                __syncwarp();
                const double a = pair_dot7(dc, sc, hh);
                if (hh == 0 && rv) xv[NS * k + r] = tv[NS * k + r] + a;
                __syncwarp();
            }
        }
        __syncthreads();
    };

    // ---- CG on the instance (the iteration of pcg_chain_kernel with one CTA)
    int set = 0;
    auto block_sum = [&](double *v, int cnt) {
        for (int q = 0; q < cnt; ++q) {
            const double s = warp_sum(v[q]);
            if (lane == 0) red[set * PAIR_NWARP * 3 + warp * 3 + q] = s;
        }
        __syncthreads();
        for (int q = 0; q < cnt; ++q) {
            const double *rs = red + set * PAIR_NWARP * 3 + q;
            v[q] = ((rs[0] + rs[3]) + rs[6]) + rs[9];
        }
        set ^= 1;
    };
    auto true_residual = [&]() {
        __syncthreads();
        for (int e = tid; e < nv; e += PAIR_THREADS) xv[e] = wsv(PW_LAM, e);
        __syncthreads();
        for (int e = tid; e < nv; e += PAIR_THREADS) wsv(PW_RES, e) = gam(e) - srow(e, xv);
    };
    // z = S^{-1} r = -x of M x = r (left in xv); d[1] += r.z, d[2] += r.r
    auto precond = [&](double *d) {
        __syncthreads();
        for (int e = tid; e < nv; e += PAIR_THREADS) xv[e] = wsv(PW_RES, e);
        __syncthreads();
        solve();
        for (int e = tid; e < nv; e += PAIR_THREADS) {
            const double rr = wsv(PW_RES, e), z = -xv[e];
            d[1] += rr * z;
            d[2] += rr * rr;
        }
    };
    auto sum_res2 = [&]() {
        double d0[1] = {0.0};
        for (int e = tid; e < nv; e += PAIR_THREADS) {
            const double rr = wsv(PW_RES, e);
            d0[0] += rr * rr;
        }
        block_sum(d0, 1);
        return d0[0];
    };
    auto converged = [&](double e, double r2) {
        return exit_mode == 0 ? (r2 <= (double)tol * (double)tol * gg) : (fabs(e) < (double)tol);
    };

    double eta;
    bool conv, bad = false;
    {
        double acc3[3] = {0.0, 0.0, 0.0};
        precond(acc3);
        block_sum(acc3, 3);
        eta = acc3[1];
        for (int e = tid; e < nv; e += PAIR_THREADS) wsv(PW_P, e) = -xv[e];  // p = z
        conv = converged(eta, acc3[2]);
    }
    int it = 0;
    while (!conv && it < max_iter) {
        __syncthreads();
        for (int e = tid; e < nv; e += PAIR_THREADS) xv[e] = wsv(PW_P, e);
        __syncthreads();
        double d1[1] = {0.0};
        for (int e = tid; e < nv; e += PAIR_THREADS) {
            const double v = srow(e, xv);
            wsv(PW_V, e) = v;
            d1[0] += xv[e] * v;
        }
        block_sum(d1, 1);
        const double alpha = eta / d1[0];
        if (!isfinite(alpha)) {
            bad = true;
            break;
        }
        double r2acc = 0.0;
        for (int e = tid; e < nv; e += PAIR_THREADS) {
            wsv(PW_LAM, e) = fma(alpha, xv[e], wsv(PW_LAM, e));
            const double rn = fma(-alpha, wsv(PW_V, e), wsv(PW_RES, e));
            wsv(PW_RES, e) = rn;
            r2acc += rn * rn;
        }
        ++it;
        bool replaced = false;
        if (it % RR_PERIOD == 0) {
            true_residual();
            replaced = true;
        }
        if (exit_mode == 0) {
            // ||r|| <= tol ||gamma||: tested before preconditioning; confirmed on the true residual from
            // the second iteration on (after the first, r = r0 - alpha S p equals gamma - S lambda up to
            // FP64 rounding, ~eps64 cond(S) relative, as in pcg_chain_kernel)
            double r2;
            if (replaced) {
                r2 = sum_res2();
            } else {
                double t1[1] = {r2acc};  // the update pass's sum, in sum_res2's order
                block_sum(t1, 1);
                r2 = t1[0];
            }
            if (!isfinite(r2)) {
                bad = true;
                break;
            }
            if (converged(0.0, r2) && !replaced && it > 1) {
                true_residual();
                r2 = sum_res2();
            }
            if (converged(0.0, r2)) {
                conv = true;
                break;
            }
        }
        double d2[3] = {0.0, 0.0, 0.0};
        precond(d2);
        block_sum(d2, 3);
        if (exit_mode != 0) conv = converged(d2[1], d2[2]);
        if (!isfinite(d2[1])) {
            bad = true;
            conv = false;
            break;
        }
        if (conv) break;
        const double beta = d2[1] / eta;
        eta = d2[1];
        for (int e = tid; e < nv; e += PAIR_THREADS) wsv(PW_P, e) = fma(beta, wsv(PW_P, e), -xv[e]);
    }
    for (int e = tid; e < nv; e += PAIR_THREADS) {
        const double lam = wsv(PW_LAM, e);
        lb[e] = (float)lam;
        if (lambda64) lambda64[NS * kg0 + e] = lam;
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
}

// ---------------------------------------------------------------------------
// Partitioned PCG: one 128-thread CTA per instance whose four warps factor four parts of the
// horizon (pcg_cluster_size PCG_WARP_QUAD).
//
// The exact preconditioner of pcg_pair_kernel (S^{-1} up to rounding), with the factorisation
// split four ways so that each warp walks about a quarter of the horizon instead of half of it,
// and every warp of the CTA (hence every SM sub-partition) factors.  With M = -S (SPD), A_k = M_kk,
// E_k = M_{k,k-1} = -L_k, the horizon is cut by P - 1 separator knots s_1 < ... < s_{P-1}
// (P = 4 from n = 7 on) into P parts.  Part 0 is factored top-down toward s_1 and part P-1
// bottom-up toward s_{P-1} (the two ends of the twisted factorisation); a middle part a .. b
// between s_p and s_{p+1} top-down, which couples its two separators: with F_k = M_{k, s_p}
// (F_a = E_a = -L_a) it carries
//   F_{k+1} = L_{k+1} D_k^{-1} F_k   and accumulates   Acc = sum_k F_k^T D_k^{-1} F_k,
// and ends with E^ = L_{s_{p+1}} D_b^{-1} F_b = M_{s_{p+1}, s_p} after its elimination.  The
// separators' reduced system (block tridiagonal, P - 1 blocks) has the diagonal blocks
//   A_{s_j} - (update of the part on its left) - (Acc of the middle part on its right, or the
//   update of the last part)
// and is factored by one warp after the parts.  The solve runs the same order: each part forward
// (t_k = D_k^{-1} y_k, pushing L_{k+1} t_k to the next knot and, in a middle part, -F_k^T t_k to
// its left separator), the reduced system forward and back, each part backward
// (x_k = t_k + D_k^{-1} (L_{k+1}^T x_{k+1} - F_k x_{s_p})).  This is the block LDL^T of M with the
// parts' knots ordered before the separators, so the preconditioner stays exact (z = S^{-1} r =
// -x) and the CG of pcg_pair_kernel stops after one iteration.  For that reason the iteration starts
// from lambda = 0 (r_0 = gamma, no product with S before the factorisation; the caller's warm start
// cannot save the one iteration), unlike pcg_pair_kernel.  Edge parts have two block products per
// step, middle parts five, so edge parts are made 1.3 times as long.
//
// Storage: per knot 2 x 196 doubles of the FP64 workspace: the pair kernel's slots (packed inverse
// factor, lambda, r, p, S p) and the middle parts' F_k (full); the solve's t_k overwrites y_k in
// the shared vector and x_k overwrites t_k.  Shared memory: the vector (14 n), per warp the
// factorisation scratch of the pair kernel, per middle part F, D^{-1} F and Acc, the separators'
// right-hand-side contributions.
constexpr int QUAD_THREADS = 128;
constexpr int QW_STRIDE = 2 * SS;  // workspace doubles per knot
constexpr int QW_SPIKE = SS;       // F_k (full 14 x 14) at this offset of a middle part's knot
constexpr int QSP = 3 * SS;        // per middle part: F, X = D^{-1} F, Acc

// The backward solve sweep stages each step's packed inverse factor (106 doubles, read as 53 16-byte
// chunks; the last double is the knot's first lambda entry) and coupling block (196 entries of S) into
// shared memory by cp.async, QSTAGE slots per warp (two steps ahead), in the factorisation's scratch.
constexpr int QSTAGE = 3, QINV_D = 106, QSLOT = QINV_D + SS;
constexpr int QREGION = QUAD_NWARP * PAIR_FWARP > QUAD_NWARP * QSTAGE * QSLOT ? QUAD_NWARP * PAIR_FWARP
                                                                               : QUAD_NWARP * QSTAGE * QSLOT;
__host__ __device__ constexpr int quad_smem_doubles(int n)
{
    return NS * n + QREGION + (QUAD_NWARP - 2) * QSP + (QUAD_NWARP - 1) * 2 * NS + 2 * QUAD_NWARP * 3 +
           QUAD_NWARP + QUAD_NWARP * NS + 2;
}

// the lanes of a warp copy `chunks` 16-byte chunks (both addresses 16-byte aligned)
__device__ __forceinline__ void warp_cp_async(void *sdst, const void *gsrc, int chunks, int lane)
{
    for (int i = lane; i < chunks; i += 32)
        cp_async16(reinterpret_cast<char *>(sdst) + 16 * i, reinterpret_cast<const char *>(gsrc) + 16 * i);
}
size_t pcg_quad_smem_bytes(int n) { return sizeof(double) * (size_t)quad_smem_doubles(n); }

// C (<-|+=) op(A) op(B) for 14 x 14 blocks (column-major, shared memory), FP64 tensor cores; one warp.
// C must not alias A or B.
template <bool TA, bool TB, bool ACC>
__device__ __forceinline__ void blk_mm(const double *A, const double *B, double *C, int lane)
{
    const int g = lane >> 2, t = lane & 3;
    double c[2][2][2];
#pragma unroll
    for (int I = 0; I < 2; ++I)
#pragma unroll
        for (int J = 0; J < 2; ++J)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int i = 8 * I + g, j = 8 * J + 2 * t + e;
                c[I][J][e] = (ACC && i < NS && j < NS) ? C[i + NS * j] : 0.0;
            }
    warp_dmma<2, 2, 4>([&](int i, int k) { return (i < NS && k < NS) ? (TA ? A[k + NS * i] : A[i + NS * k]) : 0.0; },
                       [&](int k, int j) { return (k < NS && j < NS) ? (TB ? B[j + NS * k] : B[k + NS * j]) : 0.0; },
                       c, lane);
    __syncwarp();
    warp_dmma_store(c, [&](int i, int j, double v) { if (i < NS && j < NS) C[i + NS * j] = v; }, lane);
    __syncwarp();
}

template <int FMT>
__global__ void __launch_bounds__(QUAD_THREADS, 4)
    pcg_quad_kernel(BatchView bv, const void *__restrict__ Sv, const float *__restrict__ gamma,
                    const double *__restrict__ gamma64, float *__restrict__ lambda, double *__restrict__ lambda64,
                    double *__restrict__ ws, int max_iter, float tol, int exit_mode, uint32_t *__restrict__ out_iters,
                    uint32_t *__restrict__ pcg_log, int log_stride)
{
    static_assert(FMT == 1 || FMT == 2, "packed rows only");
    using ST = typename std::conditional<FMT == 2, double, float>::type;
    const ST *S = reinterpret_cast<const ST *>(Sv);
    const size_t ks = FMT == 2 ? PK64 : PK;
    const int b = bv.b0 + (int)blockIdx.x;
    if (b >= bv.b0 + bv.B || !bv.active(b)) return;
    const int n = bv.N(b), nv = NS * n;
    const QuadLayout lay = quad_layout(n);
    const int P = lay.P;
    const size_t kg0 = (size_t)bv.off(b);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    extern __shared__ double quad_dyn_smem[];
    double *xv = quad_dyn_smem;                       // 14 n: y, then t (forward), then x (backward)
    double *fwall = xv + nv;                          // per warp: inverse factor (full), coupling, A_k, product;
                                                      // the backward sweep's staging slots
    double *spall = fwall + QREGION;                  // middle parts 1, 2: F, X = D^{-1} F, Acc
    double *sacc = spall + (QUAD_NWARP - 2) * QSP;    // per separator: right-hand-side pushes from left, right
    double *red = sacc + (QUAD_NWARP - 1) * 2 * NS;   // 2 sets x 4 warps x 3
    double *ginit = red + 2 * QUAD_NWARP * 3;         // gamma . gamma per warp
    double *scw = ginit + QUAD_NWARP;                 // per warp: 14 doubles of the backward sweep

    const ST *Sb = S + kg0 * ks;
    double *wsb = ws + kg0 * QW_STRIDE;
    auto wsv = [&](int slot, int e) -> double & { return wsb[(size_t)(e / NS) * QW_STRIDE + slot + e % NS]; };
    const float *gb = (FMT == 2) ? nullptr : gamma + NS * kg0;
    const double *gb64 = (FMT == 2) ? gamma64 + NS * kg0 : nullptr;
    auto gam = [&](int e) -> double { return (FMT == 2) ? gb64[e] : (double)gb[e]; };
    float *lb = lambda + NS * kg0;

    // (S v)_e with FP64 accumulation (the order of pcg_pair_kernel)
    auto srow = [&](int e, const double *v) -> double {
        const int k = e / NS, r = e - NS * k;
        const ST *row = Sb + (size_t)k * ks;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        ST fd[NS];
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) fd[cc] = __ldg(row + PK_DIAG + tri_lo(r, cc));
        if (k > 0) {
            ST fl[NS];
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) fl[cc] = __ldg(row + r + NS * cc);
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) a0 = fma((double)fl[cc], v[NS * (k - 1) + cc], a0);
        }
#pragma unroll
        for (int cc = 0; cc < NS; ++cc) a1 = fma((double)fd[cc], v[NS * k + cc], a1);
        if (k < n - 1) {
            ST fr[NS];
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) fr[cc] = __ldg(row + ks + cc + NS * r);
#pragma unroll
            for (int cc = 0; cc < NS; ++cc) a2 = fma((double)fr[cc], v[NS * (k + 1) + cc], a2);
        }
        return (a0 + a1) + a2;
    };

    const int c = lane >> 1, hh = lane & 1;
    const bool cval = c < NS;
    const int cq = cval ? c : NS - 1;
    auto keep_inv = [&](double *F, const double (&a)[7], int k) {
        __syncwarp();
        if (cval) {
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                const int i = 7 * hh + q;
                if (F) F[i + NS * c] = a[q];
                if (i >= c) wsb[(size_t)k * QW_STRIDE + PW_INV + ((i * (i + 1)) >> 1) + c] = a[q];
            }
        }
        __syncwarp();
    };

    // ---- the iteration starts from lambda = 0: with the exact preconditioner one iteration reaches
    // the solution from any start, and r_0 = gamma needs no product with S
    double g2acc = 0.0;  // gamma . gamma, this thread's entries
    for (int e = tid; e < nv; e += QUAD_THREADS) {
        const double gv = gam(e);
        wsv(PW_RES, e) = gv;
        wsv(PW_LAM, e) = 0.0;
        xv[e] = gv;  // y of the first preconditioner solve, M x = r_0
        g2acc = fma(gv, gv, g2acc);
    }
    const int r = c;
    const bool rv = cval;
    // row r of a 14 x 14 block in shared memory (column-major) times v, on the lane pair (r, hh)
    auto blk_row_dot = [&](const double *Mb, const double *v) -> double {
        double acc = 0.0;
#pragma unroll
        for (int q = 0; q < 7; ++q) acc = fma(Mb[r + NS * (7 * hh + q)], v[7 * hh + q], acc);
        return acc + __shfl_xor_sync(0xffffffffu, acc, 1);
    };
    __syncthreads();
    // ---- factorisation of the parts: warp w walks part w (top-down, or bottom-up for the last part).
    // The forward half of the first preconditioner solve runs in the same walk: after knot k's inverse
    // factor, t_k = D_k^{-1} y_k, and the next step pushes its coupling times t_k onto y (or, after the
    // part's last knot, onto the separator's right-hand side); a middle part accumulates -F_k^T t_k for
    // its left separator.  r_0 = gamma is known before the factorisation (the iteration starts from 0).
    if (warp < P) {
        const int w = warp;
        const bool top = (w < P - 1) || (P == 1);
        const bool spk = top && w > 0;                 // middle part: carries F toward separator s_{w-1}
        const bool has_sep = top ? (w < P - 1) : true;  // a separator after the walk
        const int pa = lay.a[w], pb = lay.b[w];
        const int len = pb >= pa ? pb - pa + 1 : 0;
        double *fw = fwall + w * PAIR_FWARP;
        double *Fi = fw + PF_INV, *Lw = fw + PF_L, *Ap = fw + PF_A, *Wb = fw + PF_W;
        double *Fsp = spk ? spall + (w - 1) * QSP : nullptr;
        double *Xb = spk ? Fsp + SS : nullptr, *Acc = spk ? Fsp + 2 * SS : nullptr;
        const int k0 = top ? pa : pb, dir = top ? 1 : -1, lofs = top ? 0 : 1;
        const int sep_slot = top ? 2 * w : 2 * (P - 2) + 1;  // this part's push onto its separator
        double accv = 0.0;                                   // -F_k^T t_k summed (middle part), this lane's half
        double pd[4] = {0.0, 0.0, 0.0, 0.0}, pl[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (len > 0) warp_fetch<ST, 4>(Sb + (size_t)k0 * ks + PK_DIAG, 105, lane, pd);
        if (spk) {
            // F_a = E_a = -L_a (row a's left block couples a to s_{w-1}); for an empty part a is s_w and
            // -L_{s_w} is the separators' own coupling
            double fl[7];
            warp_fetch<ST, 7>(Sb + (size_t)pa * ks, SS, lane, fl);
#pragma unroll
            for (int i = 0; i < 7; ++i) {
                const int e = lane + 32 * i;
                if (e < SS) {
                    Fsp[e] = -fl[i];
                    Acc[e] = 0.0;
                }
            }
        }
        if (len == 0) {
            for (int e = lane; e < SS; e += 32) Wb[e] = 0.0;  // no update of the separator
        } else if (len > 1 || has_sep) {
            warp_fetch<ST, 7>(Sb + (size_t)(k0 + dir + lofs) * ks, SS, lane, pl);
        }
        __syncwarp();
        for (int st = 0; st < len || (st == len && has_sep && len > 0); ++st) {
            const bool sep_step = st == len;
            const int k = k0 + dir * st;
            if (!sep_step) {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int e = lane + 32 * i;
                    if (e < 105) Ap[e] = -pd[i];
                }
            }
            if (st > 0) {
#pragma unroll
                for (int i = 0; i < 7; ++i) {
                    const int e = lane + 32 * i;
                    if (e < SS) Lw[top ? e : (e / NS) + NS * (e % NS)] = pl[i];
                }
            }
            __syncwarp();
            if (!sep_step) {
                if (st + 1 < len) {
                    warp_fetch<ST, 4>(Sb + (size_t)(k + dir) * ks + PK_DIAG, 105, lane, pd);
                    warp_fetch<ST, 7>(Sb + (size_t)(k + dir + lofs) * ks, SS, lane, pl);
                } else if (has_sep) {
                    warp_fetch<ST, 7>(Sb + (size_t)(k + dir + lofs) * ks, SS, lane, pl);
                }
            }
            if (spk && st > 0) blk_mm<false, false, false>(Lw, Xb, Fsp, lane);  // F_k = L_k D_{k-1}^{-1} F_{k-1}
            if (st > 0) {
                // Wb <- L D_prev^{-1} L^T = L (D_prev^{-1} L^T): W = D^{-1} L^T, then L W
                blk_mm<false, true, false>(Fi, Lw, Wb, lane);
                double cd[2][2][2] = {};
                warp_dmma<2, 2, 4>([&](int i, int kk) { return (i < NS && kk < NS) ? Lw[i + NS * kk] : 0.0; },
                                   [&](int kk, int j) { return (kk < NS && j < NS) ? Wb[kk + NS * j] : 0.0; }, cd,
                                   lane);
                __syncwarp();
                warp_dmma_store(cd, [&](int i, int j, double v) { if (i < NS && j < NS) Wb[i + NS * j] = v; }, lane);
                __syncwarp();
                // forward solve: the previous knot's t through the coupling block Lw
                const double u = blk_row_dot(Lw, xv + NS * (k - dir));
                if (hh == 0 && rv) {
                    if (sep_step) sacc[sep_slot * NS + r] = u;
                    else xv[NS * k + r] += u;
                }
                __syncwarp();
            }
            if (sep_step) break;  // Wb: the separator's update; Fsp (middle part): E^ = M_{s_w, s_{w-1}}
            double a[7];
#pragma unroll
            for (int q = 0; q < 7; ++q)
                a[q] = Ap[tri_lo(7 * hh + q, cq)] - (st > 0 ? Wb[7 * hh + q + NS * cq] : 0.0);
            pair_gj_inverse(a, c, hh);
            keep_inv(Fi, a, k);
            {
                const double t = pair_dot7(a, xv + NS * k, hh);  // t_k = D_k^{-1} y_k (D_k^{-1} symmetric)
                __syncwarp();
                if (hh == 0 && rv) xv[NS * k + r] = t;
                __syncwarp();
                if (spk) {
                    double pf = 0.0;
#pragma unroll
                    for (int q = 0; q < 7; ++q) pf = fma(Fsp[7 * hh + q + NS * r], xv[NS * k + 7 * hh + q], pf);
                    accv -= pf;
                }
            }
            if (spk) {
                double *fg = wsb + (size_t)k * QW_STRIDE + QW_SPIKE;
                for (int e = lane; e < SS; e += 32) fg[e] = Fsp[e];
                blk_mm<false, false, false>(Fi, Fsp, Xb, lane);  // X_k = D_k^{-1} F_k
                blk_mm<true, false, true>(Fsp, Xb, Acc, lane);   // Acc += F_k^T X_k
            }
        }
        if (spk) {
            accv += __shfl_xor_sync(0xffffffffu, accv, 1);
            if (hh == 0 && rv) sacc[(2 * (w - 1) + 1) * NS + r] = accv;
        }
        if (len == 0 && has_sep && lane < NS) sacc[sep_slot * NS + lane] = 0.0;
    }
    {
        const double g2 = warp_sum(g2acc);
        if (lane == 0) ginit[warp] = g2;
    }
    __syncthreads();
    const double gg = ((ginit[0] + ginit[1]) + ginit[2]) + ginit[3];

    // ---- the separators' reduced system, factored top-down by warp 0:
    //   D^_j = A_{s_j} - (left part's update) - (right part's Acc or update) - E^_j D^_{j-1}^{-1} E^_j^T
    if (warp == 0 && P >= 2) {
        double *Fi0 = fwall + PF_INV, *T0 = fwall + PF_L, *Ap0 = fwall + PF_A, *W0 = fwall + PF_W;
        for (int j = 0; j < P - 1; ++j) {
            const int s = lay.s[j];
            double pd[4];
            warp_fetch<ST, 4>(Sb + (size_t)s * ks + PK_DIAG, 105, lane, pd);
            const double *cl = fwall + j * PAIR_FWARP + PF_W;  // j = 0: W0, read before W0 is reused
            const double *cr = (j + 1 == P - 1) ? fwall + (P - 1) * PAIR_FWARP + PF_W : spall + j * QSP + 2 * SS;
            double a[7];
            if (j > 0) {
                const double *Eh = spall + (j - 1) * QSP;  // E^_j: the middle part between s_{j-1} and s_j
                blk_mm<false, false, false>(Eh, Fi0, T0, lane);  // E^_j D^_{j-1}^{-1}
                blk_mm<false, true, false>(T0, Eh, W0, lane);    // ... E^_j^T
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int e = lane + 32 * i;
                if (e < 105) Ap0[e] = -pd[i];
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                const int i = 7 * hh + q;
                a[q] = ((Ap0[tri_lo(i, cq)] - cl[i + NS * cq]) - cr[i + NS * cq]) - (j > 0 ? W0[i + NS * cq] : 0.0);
            }
            pair_gj_inverse(a, c, hh);
            keep_inv(Fi0, a, s);
        }
    }
    __syncthreads();

    // ---- M x = y in place on xv (every thread takes the barriers)
    auto ld_inv = [&](int k, double (&v)[7]) {
#pragma unroll
        for (int q = 0; q < 7; ++q) v[q] = rv ? wsb[(size_t)k * QW_STRIDE + PW_INV + tri_lo(r, 7 * hh + q)] : 0.0;
    };
    // row r of L_k (TR: of L_k^T), columns 7 hh .. 7 hh + 6
    auto ld_left = [&](int k, bool tr, double (&v)[7]) {
        const ST *p = Sb + (size_t)k * ks;
#pragma unroll
        for (int q = 0; q < 7; ++q)
            v[q] = rv ? (double)__ldg(p + (tr ? 7 * hh + q + NS * r : r + NS * (7 * hh + q))) : 0.0;
    };
    // row r of F_k (TR: of F_k^T)
    auto ld_spike = [&](int k, bool tr, double (&v)[7]) {
        const double *p = wsb + (size_t)k * QW_STRIDE + QW_SPIKE;
#pragma unroll
        for (int q = 0; q < 7; ++q) v[q] = rv ? p[tr ? 7 * hh + q + NS * r : r + NS * (7 * hh + q)] : 0.0;
    };
    // L2 prefetch of the blocks a sweep step loads QPF steps later: the packed inverse factor (840 B), the
    // coupling block of S and, for a middle part, F_k; every address lies inside its block
    constexpr int QPF = 4;
    constexpr int INV_LINES = (105 * 8 + 127) / 128, L_LINES = (SS * (int)sizeof(ST) + 127) / 128,
                  F_LINES = (SS * 8 + 127) / 128;
    auto l2_pf = [&](int ki, int kl, int kf) {
        const char *pi = reinterpret_cast<const char *>(wsb + (size_t)ki * QW_STRIDE);
        const char *pl = reinterpret_cast<const char *>(Sb + (size_t)kl * ks);
        const char *pf = reinterpret_cast<const char *>(wsb + (size_t)kf * QW_STRIDE + QW_SPIKE);
        if (lane < INV_LINES) {
            if (ki >= 0 && ki < n) asm volatile("prefetch.global.L2 [%0];" ::"l"(pi + 128 * lane));
        } else if (lane < INV_LINES + L_LINES) {
            if (kl >= 0 && kl < n) asm volatile("prefetch.global.L2 [%0];" ::"l"(pl + 128 * (lane - INV_LINES)));
        }
        if (lane < F_LINES && kf >= 0 && kf < n) asm volatile("prefetch.global.L2 [%0];" ::"l"(pf + 128 * lane));
    };
    // fwd: run the forward half (false when the factorisation's walk already ran it)
    auto solve = [&](bool fwd) {
        // forward through every part: t_k = D_k^{-1} y_k overwrites y_k
        if (fwd && warp < P) {
            const int w = warp;
            const bool top = (w < P - 1) || (P == 1);
            const bool spk = top && w > 0;
            const bool has_sep = top ? (w < P - 1) : true;
            const int pa = lay.a[w], pb = lay.b[w];
            if (top) {
                double accv = 0.0;
                for (int k = pa; k <= pb; ++k) {
                    double dc[7], lc[7], fc[7];
                    const int kn0 = k < pb ? k + 1 : (has_sep ? lay.s[w] : -1);
                    ld_inv(k, dc);
                    if (kn0 >= 0) ld_left(kn0, false, lc);
                    if (spk) ld_spike(k, true, fc);
                    l2_pf(k + QPF <= pb ? k + QPF : -1, k + QPF + 1 <= pb ? k + QPF + 1 : -1,
                          spk && k + QPF <= pb ? k + QPF : -1);
                    const int kn = k < pb ? k + 1 : (has_sep ? lay.s[w] : -1);
                    const double t = pair_dot7(dc, xv + NS * k, hh);
                    __syncwarp();
                    if (hh == 0 && rv) xv[NS * k + r] = t;
                    __syncwarp();
                    if (spk) {
                        double p = 0.0;
#pragma unroll
                        for (int q2 = 0; q2 < 7; ++q2) p = fma(fc[q2], xv[NS * k + 7 * hh + q2], p);
                        accv -= p;  // -F_k^T t_k, this lane's half
                    }
                    if (kn >= 0) {
                        const double u = pair_dot7(lc, xv + NS * k, hh);
                        if (hh == 0 && rv) {
                            if (k < pb) xv[NS * kn + r] += u;
                            else sacc[(2 * w) * NS + r] = u;
                        }
                    }
                    __syncwarp();
                }
                if (pb < pa && has_sep && lane < NS) sacc[(2 * w) * NS + lane] = 0.0;
                if (spk) {
                    accv += __shfl_xor_sync(0xffffffffu, accv, 1);
                    if (hh == 0 && rv) sacc[(2 * (w - 1) + 1) * NS + r] = accv;
                }
            } else {
                for (int k = pb; k >= pa; --k) {
                    double dc[7], lc[7];
                    ld_inv(k, dc);
                    ld_left(k, true, lc);
                    l2_pf(k - QPF >= pa ? k - QPF : -1, k - QPF >= pa ? k - QPF : -1, -1);
                    const double t = pair_dot7(dc, xv + NS * k, hh);
                    __syncwarp();
                    if (hh == 0 && rv) xv[NS * k + r] = t;
                    __syncwarp();
                    const double u = pair_dot7(lc, xv + NS * k, hh);
                    if (hh == 0 && rv) {
                        if (k > pa) xv[NS * (k - 1) + r] += u;
                        else sacc[(2 * (P - 2) + 1) * NS + r] = u;
                    }
                    __syncwarp();
                }
                if (pb < pa && lane < NS) sacc[(2 * (P - 2) + 1) * NS + lane] = 0.0;
            }
        }
        __syncthreads();
        // the reduced system (warp 0): forward t^_j, then x_{s_j} = t^_j - D^_j^{-1} E^_{j+1}^T x_{s_{j+1}}
        if (warp == 0 && P >= 2) {
            double *sc = fwall + PF_L;
            for (int j = 0; j < P - 1; ++j) {
                const int s = lay.s[j];
                double di[7];
                ld_inv(s, di);
                if (lane < NS) {
                    double z = (xv[NS * s + lane] + sacc[(2 * j) * NS + lane]) + sacc[(2 * j + 1) * NS + lane];
                    if (j > 0) {
                        const double *Eh = spall + (j - 1) * QSP;
                        const int sp = lay.s[j - 1];
#pragma unroll
                        for (int t = 0; t < NS; ++t) z = fma(-Eh[lane + NS * t], xv[NS * sp + t], z);
                    }
                    sc[lane] = z;
                }
                __syncwarp();
                const double t = pair_dot7(di, sc, hh);
                __syncwarp();
                if (hh == 0 && rv) xv[NS * s + r] = t;
                __syncwarp();
            }
            for (int j = P - 3; j >= 0; --j) {
                const int s = lay.s[j], sn = lay.s[j + 1];
                const double *Eh = spall + j * QSP;  // E^_{j+1}
                double di[7];
                ld_inv(s, di);
                if (lane < NS) {
                    double z = 0.0;
#pragma unroll
                    for (int t = 0; t < NS; ++t) z = fma(Eh[t + NS * lane], xv[NS * sn + t], z);
                    sc[lane] = z;
                }
                __syncwarp();
                const double u = pair_dot7(di, sc, hh);
                __syncwarp();
                if (hh == 0 && rv) xv[NS * s + r] -= u;
                __syncwarp();
            }
        }
        __syncthreads();
        // backward through every part: x_k = t_k + D_k^{-1} (coupling to the knots after it).  Step i of a
        // part (knot pb - i top-down, pa + i bottom-up) reads its inverse factor and coupling block from
        // a shared-memory slot filled by cp.async two steps earlier
        if (warp < P) {
            const int w = warp;
            const bool top = (w < P - 1) || (P == 1);
            const bool spk = top && w > 0;
            const bool has_sep = top ? (w < P - 1) : true;
            const int pa = lay.a[w], pb = lay.b[w];
            const int len = pb >= pa ? pb - pa + 1 : 0;
            double *sc = scw + w * NS;
            double *stg = fwall + w * QSTAGE * QSLOT;
            constexpr int LEFT_CHUNKS = SS * (int)sizeof(ST) / 16;
            auto knot_of = [&](int i) { return top ? pb - i : pa + i; };
            // the row whose left block step i needs (top-down: L_{k+1}, or the separator's; bottom-up: L_k)
            auto cpl_of = [&](int i) {
                const int k = knot_of(i);
                return top ? (k < pb ? k + 1 : (has_sep ? lay.s[w] : -1)) : k;
            };
            auto stage = [&](int i) {
                if (i < len) {
                    double *sl = stg + (i % QSTAGE) * QSLOT;
                    const int kl = cpl_of(i);
                    warp_cp_async(sl, wsb + (size_t)knot_of(i) * QW_STRIDE + PW_INV, QINV_D / 2, lane);
                    if (kl >= 0) warp_cp_async(sl + QINV_D, Sb + (size_t)kl * ks, LEFT_CHUNKS, lane);
                }
                cp_async_commit();
            };
            stage(0);
            stage(1);
            double fcn[7];  // middle part: row r of F_k of the next step (the term -F_k x_{s_{w-1}})
            if (spk && len > 0) ld_spike(knot_of(0), false, fcn);
            for (int i = 0; i < len; ++i) {
                stage(i + 2);
                {
                    const int ip = i + QPF < len ? i + QPF : -1, kp = ip >= 0 ? knot_of(ip) : -1;
                    l2_pf(kp, ip >= 0 ? cpl_of(ip) : -1, spk ? kp : -1);
                }
                cp_async_wait<QSTAGE - 1>();
                __syncwarp();
                const int k = knot_of(i), kl = cpl_of(i);
                const double *sl = stg + (i % QSTAGE) * QSLOT;
                const ST *sleft = reinterpret_cast<const ST *>(sl + QINV_D);
                double dc[7], lc[7];
#pragma unroll
                for (int q = 0; q < 7; ++q) {
                    dc[q] = rv ? sl[tri_lo(r, 7 * hh + q)] : 0.0;
                    lc[q] = (rv && kl >= 0) ? (double)sleft[top ? 7 * hh + q + NS * r : r + NS * (7 * hh + q)] : 0.0;
                }
                double v = 0.0;
                if (top) {
                    if (kl >= 0) v = pair_dot7(lc, xv + NS * kl, hh);  // L_{k+1}^T x_{k+1}
                    if (spk) {
                        double p = 0.0;
#pragma unroll
                        for (int q2 = 0; q2 < 7; ++q2) p = fma(fcn[q2], xv[NS * (pa - 1) + 7 * hh + q2], p);
                        v -= p + __shfl_xor_sync(0xffffffffu, p, 1);  // - F_k x_{s_{w-1}}
                        if (i + 1 < len) ld_spike(knot_of(i + 1), false, fcn);
                    }
                } else {
                    v = pair_dot7(lc, xv + NS * (k - 1), hh);  // L_k x_{k-1}
                }
                if (hh == 0 && rv) sc[r] = v;
                __syncwarp();
                const double a = pair_dot7(dc, sc, hh);
                if (hh == 0 && rv) xv[NS * k + r] += a;
                __syncwarp();
            }
            cp_async_wait<0>();
        }
        __syncthreads();
    };

    // ---- CG on the instance (the iteration of pcg_pair_kernel)
    int set = 0;
    auto block_sum = [&](double *v, int cnt) {
        for (int q = 0; q < cnt; ++q) {
            const double s = warp_sum(v[q]);
            if (lane == 0) red[set * QUAD_NWARP * 3 + warp * 3 + q] = s;
        }
        __syncthreads();
        for (int q = 0; q < cnt; ++q) {
            const double *rs = red + set * QUAD_NWARP * 3 + q;
            v[q] = ((rs[0] + rs[3]) + rs[6]) + rs[9];
        }
        set ^= 1;
    };
    auto true_residual = [&]() {
        __syncthreads();
        for (int e = tid; e < nv; e += QUAD_THREADS) xv[e] = wsv(PW_LAM, e);
        __syncthreads();
        for (int e = tid; e < nv; e += QUAD_THREADS) wsv(PW_RES, e) = gam(e) - srow(e, xv);
    };
    // z = S^{-1} r = -x of M x = r (left in xv); d[1] += r.z, d[2] += r.r.  The first call finds the
    // forward half done by the factorisation (y = r_0 = gamma)
    auto precond = [&](double *d, bool first) {
        if (!first) {
            __syncthreads();
            for (int e = tid; e < nv; e += QUAD_THREADS) xv[e] = wsv(PW_RES, e);
            __syncthreads();
        }
        solve(!first);
        for (int e = tid; e < nv; e += QUAD_THREADS) {
            const double rr = wsv(PW_RES, e), z = -xv[e];
            d[1] += rr * z;
            d[2] += rr * rr;
        }
    };
    auto sum_res2 = [&]() {
        double d0[1] = {0.0};
        for (int e = tid; e < nv; e += QUAD_THREADS) {
            const double rr = wsv(PW_RES, e);
            d0[0] += rr * rr;
        }
        block_sum(d0, 1);
        return d0[0];
    };
    auto converged = [&](double e, double r2) {
        return exit_mode == 0 ? (r2 <= (double)tol * (double)tol * gg) : (fabs(e) < (double)tol);
    };

    double eta;
    bool conv, bad = false;
    {
        double acc3[3] = {0.0, 0.0, 0.0};
        precond(acc3, true);
        block_sum(acc3, 3);
        eta = acc3[1];
        for (int e = tid; e < nv; e += QUAD_THREADS) wsv(PW_P, e) = -xv[e];  // p = z
        conv = converged(eta, acc3[2]);
    }
    int it = 0;
    while (!conv && it < max_iter) {
        __syncthreads();
        for (int e = tid; e < nv; e += QUAD_THREADS) xv[e] = wsv(PW_P, e);
        __syncthreads();
        double d1[1] = {0.0};
        // S p: warp w takes the knots w n / 4 .. (w + 1) n / 4 - 1 in order; each row of S (the left block
        // and the diagonal triangle) is staged in shared memory by cp.async, the next two rows in flight
        {
            const int kb = (warp * n) / QUAD_NWARP, ke = ((warp + 1) * n) / QUAD_NWARP;
            double *stg = fwall + warp * QSTAGE * QSLOT;
            constexpr int ROW_CHUNKS = (PK_DIAG + 105) * (int)sizeof(ST) / 16 + 1;  // left + triangle, rounded up
            static_assert(ROW_CHUNKS * 16 <= QSLOT * 8 && ROW_CHUNKS * 16 <= (FMT == 2 ? PK64 * 8 : PK * 4),
                          "a staged row fits its slot and its row of S");
            auto stage = [&](int i) {
                if (kb + i < n && i <= ke - kb) warp_cp_async(stg + (i % QSTAGE) * QSLOT, Sb + (size_t)(kb + i) * ks,
                                                             ROW_CHUNKS, lane);
                cp_async_commit();
            };
            stage(0);
            stage(1);
            for (int i = 0; i < ke - kb; ++i) {
                stage(i + 2);
                cp_async_wait<QSTAGE - 2>();  // the rows of knots k and k + 1 have landed
                __syncwarp();
                const int k = kb + i;
                const ST *row = reinterpret_cast<const ST *>(stg + (i % QSTAGE) * QSLOT);
                const ST *nxt = reinterpret_cast<const ST *>(stg + ((i + 1) % QSTAGE) * QSLOT);
                const bool hl = k > 0, hr = k < n - 1;
                double acc = 0.0;
                if (rv) {
#pragma unroll
                    for (int q = 0; q < 7; ++q) {
                        const int cc = 7 * hh + q;
                        if (hl) acc = fma((double)row[r + NS * cc], xv[NS * (k - 1) + cc], acc);
                        acc = fma((double)row[PK_DIAG + tri_lo(r, cc)], xv[NS * k + cc], acc);
                        if (hr) acc = fma((double)nxt[cc + NS * r], xv[NS * (k + 1) + cc], acc);
                    }
                }
                const double v1 = acc + __shfl_xor_sync(0xffffffffu, acc, 1);
                if (hh == 0 && rv) {
                    wsb[(size_t)k * QW_STRIDE + PW_V + r] = v1;
                    d1[0] = fma(xv[NS * k + r], v1, d1[0]);
                }
                __syncwarp();
            }
            cp_async_wait<0>();
        }
        block_sum(d1, 1);
        const double alpha = eta / d1[0];
        if (!isfinite(alpha)) {
            bad = true;
            break;
        }
        double r2acc = 0.0;
        for (int e = tid; e < nv; e += QUAD_THREADS) {
            wsv(PW_LAM, e) = fma(alpha, xv[e], wsv(PW_LAM, e));
            const double rn = fma(-alpha, wsv(PW_V, e), wsv(PW_RES, e));
            wsv(PW_RES, e) = rn;
            r2acc += rn * rn;
        }
        ++it;
        bool replaced = false;
        if (it % RR_PERIOD == 0) {
            true_residual();
            replaced = true;
        }
        if (exit_mode == 0) {
            double r2;
            if (replaced) {
                r2 = sum_res2();
            } else {
                double t1[1] = {r2acc};
                block_sum(t1, 1);
                r2 = t1[0];
            }
            if (!isfinite(r2)) {
                bad = true;
                break;
            }
            if (converged(0.0, r2) && !replaced && it > 1) {
                true_residual();
                r2 = sum_res2();
            }
            if (converged(0.0, r2)) {
                conv = true;
                break;
            }
        }
        double d2[3] = {0.0, 0.0, 0.0};
        precond(d2, false);
        block_sum(d2, 3);
        if (exit_mode != 0) conv = converged(d2[1], d2[2]);
        if (!isfinite(d2[1])) {
            bad = true;
            conv = false;
            break;
        }
        if (conv) break;
        const double beta = d2[1] / eta;
        eta = d2[1];
        for (int e = tid; e < nv; e += QUAD_THREADS) wsv(PW_P, e) = fma(beta, wsv(PW_P, e), -xv[e]);
    }
    for (int e = tid; e < nv; e += QUAD_THREADS) {
        const double lam = wsv(PW_LAM, e);
        lb[e] = (float)lam;
        if (lambda64) lambda64[NS * kg0 + e] = lam;
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
}

template <int FMT>
static cudaError_t launch_pcg_quad_t(const BatchView &bv, int max_n, const void *S, const float *gamma,
                                     const double *gamma64, float *lambda, double *lambda64, double *ws, int max_iter,
                                     float tol, int exit_mode, uint32_t *out_iters, uint32_t *pcg_log, int log_stride,
                                     cudaStream_t s)
{
    auto kern = pcg_quad_kernel<FMT>;
    const size_t smem = pcg_quad_smem_bytes(max_n);
    {
        const cudaError_t e = ensure_func_attrs((const void *)kern, smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<bv.B, QUAD_THREADS, smem, s>>>(bv, S, gamma, gamma64, lambda, lambda64, ws, max_iter, tol, exit_mode,
                                          out_iters, pcg_log, log_stride);
    return cudaGetLastError();
}

// FP64 packed rows (PK64: left block, diagonal lower triangle, pad) and FP64 gamma from the
// reference's FP32 3-block rows, for pcg_pair_kernel on a caller's S (gpt_pcg)
__global__ void pack_rows64_kernel(int N, const float *__restrict__ S, const float *__restrict__ gamma,
                                   double *__restrict__ S64, double *__restrict__ gamma64)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * PK64; i += gridDim.x * blockDim.x) {
        const int k = i / PK64, t = i - k * PK64;
        double v = 0.0;
        if (t < SS) {
            v = (double)S[(size_t)S_STRIDE * k + t];
        } else if (t < SS + 105) {
            const int q = t - SS;
            int rr = 0;
            while (((rr + 1) * (rr + 2)) / 2 <= q) ++rr;
            const int cc = q - (rr * (rr + 1)) / 2;
            v = (double)S[(size_t)S_STRIDE * k + SS + rr + NS * cc];
        }
        S64[i] = v;
        if (t < NS) gamma64[NS * k + t] = (double)gamma[NS * k + t];
    }
}

cudaError_t launch_pack_rows64(int N, const float *S, const float *gamma, double *S64, double *gamma64, int num_sms,
                               cudaStream_t s)
{
    int blocks = (N * PK64 + 255) / 256;
    if (blocks > 4 * num_sms) blocks = 4 * num_sms;
    pack_rows64_kernel<<<blocks, 256, 0, s>>>(N, S, gamma, S64, gamma64);
    return cudaGetLastError();
}

template <int FMT>
static cudaError_t launch_pcg_pair_t(const BatchView &bv, int max_n, const void *S, const float *gamma,
                                     const double *gamma64, float *lambda, double *lambda64, double *ws, int max_iter,
                                     float tol, int exit_mode, uint32_t *out_iters, uint32_t *pcg_log, int log_stride,
                                     cudaStream_t s)
{
    auto kern = pcg_pair_kernel<FMT>;
    const size_t smem = pcg_pair_smem_bytes(max_n);
    {
        const cudaError_t e = ensure_func_attrs((const void *)kern, smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<bv.B, PAIR_THREADS, smem, s>>>(bv, S, gamma, gamma64, lambda, lambda64, ws, max_iter, tol, exit_mode,
                                          out_iters, pcg_log, log_stride);
    return cudaGetLastError();
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

template <int CS, int FMT, int PRE = 0>
static cudaError_t launch_pcg_cs(const BatchView &bv, int kpc_max, const float *S, const float *Pinv,
                                 const float *gamma, float *lambda, double *lambda64, int max_iter, float tol,
                                 int exit_mode, uint32_t *out_iters, uint32_t *pcg_log, int log_stride, cudaStream_t s)
{
    auto kern = pcg_cluster_kernel<CS, FMT, PRE>;
    const size_t smem = pcg_cluster_smem_bytes(kpc_max, PRE == 2);
    {
        const cudaError_t e = ensure_func_attrs((const void *)kern, smem, CS > 8);
        if (e != cudaSuccess) return e;
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

template <int CS, int FMT>
static cudaError_t launch_pcg_chain_cs(const BatchView &bv, int kpc_max, const void *S, const float *gamma,
                                       const double *gamma64, float *lambda, double *lambda64, double *cr_ws,
                                       int max_iter, float tol, int exit_mode, uint32_t *out_iters, uint32_t *pcg_log,
                                       int log_stride, cudaStream_t s)
{
    auto kern = pcg_chain_kernel<CS, FMT>;
    const size_t smem = pcg_chain_smem_bytes(kpc_max);
    {
        const cudaError_t e = ensure_func_attrs((const void *)kern, smem, CS > 8);
        if (e != cudaSuccess) return e;
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
    return cudaLaunchKernelEx(&cfg, kern, bv, kpc_max, S, gamma, gamma64, lambda, lambda64, cr_ws, max_iter, tol,
                              exit_mode, out_iters, pcg_log, log_stride);
}

cudaError_t launch_pcg(const BatchView &bv, int max_n_knots, int min_n_knots, int fmt, int precond, const float *S,
                       const float *Pinv, const float *gamma, const double *gamma64, float *lambda,
                       double *lambda64, double *cr_ws, int max_iter, float tol, int exit_mode, uint32_t *out_iters,
                       uint32_t *pcg_log, int log_stride, int cluster_size, int num_sms, cudaStream_t s)
{
    if (bv.B <= 0) return cudaSuccess;
    if (precond == 1 && !cr_ws) return cudaErrorInvalidValue;
    if (fmt == 2 && (precond != 1 || !gamma64)) return cudaErrorInvalidValue;  // FP64 rows: chain preconditioner only
    if (max_n_knots > MAX_PCG_KNOTS) return cudaErrorInvalidValue;
    if (cluster_size == PCG_WARP_QUAD) {
        if (precond != 1 || fmt == 0) return cudaErrorInvalidValue;  // packed rows, exact preconditioner
        return fmt == 2 ? launch_pcg_quad_t<2>(bv, max_n_knots, S, gamma, gamma64, lambda, lambda64, cr_ws, max_iter,
                                               tol, exit_mode, out_iters, pcg_log, log_stride, s)
                        : launch_pcg_quad_t<1>(bv, max_n_knots, S, gamma, gamma64, lambda, lambda64, cr_ws, max_iter,
                                               tol, exit_mode, out_iters, pcg_log, log_stride, s);
    }
    if (cluster_size == PCG_WARP_PAIR) {
        if (precond != 1 || fmt == 0) return cudaErrorInvalidValue;  // packed rows, exact preconditioner
        return fmt == 2 ? launch_pcg_pair_t<2>(bv, max_n_knots, S, gamma, gamma64, lambda, lambda64, cr_ws, max_iter,
                                               tol, exit_mode, out_iters, pcg_log, log_stride, s)
                        : launch_pcg_pair_t<1>(bv, max_n_knots, S, gamma, gamma64, lambda, lambda64, cr_ws, max_iter,
                                               tol, exit_mode, out_iters, pcg_log, log_stride, s);
    }
    if (precond == 2 && fmt != 0) return cudaErrorInvalidValue;  // the stair Pinv comes in the reference layout
    const int kpc_cap = precond == 2 ? PCG_KPC_STAIR : PCG_KPC_MAX;
    int cs = (precond == 1 && cluster_size == 0) ? 1 : pcg_pick_cluster(max_n_knots, bv.B, num_sms, cluster_size);
    while ((max_n_knots + cs - 1) / cs > kpc_cap) cs *= 2;
    while (cs > 1 && cs > min_n_knots) cs /= 2;  // every CTA owns at least one knot
    const int kpc_max = (max_n_knots + cs - 1) / cs;
    if (kpc_max > kpc_cap || cs > 16) return cudaErrorInvalidValue;
#define GPT_PCG_CASE(CSV)                                                                                      \
    case CSV:                                                                                                  \
        if (precond == 1) {                                                                                    \
            if (fmt == 2)                                                                                      \
                return launch_pcg_chain_cs<CSV, 2>(bv, kpc_max, S, gamma, gamma64, lambda, lambda64, cr_ws,    \
                                                   max_iter, tol, exit_mode, out_iters, pcg_log, log_stride, s); \
            return fmt ? launch_pcg_chain_cs<CSV, 1>(bv, kpc_max, S, gamma, gamma64, lambda, lambda64, cr_ws,  \
                                                     max_iter, tol, exit_mode, out_iters, pcg_log, log_stride, s) \
                       : launch_pcg_chain_cs<CSV, 0>(bv, kpc_max, S, gamma, gamma64, lambda, lambda64, cr_ws,  \
                                                     max_iter, tol, exit_mode, out_iters, pcg_log, log_stride, s); \
        }                                                                                                      \
        if (precond == 2)                                                                                      \
            return launch_pcg_cs<CSV, 0, 2>(bv, kpc_max, S, Pinv, gamma, lambda, lambda64, max_iter, tol,      \
                                            exit_mode, out_iters, pcg_log, log_stride, s);                     \
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
