// gpt_schur.cu -- Schur complement, block-Jacobi preconditioner and the CSC
// values of the Schur matrix: one warp per block row.
//
// Replaces gato_form_schur_jacobi / gato_form_schur_jacobi_inner
// (schur.cuh:12-54, oldschur.cuh:518-963) and form_schur_qdl_kernel
// (schur.cuh:57-383 with store_block_csr_lowertri, utils.cuh:55-81).
//
// Block row k >= 1 (A, B = dynamics Jacobians of knot k-1; C stores -A, -B):
//   phi_k   = (-A) Qt_{k-1}^{-1}                     Qt = Q + rho I, Rt = R + rho I
//   theta_k = phi_k (-A)^T + Qt_k^{-1} + (-B) Rt^{-1} (-B)^T
//   gamma_k = Qt_k^{-1} q_k - c_k + phi_k q_{k-1} + (-B) Rt^{-1} r_{k-1}
//   S[k] = [-phi_k, -theta_k, .], S[k-1].right = -phi_k^T,
//   Pinv[k].diag = -theta_k^{-1}, gamma_out[k] = -gamma_k
// Block row 0: S[0].diag = -Qt_0^{-1}, Pinv[0].diag = -Qt_0, gamma_out[0] = -Qt_0^{-1} q_0.
// Inverses (Qt, Rt, theta) are Gauss-Jordan in FP64 with the augmented
// columns spread over the lanes; the products are FP32 from shared memory.
// The inverses Qt_k^{-1}, Rt_k^{-1} go to a separate Ginv buffer (the
// reference overwrites G in place, which races with the neighbouring block's
// read of the same slot, oldschur.cuh:700 vs :751).
#include "gpt_common.cuh"
#include "gpt_internal.h"

namespace gpt {

// FP64 Gauss-Jordan inverse of the n x n matrix (A + shift I) held column-major
// in A (global or shared).  Lanes 0..2n-1 hold the columns of [A | I]; the
// inverse is written column-major (float) to Ainv.
template <int n>
__device__ __forceinline__ void warp_inverse(const float *A, float shift, float *Ainv, int lane,
                                             double *Ainv64 = nullptr)
{
    double col[n];
    const bool left = lane < n, right = (lane >= n) && (lane < 2 * n);
#pragma unroll
    for (int r = 0; r < n; ++r) {
        double v = 0.0;
        if (left) v = (double)A[r + n * lane] + ((r == lane) ? (double)shift : 0.0);
        else if (right) v = (r == lane - n) ? 1.0 : 0.0;
        col[r] = v;
    }
    // pivot p: the pivot element first, then each row's element of the pivot column is
    // broadcast just before it is used, so only the 14 column entries stay live
#pragma unroll
    for (int p = 0; p < n; ++p) {
        const double piv = __shfl_sync(0xffffffffu, col[p], p);
        const double prow = col[p] * __drcp_rn(piv);  // correctly rounded reciprocal: ~3x less latency than a divide
#pragma unroll
        for (int r = 0; r < n; ++r) {
            if (r == p) continue;
            const double pr = __shfl_sync(0xffffffffu, col[r], p);
            col[r] = fma(-pr, prow, col[r]);
        }
        col[p] = prow;
    }
    if (right) {
#pragma unroll
        for (int r = 0; r < n; ++r) Ainv[r + n * (lane - n)] = (float)col[r];
        if (Ainv64) {
#pragma unroll
            for (int r = 0; r < n; ++r) Ainv64[r + n * (lane - n)] = col[r];
        }
    }
}

// out (14 x NCOL, col-major) = A (14 x K, col-major) * op(B)
//   op(B) = B (K x NCOL, ld 14 or 7) or B^T with B (NCOL x K, ld 14)
template <int K, int NCOL, bool TRANS_B>
__device__ __forceinline__ void warp_mm(const float *A, const float *B, int ldb, float *out, int lane)
{
    if (lane < 2 * NCOL) {
        const int col = lane % NCOL, r0 = (lane / NCOL) * 7;
        float acc[7];
#pragma unroll
        for (int i = 0; i < 7; ++i) acc[i] = 0.f;
#pragma unroll
        for (int t = 0; t < K; ++t) {
            const float bv = TRANS_B ? B[col + ldb * t] : B[t + ldb * col];
#pragma unroll
            for (int i = 0; i < 7; ++i) acc[i] = fmaf(A[r0 + i + NS * t], bv, acc[i]);
        }
#pragma unroll
        for (int i = 0; i < 7; ++i) out[r0 + i + NS * col] = acc[i];
    }
}

struct SchurWarpSmem {
    float A[SS], B[SC];
    float Qki[SS], Qkp1i[SS], Rki[CC];
    float phi[SS], BRi[SC], theta[SS], tmp[SS], thetai[SS];
    float qk[NS], qkp1[NS], rk[NC], ck[NS];
};

constexpr int SCHUR_WARPS = 4;

// MODE 0: S, Pinv (reference 3-block layout, off-diagonal Pinv blocks zero), gamma, Ginv
// MODE 1: packed rows for the PCG (PK = 408 floats per knot: left block, lower
//         triangle of the diagonal block, lower triangle of Pinv, 2 pad), gamma, Ginv
// MODE 2: CSC values of the upper triangle (utils.cuh:55-118 layout), gamma, Ginv
template <int MODE>
__global__ void __launch_bounds__(32 * SCHUR_WARPS)
    schur_kernel(BatchView bv, float rho_scalar, const float *__restrict__ G,
                 const float *__restrict__ Cm, const float *__restrict__ g, const float *__restrict__ c,
                 float *__restrict__ S, float *__restrict__ Pinv, float *__restrict__ gamma,
                 float *__restrict__ Ginv, double *__restrict__ Ginv64, float *__restrict__ csc_val, int need_pinv)
{
    extern __shared__ float4 schur_dyn_smem[];
    SchurWarpSmem *smem_all = reinterpret_cast<SchurWarpSmem *>(schur_dyn_smem);
    const int lane = threadIdx.x & 31;
    SchurWarpSmem &sm = smem_all[threadIdx.x >> 5];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;

    for (int j = bv.j0 + gw; j < bv.j0 + bv.total_knots; j += nw) {
        const int b = bv.inst(j);
        if (!bv.active(b)) continue;
        const int N = bv.N(b);
        const int k = j - bv.off(b);
        const float rho = bv.st ? bv.st[b].rho : rho_scalar;
        float *Srow = (MODE == 0) ? S + (size_t)S_STRIDE * j : nullptr;

        if (k == 0) {
            const float *Q0 = G + (size_t)G_STRIDE * j;
            warp_inverse<NS>(Q0, rho, sm.Qki, lane, (N == 1 && Ginv64) ? Ginv64 + (size_t)G_STRIDE * j : nullptr);
            if (lane < NS) sm.qk[lane] = g[(size_t)NX * j + lane];
            __syncwarp();
            if (lane < NS) {
                float acc = 0.f;
#pragma unroll
                for (int t = 0; t < NS; ++t) acc = fmaf(sm.Qki[lane + NS * t], sm.qk[t], acc);
                gamma[(size_t)NS * j + lane] = -acc;
            }
            for (int e = lane; e < SS; e += 32) {
                const float qv = Q0[e] + ((e % (NS + 1)) == 0 ? rho : 0.f);
                if (MODE == 0) {
                    Pinv[(size_t)S_STRIDE * j + e] = 0.f;
                    Pinv[(size_t)S_STRIDE * j + SS + e] = -qv;
                    Srow[e] = 0.f;
                    Srow[SS + e] = -sm.Qki[e];
                } else if (MODE == 1) {
                    float *Pk = S + (size_t)PK * j;
                    const int r = e % NS, cc = e / NS;
                    Pk[e] = 0.f;  // no left block in row 0
                    if (r >= cc) {
                        const int t = ((r * (r + 1)) >> 1) + cc;
                        Pk[SS + t] = -sm.Qki[e];
                        Pk[SS + 105 + t] = -qv;
                    }
                    if (e < PK - SS - 210) Pk[SS + 210 + e] = 0.f;
                }
                if (N == 1) Ginv[(size_t)G_STRIDE * j + e] = sm.Qki[e];
            }
            if (MODE == 2) {
                // first block row: lower triangle of -Qt_0^{-1}, row r holds cols 0..r
                const size_t base = 0;
                for (int e = lane; e < SS; e += 32) {
                    const int r = e / NS, cc = e - NS * r;
                    if (cc <= r) csc_val[base + (r * (r + 1)) / 2 + cc] = -sm.Qki[r + NS * cc];
                }
            }
            if (MODE == 0) {
                for (int e = lane; e < SS; e += 32) {
                    Pinv[(size_t)S_STRIDE * j + 2 * SS + e] = 0.f;
                    if (N == 1) Srow[2 * SS + e] = 0.f;
                }
            }
            __syncwarp();
            continue;
        }

        // ---- rows k >= 1
        const float *Ck = Cm + (size_t)C_STRIDE * (j - 1);
        for (int e = lane; e < C_STRIDE; e += 32) {
            const float v = Ck[e];
            if (e < SS) sm.A[e] = v;
            else sm.B[e - SS] = v;
        }
        if (lane < NS) {
            sm.qk[lane] = g[(size_t)NX * (j - 1) + lane];
            sm.qkp1[lane] = g[(size_t)NX * j + lane];
            sm.ck[lane] = c[(size_t)NS * j + lane];
        } else if (lane < NS + NC) {
            sm.rk[lane - NS] = g[(size_t)NX * (j - 1) + lane];
        }
        const float *Gkm1 = G + (size_t)G_STRIDE * (j - 1);
        const float *Gk = G + (size_t)G_STRIDE * j;
        double *G64m1 = Ginv64 ? Ginv64 + (size_t)G_STRIDE * (j - 1) : nullptr;
        warp_inverse<NS>(Gkm1, rho, sm.Qki, lane, G64m1);
        warp_inverse<NS>(Gk, rho, sm.Qkp1i, lane, (Ginv64 && k == N - 1) ? Ginv64 + (size_t)G_STRIDE * j : nullptr);
        warp_inverse<NC>(Gkm1 + SS, rho, sm.Rki, lane, G64m1 ? G64m1 + SS : nullptr);
        __syncwarp();
        // Ginv slots (schur.cuh:236-256): Qt_{k-1}^{-1}, Rt_{k-1}^{-1}; the last row also Qt_{N-1}^{-1}
        {
            float *Gi = Ginv + (size_t)G_STRIDE * (j - 1);
            for (int e = lane; e < G_STRIDE; e += 32) Gi[e] = (e < SS) ? sm.Qki[e] : sm.Rki[e - SS];
            if (k == N - 1) {
                float *Gl = Ginv + (size_t)G_STRIDE * j;
                for (int e = lane; e < SS; e += 32) Gl[e] = sm.Qkp1i[e];
            }
        }
        warp_mm<NS, NS, false>(sm.A, sm.Qki, NS, sm.phi, lane);   // phi = (-A) Qt^{-1}
        warp_mm<NC, NC, false>(sm.B, sm.Rki, NC, sm.BRi, lane);   // (-B) Rt^{-1}
        __syncwarp();
        warp_mm<NS, NS, true>(sm.phi, sm.A, NS, sm.theta, lane);  // phi (-A)^T
        warp_mm<NC, NS, true>(sm.BRi, sm.B, NS, sm.tmp, lane);    // (-B) Rt^{-1} (-B)^T
        if (lane < NS) {
            float a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                a1 = fmaf(sm.Qkp1i[lane + NS * t], sm.qkp1[t], a1);
                a2 = fmaf(sm.phi[lane + NS * t], sm.qk[t], a2);
            }
#pragma unroll
            for (int t = 0; t < NC; ++t) a3 = fmaf(sm.BRi[lane + NS * t], sm.rk[t], a3);
            gamma[(size_t)NS * j + lane] = -((a1 - sm.ck[lane]) + (a3 + a2));
        }
        __syncwarp();
        for (int e = lane; e < SS; e += 32) sm.theta[e] = (sm.theta[e] + sm.Qkp1i[e]) + sm.tmp[e];
        __syncwarp();
        if (MODE == 0 || need_pinv) warp_inverse<NS>(sm.theta, 0.f, sm.thetai, lane);
        __syncwarp();
        if (MODE == 0) {
            float *Sprev_right = S + (size_t)S_STRIDE * (j - 1) + 2 * SS;
            for (int e = lane; e < SS; e += 32) {
                const int r = e % NS, cc = e / NS;
                Srow[e] = -sm.phi[e];
                Srow[SS + e] = -sm.theta[e];
                Sprev_right[e] = -sm.phi[cc + NS * r];
                Pinv[(size_t)S_STRIDE * j + e] = 0.f;
                Pinv[(size_t)S_STRIDE * j + SS + e] = -sm.thetai[e];
                Pinv[(size_t)S_STRIDE * j + 2 * SS + e] = 0.f;
                if (k == N - 1) Srow[2 * SS + e] = 0.f;
            }
        } else if (MODE == 1) {
            // packed row: left block, lower triangles of the diagonal block and of Pinv
            float *Pk = S + (size_t)PK * j;
            for (int e = lane; e < SS; e += 32) {
                const int r = e % NS, cc = e / NS;
                Pk[e] = -sm.phi[e];
                if (r >= cc) {
                    const int t = ((r * (r + 1)) >> 1) + cc;
                    Pk[SS + t] = -sm.theta[e];
                    Pk[SS + 105 + t] = need_pinv ? -sm.thetai[e] : 0.f;
                }
                if (e < PK - SS - 210) Pk[SS + 210 + e] = 0.f;
            }
        } else {
            // block row k of the CSC (utils.cuh:55-81): row r holds 14 left entries then r+1 diagonal entries
            const int tri = (NS + 1) * NS / 2, brow = SS + tri;
            const size_t base = (size_t)tri + (size_t)(k - 1) * brow;
            for (int e = lane; e < SS; e += 32) {
                const int r = e / NS, cc = e - NS * r;
                const size_t off = base + (size_t)r * NS + (r * (r + 1)) / 2;
                csc_val[off + cc] = -sm.phi[r + NS * cc];
                if (cc <= r) csc_val[off + NS + cc] = -sm.theta[r + NS * cc];
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// FP64 formation for the cyclic-reduction PCG: the same block row as MODE 1,
// with every product, gamma and the stored row in FP64 (PK64 doubles per knot:
// left block 196 column-major, lower triangle of the diagonal block 105, pad).
// FP32 formation perturbs S by ~10 eps32 relative per entry, which cond(S)
// ~1e7 turns into ~1e-2 relative error of the solution; FP64 formation leaves
// only the FP32 rounding of the KKT data (G, C, g, c).
// ---------------------------------------------------------------------------

// Pivot test of the Schur complement's inverses: (Q + rho I) and (R + rho I) must be positive
// definite, so every Gauss-Jordan pivot must be positive and not vanish against the diagonal entry it
// came from (a relative 1e-13 catches a singular matrix whose exact zero pivot rounding turned into a
// tiny number of either sign; NaN fails too)
constexpr double PIVOT_REL_MIN = 1e-13;

// FP64 Gauss-Jordan inverse of the n x n matrix (A + shift I), A column-major with leading
// dimension LD; the inverse goes column-major with leading dimension LD to Ainv (and, when given,
// Ainv32 / Ainv64g).  Returns false (on every lane) if a pivot failed the test above.
template <int n, int LD = n>
__device__ __forceinline__ bool warp_inverse64(const float *A, double shift, double *Ainv, int lane,
                                               float *Ainv32, double *Ainv64g)
{
    double col[n];
    double diag_own = 0.0;  // lane p < n: the diagonal entry (p, p) of A + shift I
    const bool left = lane < n, right = (lane >= n) && (lane < 2 * n);
#pragma unroll
    for (int r = 0; r < n; ++r) {
        double v = 0.0;
        if (left) v = (double)A[r + LD * lane] + ((r == lane) ? shift : 0.0);
        else if (right) v = (r == lane - n) ? 1.0 : 0.0;
        col[r] = v;
        if (left && r == lane) diag_own = v;
    }
    bool ok = true;
#pragma unroll
    for (int p = 0; p < n; ++p) {
        const double piv = __shfl_sync(0xffffffffu, col[p], p);
        const double d0 = __shfl_sync(0xffffffffu, diag_own, p);
        ok = ok && (piv > PIVOT_REL_MIN * d0) && (d0 > 0.0);
        const double prow = col[p] * __drcp_rn(piv);
#pragma unroll
        for (int r = 0; r < n; ++r) {
            if (r == p) continue;
            const double pr = __shfl_sync(0xffffffffu, col[r], p);
            col[r] = fma(-pr, prow, col[r]);
        }
        col[p] = prow;
    }
    if (right) {
        const int cc = lane - n;
#pragma unroll
        for (int r = 0; r < n; ++r) Ainv[r + LD * cc] = col[r];
        if (Ainv32) {
#pragma unroll
            for (int r = 0; r < n; ++r) Ainv32[r + LD * cc] = (float)col[r];
        }
        if (Ainv64g) {
#pragma unroll
            for (int r = 0; r < n; ++r) Ainv64g[r + LD * cc] = col[r];
        }
    }
    return ok;
}

// FP64 inverse of the 7x7 position block (A + shift I) of a state block (A column-major with leading
// dimension LD), by Gauss-Jordan with 2x2 block pivots {0,1}, {2,3}, {4,5} and the scalar pivot 6
// (no pivoting: the blocks are diagonal blocks of Schur complements of an SPD matrix).  Lanes 0..6 hold
// A's columns, lanes 7..13 the identity's; a 2x2 step needs the block's three entries and the two pivot
// columns' rows (shuffles), and one reciprocal of its determinant, so the chain of dependent steps is
// four long instead of seven.  The pivot test is the scalar elimination's, pivot by pivot: x > 1e-13 d_p
// and det / x > 1e-13 d_{p+1} (d the entries of A + shift I's diagonal).  Lanes 7..13 write the inverse.
template <int LD>
__device__ __forceinline__ bool warp_inverse64_pos7(const float *A, double shift, double *Ainv, int lane,
                                                    float *Ainv32, double *Ainv64g)
{
    constexpr int n = NC;
    double col[n];
    double diag_own = 0.0;
    const bool left = lane < n, right = (lane >= n) && (lane < 2 * n);
#pragma unroll
    for (int r = 0; r < n; ++r) {
        double v = 0.0;
        if (left) v = (double)A[r + LD * lane] + ((r == lane) ? shift : 0.0);
        else if (right) v = (r == lane - n) ? 1.0 : 0.0;
        col[r] = v;
        if (left && r == lane) diag_own = v;
    }
    bool ok = true;
#pragma unroll
    for (int p = 0; p + 1 < n; p += 2) {
        const double x = __shfl_sync(0xffffffffu, col[p], p);
        const double y = __shfl_sync(0xffffffffu, col[p + 1], p);
        const double z = __shfl_sync(0xffffffffu, col[p + 1], p + 1);
        const double d0 = __shfl_sync(0xffffffffu, diag_own, p), d1 = __shfl_sync(0xffffffffu, diag_own, p + 1);
        double pr0[n], pr1[n];  // rows r of the pivot columns p, p + 1
#pragma unroll
        for (int r = 0; r < n; ++r) {
            if (r == p || r == p + 1) continue;
            pr0[r] = __shfl_sync(0xffffffffu, col[r], p);
            pr1[r] = __shfl_sync(0xffffffffu, col[r], p + 1);
        }
        const double det = fma(x, z, -y * y);
        ok = ok && (d0 > 0.0) && (d1 > 0.0) && (x > PIVOT_REL_MIN * d0) && (det > PIVOT_REL_MIN * d1 * x);
        const double rd = __drcp_rn(det);
        const double i00 = z * rd, i01 = -y * rd, i11 = x * rd;
        const double w0 = col[p], w1 = col[p + 1];
        const double n0 = fma(i00, w0, i01 * w1), n1 = fma(i01, w0, i11 * w1);
#pragma unroll
        for (int r = 0; r < n; ++r) {
            if (r == p || r == p + 1) continue;
            col[r] = fma(-pr0[r], n0, fma(-pr1[r], n1, col[r]));
        }
        col[p] = n0;
        col[p + 1] = n1;
    }
    {
        constexpr int p = n - 1;
        const double piv = __shfl_sync(0xffffffffu, col[p], p);
        const double d0 = __shfl_sync(0xffffffffu, diag_own, p);
        ok = ok && (d0 > 0.0) && (piv > PIVOT_REL_MIN * d0);
        double pr[n];
#pragma unroll
        for (int r = 0; r < p; ++r) pr[r] = __shfl_sync(0xffffffffu, col[r], p);
        const double prow = col[p] * __drcp_rn(piv);
#pragma unroll
        for (int r = 0; r < p; ++r) col[r] = fma(-pr[r], prow, col[r]);
        col[p] = prow;
    }
    if (right) {
        const int cc = lane - n;
#pragma unroll
        for (int r = 0; r < n; ++r) Ainv[r + LD * cc] = col[r];
        if (Ainv32) {
#pragma unroll
            for (int r = 0; r < n; ++r) Ainv32[r + LD * cc] = (float)col[r];
        }
        if (Ainv64g) {
#pragma unroll
            for (int r = 0; r < n; ++r) Ainv64g[r + LD * cc] = col[r];
        }
    }
    return ok;
}

// (Q + shift I)^{-1} of a 14x14 state block.  The blocks kkt_kernel writes are block diagonal --
// a 7x7 position block (q q^T), a diagonal velocity block (QD) -- and then the inverse is the
// position block's inverse (warp_inverse64_pos7) and the reciprocals of the velocity diagonal (lanes
// 0..6, one each); any other Q takes the full 14x14 elimination.  The structure test reads every
// entry outside the blocks without branching on the running result (the loads issue together).
// *blockdiag (optional) tells which path ran: true when the inverse has that block-diagonal zero pattern.
__device__ __forceinline__ bool warp_inverse64_state(const float *Q, double shift, double *Ainv, int lane,
                                                     float *Ainv32, double *Ainv64g, bool *blockdiag = nullptr)
{
    bool ok = true;
#pragma unroll
    for (int i = 0; i < (SS + 31) / 32; ++i) {
        const int e = lane + 32 * i;
        const int r = e % NS, cc = e / NS;
        const bool outside = (e < SS) && (((r < NC) != (cc < NC)) || (r >= NC && cc >= NC && r != cc));
        ok &= !outside || (Q[e < SS ? e : 0] == 0.f);
    }
    const bool bd = __all_sync(0xffffffffu, ok);
    if (blockdiag) *blockdiag = bd;
    if (!bd) return warp_inverse64<NS>(Q, shift, Ainv, lane, Ainv32, Ainv64g);
    bool piv_ok = warp_inverse64_pos7<NS>(Q, shift, Ainv, lane, Ainv32, Ainv64g);
    if (lane < NC) {
        const int e = (NC + lane) * (NS + 1);
        const double d = (double)Q[e] + shift;
        piv_ok = piv_ok && (d > 0.0);
        const double v = __drcp_rn(d);
        Ainv[e] = v;
        if (Ainv32) Ainv32[e] = (float)v;
        if (Ainv64g) Ainv64g[e] = v;
    }
    for (int e = lane; e < SS; e += 32) {
        const int r = e % NS, cc = e / NS;
        if ((r < NC && cc < NC) || r == cc) continue;
        Ainv[e] = 0.0;
        if (Ainv32) Ainv32[e] = 0.f;
        if (Ainv64g) Ainv64g[e] = 0.0;
    }
    return __all_sync(0xffffffffu, piv_ok);
}
// (R + shift I)^{-1} of a 7x7 control block: reciprocals when R is diagonal (kkt_kernel's R_COST I;
// the same arithmetic as the elimination), else Gauss-Jordan
// *diagonal (optional): true when R was diagonal (and so is the inverse).
__device__ __forceinline__ bool warp_inverse64_control(const float *R, double shift, double *Ainv, int lane,
                                                       float *Ainv32, double *Ainv64g, bool *diagonal = nullptr)
{
    bool ok = true;
#pragma unroll
    for (int i = 0; i < (CC + 31) / 32; ++i) {
        const int e = lane + 32 * i;
        const bool off = (e < CC) && (e % NC != e / NC);
        ok &= !off || (R[e < CC ? e : 0] == 0.f);
    }
    const bool dg = __all_sync(0xffffffffu, ok);
    if (diagonal) *diagonal = dg;
    if (!dg) return warp_inverse64<NC>(R, shift, Ainv, lane, Ainv32, Ainv64g);
    bool piv_ok = true;
    if (lane < NC) {
        const int e = lane * (NC + 1);
        const double d = (double)R[e] + shift;
        piv_ok = d > 0.0;
        const double v = __drcp_rn(d);
        Ainv[e] = v;
        if (Ainv32) Ainv32[e] = (float)v;
        if (Ainv64g) Ainv64g[e] = v;
    }
    for (int e = lane; e < CC; e += 32) {
        if (e % NC == e / NC) continue;
        Ainv[e] = 0.0;
        if (Ainv32) Ainv32[e] = 0.f;
        if (Ainv64g) Ainv64g[e] = 0.0;
    }
    return __all_sync(0xffffffffu, piv_ok);
}

// A knot's FP64 inverses for dz, from shared memory (Qi: 14 x 14, Ri: 7 x 7 or null for an
// instance's last knot), as GC64 contiguous doubles (two stores per lane) plus, only for a block
// that is not (block) diagonal, that block in the full layout (G_STRIDE doubles per knot).
__device__ __forceinline__ void write_ginv_compact(double *dc, double *dfull, const double *Qi, const double *Ri,
                                                   bool q_bd, bool r_dg, int lane)
{
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int e = lane + 32 * h;
        double v;
        if (e == 0) {
            v = (q_bd ? 0.0 : 1.0) + (r_dg ? 0.0 : 2.0);
        } else if (e < GC_VEL) {
            const int i = e - GC_POS;
            v = Qi[i % NC + NS * (i / NC)];
        } else if (e < GC_CTL) {
            v = Qi[(NC + e - GC_VEL) * (NS + 1)];
        } else {
            v = Ri ? Ri[(e - GC_CTL) * (NC + 1)] : 0.0;
        }
        dc[e] = v;
    }
    if (!q_bd)
        for (int e = lane; e < SS; e += 32) dfull[e] = Qi[e];
    if (Ri && !r_dg)
        for (int e = lane; e < CC; e += 32) dfull[SS + e] = Ri[e];
}

// One warp's shared memory: the knot's KKT blocks staged as FP32 (one batch of loads per knot), the
// FP64 inverses and products
struct Schur64WarpSmem {
    double Qinv[2][SS], Rki[CC];  // (Q_{k-1} + rho I)^{-1} and (Q_k + rho I)^{-1}, roles alternating along a run
    double phi[SS], BRi[SC], theta[SS];
    double qk[NS], qkp1[NS], rk[NC], ck[NS];
    float Gm1[G_STRIDE], Gk[SS], C[C_STRIDE];
};

// Five CTAs per SM: the shared-memory limit (43 KB per CTA); the registers fit without spilling.
__global__ void __launch_bounds__(32 * SCHUR_WARPS, 5)
    schur64_kernel(BatchView bv, const float *__restrict__ G, const float *__restrict__ Cm,
                   const float *__restrict__ g, const float *__restrict__ c, double *__restrict__ S64,
                   double *__restrict__ gamma64, float *__restrict__ Ginv, double *__restrict__ Ginv64,
                   double *__restrict__ Ginv64c)
{
    extern __shared__ double4 schur64_dyn_smem[];
    Schur64WarpSmem *smem_all = reinterpret_cast<Schur64WarpSmem *>(schur64_dyn_smem);
    const int lane = threadIdx.x & 31;
    Schur64WarpSmem &sm = smem_all[threadIdx.x >> 5];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;

    // Each warp takes a contiguous run of knots, so the inverse (Q_k + rho I)^{-1} that row k forms
    // for its diagonal block serves row k + 1 as (Q_{k} + rho I)^{-1} again instead of being formed
    // twice (the same function of the same inputs: identical bits).
    const int chunk = (bv.total_knots + nw - 1) / nw;
    const int jbeg = bv.j0 + gw * chunk;
    const int jend = min(jbeg + chunk, bv.j0 + bv.total_knots);
    bool pref = false;     // this row's R_{k-1}, Q_k and C_{k-1} arrived by cp.async during the previous row
    int have = -1;         // knot whose inverse sm.Qinv[cur] holds
    int cur = 0;
    bool have_bd = false;  // that inverse is block diagonal (position block, diagonal velocity block)
    for (int j = jbeg; j < jend; ++j) {
        const int b = bv.inst(j);
        if (!bv.active(b)) {
            have = -1;
            continue;
        }
        const int N = bv.N(b);
        const int k = j - bv.off(b);
        const double rho = (double)bv.st[b].rho;
        double *Pk = S64 + (size_t)PK64 * j;

        if (k == 0) {
            double *Q0i = sm.Qinv[cur];
            const float *Q0 = G + (size_t)G_STRIDE * j;
            for (int e = lane; e < SS; e += 32) sm.Gk[e] = Q0[e];
            if (lane < NS) sm.qk[lane] = (double)g[(size_t)NX * j + lane];
            __syncwarp();
            const bool ok0 = warp_inverse64_state(sm.Gk, rho, Q0i, lane,
                                                  (N == 1 && Ginv) ? Ginv + (size_t)G_STRIDE * j : nullptr,
                                                  nullptr, &have_bd);
            if (!ok0 && lane == 0) atomicOr(&bv.st[b].exit_flags, GPT_EXIT_FACTOR);
            __syncwarp();
            if (N == 1)
                write_ginv_compact(Ginv64c + (size_t)GC64 * j, Ginv64 + (size_t)G_STRIDE * j, Q0i, nullptr, have_bd,
                                   true, lane);
            if (lane < NS) {
                double acc = 0.0;
#pragma unroll
                for (int t = 0; t < NS; ++t) acc = fma(Q0i[lane + NS * t], sm.qk[t], acc);
                gamma64[(size_t)NS * j + lane] = -acc;
            }
            for (int e = lane; e < SS; e += 32) {
                const int r = e % NS, cc = e / NS;
                Pk[e] = 0.0;  // no left block in row 0
                if (r >= cc) Pk[SS + ((r * (r + 1)) >> 1) + cc] = -Q0i[e];
            }
            if (lane == 0) Pk[PK64 - 1] = 0.0;
            __syncwarp();
            have = j;
            continue;
        }

        // ---- rows k >= 1: every input of the knot loaded in one batch, then staged.  Q_{k-1} is needed
        // only to invert it, which the previous row of a run did already (have == j - 1): then its 196
        // entries are not loaded
        const bool reuse = have == j - 1;
        {
            if (!pref) {
                // this row's blocks were not copied ahead (the first row of a run, or of an instance
                // inside it): copy them now; Q_{k-1} only when the run's previous row did not invert it
                const float *Gkm1 = G + (size_t)G_STRIDE * (j - 1);
                const float *Gkq = G + (size_t)G_STRIDE * j;
                const float *Ck = Cm + (size_t)C_STRIDE * (j - 1);
                for (int e = reuse ? SS + lane : lane; e < G_STRIDE; e += 32) cp_async4(sm.Gm1 + e, Gkm1 + e);
                for (int e = lane; e < SS; e += 32) cp_async4(sm.Gk + e, Gkq + e);
                for (int e = lane; e < C_STRIDE; e += 32) cp_async4(sm.C + e, Ck + e);
                cp_async_commit();
            }
            double gv = 0.0;
            if (lane < NX) gv = (double)g[(size_t)NX * (j - 1) + lane];
            double g2 = 0.0, cv = 0.0;
            if (lane < NS) {
                g2 = (double)g[(size_t)NX * j + lane];
                cv = (double)c[(size_t)NS * j + lane];
            }
            cp_async_wait<0>();  // this row's blocks (copied now, or during the previous row)
            if (lane < NS) {
                sm.qk[lane] = gv;
                sm.qkp1[lane] = g2;
                sm.ck[lane] = cv;
            } else if (lane < NX) {
                sm.rk[lane - NS] = gv;
            }
        }
        __syncwarp();
        float *Gi32 = Ginv ? Ginv + (size_t)G_STRIDE * (j - 1) : nullptr;
        double *const Qki = sm.Qinv[cur], *const Qkp1i = sm.Qinv[cur ^ 1];
        bool ok = true, bd_ki = have_bd, bd_kp1 = false, r_diag = false;
        if (reuse) {
            // formed by this warp's previous row; its FP32 copy for knot j - 1 is written here, as the
            // elimination below would
            if (Gi32)
                for (int e = lane; e < SS; e += 32) Gi32[e] = (float)Qki[e];
        } else {
            ok = warp_inverse64_state(sm.Gm1, rho, Qki, lane, Gi32, nullptr, &bd_ki);
        }
        ok = warp_inverse64_state(sm.Gk, rho, Qkp1i, lane, (k == N - 1 && Ginv) ? Ginv + (size_t)G_STRIDE * j : nullptr,
                                  nullptr, &bd_kp1) && ok;
        ok = warp_inverse64_control(sm.Gm1 + SS, rho, sm.Rki, lane, Gi32 ? Gi32 + SS : nullptr, nullptr, &r_diag) &&
             ok;
        if (!ok && lane == 0) atomicOr(&bv.st[b].exit_flags, GPT_EXIT_FACTOR);
        __syncwarp();
        write_ginv_compact(Ginv64c + (size_t)GC64 * (j - 1), Ginv64 + (size_t)G_STRIDE * (j - 1), Qki, sm.Rki, bd_ki,
                           r_diag, lane);
        if (k == N - 1)
            write_ginv_compact(Ginv64c + (size_t)GC64 * j, Ginv64 + (size_t)G_STRIDE * j, Qkp1i, nullptr, bd_kp1, true,
                               lane);
        // the next row of the same instance (k + 1 < N) needs R_k, Q_{k+1} and C_k: R_k and Q_{k+1} are
        // copied now into the blocks the inverses above have finished with, C_k once the products below
        // are done with C_{k-1}; its Q_k is not needed (its inverse is this row's (Q_k + rho I)^{-1})
        const bool next = (j + 1 < jend) && (k + 1 < N);
        if (next) {
            const float *Rk = G + (size_t)G_STRIDE * j + SS, *Qn = G + (size_t)G_STRIDE * (j + 1);
            for (int e = lane; e < CC; e += 32) cp_async4(sm.Gm1 + SS + e, Rk + e);
            for (int e = lane; e < SS; e += 32) cp_async4(sm.Gk + e, Qn + e);
        }
        // the products on the FP64 tensor cores, 14x14 (14x7) blocks padded to 16x16 (16x8)
        const float *Am = sm.C, *Bm = sm.C + SS;  // -A, -B
        {
            double cp[2][2][2] = {};
            auto a_el = [&](int i, int k) { return (i < NS && k < NS) ? (double)Am[i + NS * k] : 0.0; };
            auto q_el = [&](int k, int j) { return (k < NS && j < NS) ? Qki[k + NS * j] : 0.0; };
            if (bd_ki) {
                // block-diagonal Qt^{-1}: columns 0-7 draw only on k < 8, columns 8-15 only on k >= 8
                // (every skipped product is an exact zero, so the sums are those of the full product)
                const int g = lane >> 2, t = lane & 3;
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const int kx = 4 * kk + t, J = kk < 2 ? 0 : 1;
                    const double b = q_el(kx, 8 * J + g);
#pragma unroll
                    for (int I = 0; I < 2; ++I) mma884_f64(cp[I][J], a_el(8 * I + g, kx), b);
                }
            } else {
                warp_dmma<2, 2, 4>(a_el, q_el, cp, lane);  // phi = (-A) Qt^{-1}
            }
            warp_dmma_store(cp, [&](int i, int j, double v) { if (i < NS && j < NS) sm.phi[i + NS * j] = v; }, lane);
            if (r_diag) {
                // (-B) Rt^{-1} with a diagonal Rt^{-1}: a column scaling
                for (int e = lane; e < SC; e += 32) sm.BRi[e] = (double)Bm[e] * sm.Rki[(e / NS) * (NC + 1)];
            } else {
                double cb[2][1][2] = {};
                warp_dmma<2, 1, 2>([&](int i, int k) { return (i < NS && k < NC) ? (double)Bm[i + NS * k] : 0.0; },
                                   [&](int k, int j) { return (k < NC && j < NC) ? sm.Rki[k + NC * j] : 0.0; }, cb,
                                   lane);  // (-B) Rt^{-1}
                warp_dmma_store(cb, [&](int i, int j, double v) { if (i < NS && j < NC) sm.BRi[i + NS * j] = v; },
                                lane);
            }
        }
        __syncwarp();
        {
            double ct[2][2][2] = {};
            warp_dmma<2, 2, 4>([&](int i, int k) { return (i < NS && k < NS) ? sm.phi[i + NS * k] : 0.0; },
                               [&](int k, int j) { return (k < NS && j < NS) ? (double)Am[j + NS * k] : 0.0; }, ct,
                               lane);  // phi (-A)^T
            warp_dmma<2, 2, 2>([&](int i, int k) { return (i < NS && k < NC) ? sm.BRi[i + NS * k] : 0.0; },
                               [&](int k, int j) { return (k < NC && j < NS) ? (double)Bm[j + NS * k] : 0.0; }, ct,
                               lane);  // + (-B) Rt^{-1} (-B)^T
            warp_dmma_store(ct, [&](int i, int j, double v) { if (i < NS && j < NS) sm.theta[i + NS * j] = v; }, lane);
        }
        if (next) {
            __syncwarp();  // every lane has read C_{k-1}
            const float *Cn = Cm + (size_t)C_STRIDE * j;
            for (int e = lane; e < C_STRIDE; e += 32) cp_async4(sm.C + e, Cn + e);
        }
        cp_async_commit();
        pref = next;
        if (lane < NS) {
            double a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                a1 = fma(Qkp1i[lane + NS * t], sm.qkp1[t], a1);
                a2 = fma(sm.phi[lane + NS * t], sm.qk[t], a2);
            }
#pragma unroll
            for (int t = 0; t < NC; ++t) a3 = fma(sm.BRi[lane + NS * t], sm.rk[t], a3);
            gamma64[(size_t)NS * j + lane] = -((a1 - sm.ck[lane]) + (a3 + a2));
        }
        __syncwarp();
        for (int e = lane; e < SS; e += 32) {
            const int r = e % NS, cc = e / NS;
            Pk[e] = -sm.phi[e];
            if (r >= cc) Pk[SS + ((r * (r + 1)) >> 1) + cc] = -(sm.theta[e] + Qkp1i[e]);
        }
        if (lane == 0) Pk[PK64 - 1] = 0.0;
        __syncwarp();
        have = j;  // (Q_k + rho I)^{-1} stays for row k + 1
        have_bd = bd_kp1;
        cur ^= 1;
    }
}

cudaError_t launch_schur64(const BatchView &bv, const float *G, const float *C, const float *g, const float *c,
                           double *S64, double *gamma64, float *Ginv, double *Ginv64, double *Ginv64c, int num_sms,
                           cudaStream_t s, int ctas_per_sm)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    if (!bv.st || !Ginv64 || !Ginv64c) return cudaErrorInvalidValue;
    const size_t smem = sizeof(Schur64WarpSmem) * SCHUR_WARPS;
    int blocks = (bv.total_knots + SCHUR_WARPS - 1) / SCHUR_WARPS;
    const int cap = num_sms * ctas_per_sm;
    if (blocks > cap) blocks = cap;
    {
        const cudaError_t e = ensure_func_attrs((const void *)schur64_kernel, smem);
        if (e != cudaSuccess) return e;
    }
    schur64_kernel<<<blocks, 32 * SCHUR_WARPS, smem, s>>>(bv, G, C, g, c, S64, gamma64, Ginv, Ginv64, Ginv64c);
    return cudaGetLastError();
}

cudaError_t launch_schur(int mode, const BatchView &bv, float rho_scalar, const float *G,
                         const float *C, const float *g, const float *c, float *S, float *Pinv, float *gamma,
                         float *Ginv, double *Ginv64, float *csc_val, int need_pinv, int num_sms, cudaStream_t s)
{
    if (bv.total_knots <= 0) return cudaSuccess;
    const size_t smem = sizeof(SchurWarpSmem) * SCHUR_WARPS;
    int blocks = (bv.total_knots + SCHUR_WARPS - 1) / SCHUR_WARPS;
    const int cap = num_sms * 16;
    if (blocks > cap) blocks = cap;
    {
        const void *fn = mode == 0 ? (const void *)schur_kernel<0>
                                   : (mode == 1 ? (const void *)schur_kernel<1> : (const void *)schur_kernel<2>);
        const cudaError_t e = ensure_func_attrs(fn, smem);
        if (e != cudaSuccess) return e;
    }
    switch (mode) {
    case 0:
        schur_kernel<0><<<blocks, 32 * SCHUR_WARPS, smem, s>>>(bv, rho_scalar, G, C, g, c, S, Pinv, gamma,
                                                               Ginv, Ginv64, csc_val, need_pinv);
        break;
    case 1:
        schur_kernel<1><<<blocks, 32 * SCHUR_WARPS, smem, s>>>(bv, rho_scalar, G, C, g, c, S, Pinv, gamma,
                                                               Ginv, Ginv64, csc_val, need_pinv);
        break;
    default:
        schur_kernel<2><<<blocks, 32 * SCHUR_WARPS, smem, s>>>(bv, rho_scalar, G, C, g, c, S, Pinv, gamma,
                                                               Ginv, Ginv64, csc_val, need_pinv);
        break;
    }
    return cudaGetLastError();
}

}  // namespace gpt

namespace gpt {

// gato_form_ss_inner (oldschur.cuh:334-494): the stair preconditioner's off-diagonal blocks of
// Pinv (reference 3-block rows) from S and the block-Jacobi diagonal theta_k^{-1} already in Pinv:
//   Pinv[k].left  = -(theta_k^{-1} S[k].left) theta_{k-1}^{-1}
//   Pinv[k].right = -(theta_k^{-1} S[k+1].left^T) theta_{k+1}^{-1}
// One warp per block row; the five input blocks staged in shared memory, products in FP32 with the
// reference's summation order (column-major, t = 0 .. 13).
constexpr int SS_WARPS = 4;
struct SsWarpSmem {
    float tk[SS], tm[SS], tp[SS], phi[SS], phin[SS], scr[SS];
};

__device__ __forceinline__ void ss_prod(const float *A, const float *B, float *out, int lane, bool transB)
{
    for (int e = lane; e < SS; e += 32) {
        const int row = e % NS, col = e / NS;
        float r = 0.f;
#pragma unroll
        for (int t = 0; t < NS; ++t) r = fmaf(A[t * NS + row], transB ? B[t * NS + col] : B[col * NS + t], r);
        out[e] = r;
    }
}

__global__ void __launch_bounds__(32 * SS_WARPS) ss_kernel(BatchView bv, const float *__restrict__ S,
                                                           float *__restrict__ Pinv)
{
    __shared__ SsWarpSmem sm_all[SS_WARPS];
    const int lane = threadIdx.x & 31;
    SsWarpSmem &sm = sm_all[threadIdx.x >> 5];
    const int j = bv.j0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (j >= bv.j0 + bv.total_knots) return;  // warp-uniform
    const int b = bv.inst(j);
    if (!bv.active(b)) return;
    const int N = bv.N(b), k = j - bv.off(b);
    // knot j of the batch; its neighbours j - 1, j + 1 belong to the same instance when k > 0, k < N - 1
    for (int e = lane; e < SS; e += 32) {
        sm.tk[e] = Pinv[(size_t)S_STRIDE * j + SS + e];
        if (k > 0) {
            sm.tm[e] = Pinv[(size_t)S_STRIDE * (j - 1) + SS + e];
            sm.phi[e] = S[(size_t)S_STRIDE * j + e];
        }
        if (k < N - 1) {
            sm.tp[e] = Pinv[(size_t)S_STRIDE * (j + 1) + SS + e];
            sm.phin[e] = S[(size_t)S_STRIDE * (j + 1) + e];
        }
    }
    __syncwarp();
    if (k > 0) {
        ss_prod(sm.tk, sm.phi, sm.scr, lane, false);
        __syncwarp();
        for (int e = lane; e < SS; e += 32) {
            const int row = e % NS, col = e / NS;
            float r = 0.f;
#pragma unroll
            for (int t = 0; t < NS; ++t) r = fmaf(sm.scr[t * NS + row], sm.tm[col * NS + t], r);
            Pinv[(size_t)S_STRIDE * j + e] = -r;
        }
        __syncwarp();
    }
    if (k < N - 1) {
        ss_prod(sm.tk, sm.phin, sm.scr, lane, true);  // theta_k^{-1} phi_{k+1}^T
        __syncwarp();
        for (int e = lane; e < SS; e += 32) {
            const int row = e % NS, col = e / NS;
            float r = 0.f;
#pragma unroll
            for (int t = 0; t < NS; ++t) r = fmaf(sm.scr[t * NS + row], sm.tp[col * NS + t], r);
            Pinv[(size_t)S_STRIDE * j + 2 * SS + e] = -r;
        }
    }
}

cudaError_t launch_form_ss(const BatchView &bv, const float *S, float *Pinv, int num_sms, cudaStream_t s)
{
    (void)num_sms;
    if (bv.total_knots <= 0) return cudaSuccess;
    ss_kernel<<<(bv.total_knots + SS_WARPS - 1) / SS_WARPS, 32 * SS_WARPS, 0, s>>>(bv, S, Pinv);
    return cudaGetLastError();
}

}  // namespace gpt
