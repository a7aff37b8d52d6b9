// gpt_dyn.cuh -- per-lane rigid-body dynamics and kinematics of the iiwa14.
//
// Every function here runs in ONE thread on registers: a warp evaluates 32
// independent problems (mass-matrix columns, bias force, the 14 directional
// derivatives of inverse dynamics, line-search candidates) in lock step with
// no shared memory and no barriers.  Joint kinds and offsets are compile-time
// constants, so each joint's transform is specialised by the compiler.
//
// Math: Featherstone spatial algebra (angular part first), recursive
// Newton-Euler inverse dynamics with a forward-mode tangent.  The reference
// computes the same quantities with GRiD-generated block-parallel code
// (rbdfiles/iiwa_eepos_grid.cuh: inverse_dynamics_inner :2511,
// direct_minv_inner :3753, forward_dynamics_finish :4351,
// inverse_dynamics_gradient_inner :4558, end_effector_positions_inner :2015,
// end_effector_positions_gradient_inner :2255).
#pragma once
#include "gpt_common.cuh"
#include "gpt_model.cuh"

namespace gpt {

struct JointTrig {
    float c[model::NJ], s[model::NJ];
};

__device__ __forceinline__ void joint_trig(const float *q, JointTrig &t)
{
#pragma unroll
    for (int i = 0; i < model::NJ; ++i) sincosf(q[i], &t.s[i], &t.c[i]);
}

// E = (Rf Rz(q))^T applied to a 3-vector, per joint kind (see gpt_model.cuh)
template <int J>
__device__ __forceinline__ void rot_apply(float c, float s, const float *w, float *o)
{
    constexpr int K = model::kJointKind[J];
    if constexpr (K == 0) {  // [[c,s,0],[-s,c,0],[0,0,1]]
        o[0] = c * w[0] + s * w[1];
        o[1] = -s * w[0] + c * w[1];
        o[2] = w[2];
    } else if constexpr (K == 1) {  // [[-c,0,s],[s,0,c],[0,1,0]]
        o[0] = -c * w[0] + s * w[2];
        o[1] = s * w[0] + c * w[2];
        o[2] = w[1];
    } else {  // [[c,0,s],[-s,0,c],[0,-1,0]]
        o[0] = c * w[0] + s * w[2];
        o[1] = -s * w[0] + c * w[2];
        o[2] = -w[1];
    }
}
// E^T applied to a 3-vector
template <int J>
__device__ __forceinline__ void rot_apply_T(float c, float s, const float *w, float *o)
{
    constexpr int K = model::kJointKind[J];
    if constexpr (K == 0) {  // [[c,-s,0],[s,c,0],[0,0,1]]
        o[0] = c * w[0] - s * w[1];
        o[1] = s * w[0] + c * w[1];
        o[2] = w[2];
    } else if constexpr (K == 1) {  // [[-c,s,0],[0,0,1],[s,c,0]]
        o[0] = -c * w[0] + s * w[1];
        o[1] = w[2];
        o[2] = s * w[0] + c * w[1];
    } else {  // [[c,-s,0],[0,0,-1],[s,c,0]]
        o[0] = c * w[0] - s * w[1];
        o[1] = -w[2];
        o[2] = s * w[0] + c * w[1];
    }
}

// p x w for the constant joint offset p (only its non-zero entries emitted)
template <int J>
__device__ __forceinline__ void pcross(const float *w, float *o)
{
    constexpr float px = model::kJointP[J][0], py = model::kJointP[J][1], pz = model::kJointP[J][2];
    static_assert(px == 0.f, "iiwa joint offsets have no x component");
    if constexpr (py == 0.f) {  // p = (0,0,pz): (-pz*wy, pz*wx, 0)
        o[0] = -pz * w[1];
        o[1] = pz * w[0];
        o[2] = 0.f;
    } else {  // p = (0,py,0): (py*wz, 0, -py*wx)
        static_assert(pz == 0.f, "single-axis joint offsets");
        o[0] = py * w[2];
        o[1] = 0.f;
        o[2] = -py * w[0];
    }
}

// motion transform parent -> child: [E w; E (v - p x w)]
template <int J>
__device__ __forceinline__ void xmot(float c, float s, const float *m, float *o)
{
    float t[3], u[3];
    rot_apply<J>(c, s, m, o);
    pcross<J>(m, t);
    u[0] = m[3] - t[0];
    u[1] = m[4] - t[1];
    u[2] = m[5] - t[2];
    rot_apply<J>(c, s, u, o + 3);
}
// force transform child -> parent (X^T f): [E^T n + p x (E^T f); E^T f]
template <int J>
__device__ __forceinline__ void xforce_T(float c, float s, const float *f, float *o)
{
    float a[3], b[3], t[3];
    rot_apply_T<J>(c, s, f, a);
    rot_apply_T<J>(c, s, f + 3, b);
    pcross<J>(b, t);
    o[0] = a[0] + t[0];
    o[1] = a[1] + t[1];
    o[2] = a[2] + t[2];
    o[3] = b[0];
    o[4] = b[1];
    o[5] = b[2];
}

__device__ __forceinline__ void cross3(const float *a, const float *b, float *o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// spatial inertia of link J times a motion vector: [Ibar w + m c x v; m (v - c x w)]
template <int J>
__device__ __forceinline__ void inertia_apply(const float *v, float *o)
{
    constexpr float ixx = (float)model::ibar(J, 0), iyy = (float)model::ibar(J, 1),
                    izz = (float)model::ibar(J, 2), ixy = (float)model::ibar(J, 3),
                    ixz = (float)model::ibar(J, 4), iyz = (float)model::ibar(J, 5);
    constexpr float m = (float)model::kMass[J];
    constexpr float mcx = (float)(model::kMass[J] * model::kCom[J][0]);
    constexpr float mcy = (float)(model::kMass[J] * model::kCom[J][1]);
    constexpr float mcz = (float)(model::kMass[J] * model::kCom[J][2]);
    const float w0 = v[0], w1 = v[1], w2 = v[2], l0 = v[3], l1 = v[4], l2 = v[5];
    o[0] = ixx * w0 + ixy * w1 + ixz * w2 + (mcy * l2 - mcz * l1);
    o[1] = ixy * w0 + iyy * w1 + iyz * w2 + (mcz * l0 - mcx * l2);
    o[2] = ixz * w0 + iyz * w1 + izz * w2 + (mcx * l1 - mcy * l0);
    o[3] = m * l0 - (mcy * w2 - mcz * w1);
    o[4] = m * l1 - (mcz * w0 - mcx * w2);
    o[5] = m * l2 - (mcx * w1 - mcy * w0);
}

// v x_f f
__device__ __forceinline__ void crf(const float *v, const float *f, float *o)
{
    float a[3], b[3], c[3];
    cross3(v, f, a);
    cross3(v + 3, f + 3, b);
    cross3(v, f + 3, c);
    o[0] = a[0] + b[0];
    o[1] = a[1] + b[1];
    o[2] = a[2] + b[2];
    o[3] = c[0];
    o[4] = c[1];
    o[5] = c[2];
}
// v x_m (S qdj) with S = z-rotation: [(wy, -wx, 0) qdj; (ly, -lx, 0) qdj]
__device__ __forceinline__ void crm_s(const float *v, float qdj, float *o)
{
    o[0] = v[1] * qdj;
    o[1] = -v[0] * qdj;
    o[2] = 0.f;
    o[3] = v[4] * qdj;
    o[4] = -v[3] * qdj;
    o[5] = 0.f;
}
// S x_m u and S x_f f (identical form): [z x u_ang; z x u_lin]
__device__ __forceinline__ void s_cross(const float *u, float *o)
{
    o[0] = -u[1];
    o[1] = u[0];
    o[2] = 0.f;
    o[3] = -u[4];
    o[4] = u[3];
    o[5] = 0.f;
}

template <bool TANGENT>
struct RneaState {
    float vp[6], ap[6];
    float f[model::NJ][6];
    float dvp[TANGENT ? 6 : 1], dap[TANGENT ? 6 : 1];
    float df[model::NJ][TANGENT ? 6 : 1];
};

template <int J, bool TANGENT>
__device__ __forceinline__ void rnea_fwd(const JointTrig &t, const float *qd, const float *qdd, int dq_dir,
                                         int dqd_dir, RneaState<TANGENT> &st)
{
    const float c = t.c[J], s = t.s[J];
    float Xv[6], Xa[6], v[6], a[6], cv[6], Iv[6], Ia[6], cIv[6];
    xmot<J>(c, s, st.vp, Xv);
    xmot<J>(c, s, st.ap, Xa);
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] = Xv[k];
    v[2] += qd[J];
    crm_s(v, qd[J], cv);
#pragma unroll
    for (int k = 0; k < 6; ++k) a[k] = Xa[k] + cv[k];
    a[2] += qdd[J];
    inertia_apply<J>(v, Iv);
    inertia_apply<J>(a, Ia);
    crf(v, Iv, cIv);
#pragma unroll
    for (int k = 0; k < 6; ++k) st.f[J][k] = Ia[k] + cIv[k];
    if constexpr (TANGENT) {
        const float dqj = (J == dq_dir) ? 1.f : 0.f;
        const float dqdj = (J == dqd_dir) ? 1.f : 0.f;
        float Xdv[6], Xda[6], sXv[6], sXa[6], dv[6], da[6], t1[6], t2[6], Ida[6], Idv[6], c1[6], c2[6];
        xmot<J>(c, s, st.dvp, Xdv);
        xmot<J>(c, s, st.dap, Xda);
        s_cross(Xv, sXv);
        s_cross(Xa, sXa);
#pragma unroll
        for (int k = 0; k < 6; ++k) dv[k] = Xdv[k] - dqj * sXv[k];
        dv[2] += dqdj;
        crm_s(dv, qd[J], t1);
        crm_s(v, dqdj, t2);
#pragma unroll
        for (int k = 0; k < 6; ++k) da[k] = Xda[k] - dqj * sXa[k] + t1[k] + t2[k];
        inertia_apply<J>(da, Ida);
        inertia_apply<J>(dv, Idv);
        crf(dv, Iv, c1);
        crf(v, Idv, c2);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            st.df[J][k] = Ida[k] + c1[k] + c2[k];
            st.dvp[k] = dv[k];
            st.dap[k] = da[k];
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        st.vp[k] = v[k];
        st.ap[k] = a[k];
    }
}

template <int J, bool TANGENT>
__device__ __forceinline__ void rnea_bwd(const JointTrig &t, int dq_dir, RneaState<TANGENT> &st, float *tau,
                                         float *dtau)
{
    tau[J] = st.f[J][2];
    if constexpr (TANGENT) dtau[J] = st.df[J][2];
    if constexpr (J > 0) {
        const float c = t.c[J], s = t.s[J];
        float tf[6];
        xforce_T<J>(c, s, st.f[J], tf);
        if constexpr (TANGENT) {
            const float dqj = (J == dq_dir) ? 1.f : 0.f;
            float t2[6], sf[6], t3[6];
            xforce_T<J>(c, s, st.df[J], t2);
            s_cross(st.f[J], sf);
            xforce_T<J>(c, s, sf, t3);
#pragma unroll
            for (int k = 0; k < 6; ++k) st.df[J - 1][k] += t2[k] + dqj * t3[k];
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) st.f[J - 1][k] += tf[k];
    }
}

// tau = ID(q, qd, qdd); with TANGENT also dtau = d ID / d(q_dq_dir or qd_dqd_dir)
// (a direction index of -1 means no perturbation of that argument).
template <bool TANGENT>
__device__ __forceinline__ void rnea(const JointTrig &t, const float *qd, const float *qdd, int dq_dir,
                                     int dqd_dir, float *tau, float *dtau)
{
    RneaState<TANGENT> st;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        st.vp[k] = 0.f;
        st.ap[k] = 0.f;
        if constexpr (TANGENT) {
            st.dvp[k] = 0.f;
            st.dap[k] = 0.f;
        }
    }
    rnea_fwd<0, TANGENT>(t, qd, qdd, dq_dir, dqd_dir, st);
    rnea_fwd<1, TANGENT>(t, qd, qdd, dq_dir, dqd_dir, st);
    rnea_fwd<2, TANGENT>(t, qd, qdd, dq_dir, dqd_dir, st);
    rnea_fwd<3, TANGENT>(t, qd, qdd, dq_dir, dqd_dir, st);
    rnea_fwd<4, TANGENT>(t, qd, qdd, dq_dir, dqd_dir, st);
    rnea_fwd<5, TANGENT>(t, qd, qdd, dq_dir, dqd_dir, st);
    rnea_fwd<6, TANGENT>(t, qd, qdd, dq_dir, dqd_dir, st);
    rnea_bwd<6, TANGENT>(t, dq_dir, st, tau, dtau);
    rnea_bwd<5, TANGENT>(t, dq_dir, st, tau, dtau);
    rnea_bwd<4, TANGENT>(t, dq_dir, st, tau, dtau);
    rnea_bwd<3, TANGENT>(t, dq_dir, st, tau, dtau);
    rnea_bwd<2, TANGENT>(t, dq_dir, st, tau, dtau);
    rnea_bwd<1, TANGENT>(t, dq_dir, st, tau, dtau);
    rnea_bwd<0, TANGENT>(t, dq_dir, st, tau, dtau);
}

// Joint-space mass matrix M(q) on one lane.  Column j is inverse dynamics at zero velocity with a unit
// acceleration of joint j (gravity plays no part): only links j .. 6 accelerate (a_K = X_K a_{K-1},
// f_K = I_K a_K, no velocity products), and the rows k >= j -- M's lower triangle -- are the joint
// components of the forces after the backward pass has reached link j.  About a third of the work of
// seven full inverse-dynamics passes.  M is stored packed: entry (k, j), k >= j, at k (k + 1) / 2 + j.
template <int J, int K>
__device__ __forceinline__ void mcol_fwd(const JointTrig &t, const float *ap, float (&f)[model::NJ][6])
{
    float a[6];
    xmot<K>(t.c[K], t.s[K], ap, a);
    inertia_apply<K>(a, f[K]);
    if constexpr (K + 1 < model::NJ) mcol_fwd<J, K + 1>(t, a, f);
}
template <int J, int K>
__device__ __forceinline__ void mcol_bwd(const JointTrig &t, float (&f)[model::NJ][6])
{
    if constexpr (K > J) {
        float tf[6];
        xforce_T<K>(t.c[K], t.s[K], f[K], tf);
#pragma unroll
        for (int i = 0; i < 6; ++i) f[K - 1][i] += tf[i];
        mcol_bwd<J, K - 1>(t, f);
    }
}
template <int J>
__device__ __forceinline__ void mass_column(const JointTrig &t, float (&M)[28])
{
    float f[model::NJ][6];
    const float sz[6] = {0.f, 0.f, 1.f, 0.f, 0.f, 0.f};  // S_J: rotation about the joint's z axis
    inertia_apply<J>(sz, f[J]);
    if constexpr (J + 1 < model::NJ) mcol_fwd<J, J + 1>(t, sz, f);
    mcol_bwd<J, model::NJ - 1>(t, f);
#pragma unroll
    for (int k = J; k < model::NJ; ++k) M[(k * (k + 1)) / 2 + J] = f[k][2];
}
__device__ __forceinline__ void mass_matrix_lane(const JointTrig &t, float (&M)[28])
{
    mass_column<0>(t, M);
    mass_column<1>(t, M);
    mass_column<2>(t, M);
    mass_column<3>(t, M);
    mass_column<4>(t, M);
    mass_column<5>(t, M);
    mass_column<6>(t, M);
}

// x = M^{-1} b for the SPD 7x7 M (packed lower triangle, FP32) on one lane: an FP32 Cholesky
// factorisation, the two triangular solves, then one step of iterative refinement with the residual
// b - M x accumulated in FP64 (M's FP32 entries are exact in FP64), which brings x to the accuracy
// of an FP64 solve of the same M while cond(M) eps32 << 1 (the iiwa's M: cond ~ 1e2 .. 1e3).
__device__ __forceinline__ void spd7_solve_lane(const float (&M)[28], const double (&b)[NQ], double (&x)[NQ])
{
    // Every loop runs over the full constant range with the triangle as a guard, so that all of them
    // unroll and M, L stay in registers (loops bounded by an outer index left both in local memory).
    // The diagonal's reciprocals come from rsqrtf and the triangular solves multiply by them instead
    // of dividing: the FP64 refinement step below removes the FP32 solve's rounding either way.
    auto tri = [](int i, int j) { return (i * (i + 1)) / 2 + j; };
    float L[28], Li[NQ];  // the factor below the diagonal, the reciprocals of its diagonal
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
        float d = M[tri(j, j)];
#pragma unroll
        for (int k = 0; k < NQ; ++k)
            if (k < j) d = fmaf(-L[tri(j, k)], L[tri(j, k)], d);
        const float inv = rsqrtf(d);  // 1 / L_jj
        Li[j] = inv;
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            if (i > j) {
                float v = M[tri(i, j)];
#pragma unroll
                for (int k = 0; k < NQ; ++k)
                    if (k < j) v = fmaf(-L[tri(i, k)], L[tri(j, k)], v);
                L[tri(i, j)] = v * inv;
            }
        }
    }
    auto solve = [&](const float (&r)[NQ], float (&y)[NQ]) {
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            float v = r[i];
#pragma unroll
            for (int k = 0; k < NQ; ++k)
                if (k < i) v = fmaf(-L[tri(i, k)], y[k], v);
            y[i] = v * Li[i];
        }
#pragma unroll
        for (int ii = 0; ii < NQ; ++ii) {
            const int i = NQ - 1 - ii;
            float v = y[i];
#pragma unroll
            for (int k = 0; k < NQ; ++k)
                if (k > i) v = fmaf(-L[tri(k, i)], y[k], v);
            y[i] = v * Li[i];
        }
    };
    float r[NQ], y[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) r[i] = (float)b[i];
    solve(r, y);
#pragma unroll
    for (int i = 0; i < NQ; ++i) x[i] = (double)y[i];
    // refinement: r = b - M x in FP64
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        double v = b[i];
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
            const float mik = i >= k ? M[tri(i, k)] : M[tri(k, i)];
            v = fma(-(double)mik, x[k], v);
        }
        r[i] = (float)v;
    }
    solve(r, y);
#pragma unroll
    for (int i = 0; i < NQ; ++i) x[i] += (double)y[i];
}

// Gauss-Jordan elimination with a 7x7 SPD matrix M (no pivoting: every pivot is positive) over a
// group of lanes holding the columns of [M | R]: lane base + i holds column i (7 entries).
// Afterwards the lanes of R's columns hold M^{-1} R (and M's lanes the identity).  Every lane of
// the warp calls it; lanes outside a group pass any base of a real group and ignore the result.
__device__ __forceinline__ void gj7_group(double (&col)[7], int base)
{
#pragma unroll
    for (int p = 0; p < 7; ++p) {
        const double piv = __shfl_sync(0xffffffffu, col[p], base + p);
        const double prow = col[p] * rcp_newton(piv);
#pragma unroll
        for (int r = 0; r < 7; ++r) {
            if (r == p) continue;
            const double pr = __shfl_sync(0xffffffffu, col[r], base + p);
            col[r] = fma(-pr, prow, col[r]);
        }
        col[p] = prow;
    }
}

// Forward dynamics by a group of 8 lanes (lanes base .. base+7): lane m < 7 forms mass-matrix
// column m by inverse dynamics, lane 7 the bias force c(q, qd); after an FP64 Gauss-Jordan on
// [M | u - c] (M symmetrised from the lanes' columns) lane base+7's col holds qdd = M^{-1}(u - c).
// Every lane of the warp calls it with its group's q, qd, u.
__device__ __forceinline__ void fd_group(const float (&q)[NQ], const float (&qd)[NQ], const float (&u)[NC],
                                         double (&col)[NQ], int m, int base)
{
    JointTrig t;
    joint_trig(q, t);
    float v[NQ], a[NQ], tau[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        v[i] = (m == 7) ? qd[i] : 0.f;
        a[i] = (m == i) ? 1.f : 0.f;
    }
    rnea<false>(t, v, a, -1, -1, tau, nullptr);
#pragma unroll
    for (int r = 0; r < NQ; ++r) {
        float mr = 0.f;  // M[m][r] = entry m of column r (lane base + r)
#pragma unroll
        for (int e = 0; e < NQ; ++e) {
            const float ve = __shfl_sync(0xffffffffu, tau[e], base + r);
            if (e == m) mr = ve;
        }
        col[r] = (m < NQ) ? 0.5 * ((double)tau[r] + (double)mr) : (double)u[r] - (double)tau[r];
    }
    gj7_group(col, base);
}

// Forward kinematics: end-effector position p (xyz) and, optionally, the
// position Jacobian J (3x7, col-major: J[3*j + d]).  Joint j's axis in the
// base frame is the third column of T_0...T_j; dp/dq_j = z_j x (p - o_j).
struct FkState {
    float Rm[9];  // row-major rotation of the current frame
    float o[3];
    float zs[model::NJ][3], os[model::NJ][3];
};

template <int J, bool WITH_JAC>
__device__ __forceinline__ void fk_step(const JointTrig &t, FkState &st)
{
    constexpr float py = model::kJointP[J][1], pz = model::kJointP[J][2];
    constexpr int K = model::kJointKind[J];
    st.o[0] += st.Rm[1] * py + st.Rm[2] * pz;
    st.o[1] += st.Rm[4] * py + st.Rm[5] * pz;
    st.o[2] += st.Rm[7] * py + st.Rm[8] * pz;
    const float c = t.c[J], s = t.s[J];
    float W[9];  // W = Rf Rz(q), row-major
    if constexpr (K == 0) {
        W[0] = c; W[1] = -s; W[2] = 0.f; W[3] = s; W[4] = c; W[5] = 0.f; W[6] = 0.f; W[7] = 0.f; W[8] = 1.f;
    } else if constexpr (K == 1) {
        W[0] = -c; W[1] = s; W[2] = 0.f; W[3] = 0.f; W[4] = 0.f; W[5] = 1.f; W[6] = s; W[7] = c; W[8] = 0.f;
    } else {
        W[0] = c; W[1] = -s; W[2] = 0.f; W[3] = 0.f; W[4] = 0.f; W[5] = -1.f; W[6] = s; W[7] = c; W[8] = 0.f;
    }
    float Nr[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            Nr[3 * r + k] = st.Rm[3 * r] * W[k] + st.Rm[3 * r + 1] * W[3 + k] + st.Rm[3 * r + 2] * W[6 + k];
#pragma unroll
    for (int k = 0; k < 9; ++k) st.Rm[k] = Nr[k];
    if constexpr (WITH_JAC) {
        st.zs[J][0] = st.Rm[2]; st.zs[J][1] = st.Rm[5]; st.zs[J][2] = st.Rm[8];
        st.os[J][0] = st.o[0]; st.os[J][1] = st.o[1]; st.os[J][2] = st.o[2];
    }
}

// End-effector xyz and roll / pitch / yaw of the last frame (end_effector_positions_inner,
// rbdfiles/iiwa_eepos_grid.cuh:2015-2090): roll = atan2(R21, R22),
// pitch = -atan2(R20, sqrt(R21^2 + R22^2)), yaw = atan2(R10, R00)
__device__ __forceinline__ void fk_pose_lane(const JointTrig &t, float *pose)
{
    FkState st;
#pragma unroll
    for (int k = 0; k < 9; ++k) st.Rm[k] = (k % 4 == 0) ? 1.f : 0.f;
    st.o[0] = st.o[1] = st.o[2] = 0.f;
    fk_step<0, false>(t, st);
    fk_step<1, false>(t, st);
    fk_step<2, false>(t, st);
    fk_step<3, false>(t, st);
    fk_step<4, false>(t, st);
    fk_step<5, false>(t, st);
    fk_step<6, false>(t, st);
    pose[0] = st.o[0];
    pose[1] = st.o[1];
    pose[2] = st.o[2];
    pose[3] = atan2f(st.Rm[7], st.Rm[8]);
    pose[4] = -atan2f(st.Rm[6], sqrtf(st.Rm[7] * st.Rm[7] + st.Rm[8] * st.Rm[8]));
    pose[5] = atan2f(st.Rm[3], st.Rm[0]);
}

template <bool WITH_JAC>
__device__ __forceinline__ void fk_lane(const JointTrig &t, float *p, float *Jac)
{
    FkState st;
#pragma unroll
    for (int k = 0; k < 9; ++k) st.Rm[k] = (k % 4 == 0) ? 1.f : 0.f;
    st.o[0] = st.o[1] = st.o[2] = 0.f;
    fk_step<0, WITH_JAC>(t, st);
    fk_step<1, WITH_JAC>(t, st);
    fk_step<2, WITH_JAC>(t, st);
    fk_step<3, WITH_JAC>(t, st);
    fk_step<4, WITH_JAC>(t, st);
    fk_step<5, WITH_JAC>(t, st);
    fk_step<6, WITH_JAC>(t, st);
    p[0] = st.o[0];
    p[1] = st.o[1];
    p[2] = st.o[2];
    if constexpr (WITH_JAC) {
#pragma unroll
        for (int j = 0; j < model::NJ; ++j) {
            float d[3] = {st.o[0] - st.os[j][0], st.o[1] - st.os[j][1], st.o[2] - st.os[j][2]};
            cross3(st.zs[j], d, Jac + 3 * j);
        }
    }
}

}  // namespace gpt
