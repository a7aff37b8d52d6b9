/*
 * oracle/oracle.c -- TEST INFRASTRUCTURE (CPU oracle), not the product.
 *
 * A plain-C restatement of the reference's SQP inner loop for iiwa14
 * end-effector tracking.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg use it, and only as the checker.  Compiled twice
 * (GPT_REAL=float -> orc_f32_*, GPT_REAL=double -> orc_f64_*).
 *
 * Where the reference's arithmetic order is visible (block-level mat-mat,
 * mat-vec and Gauss-Jordan loops in oldschur.cuh) the f32 build follows it,
 * so that it tracks the reference's FP32 rounding closely.  The rigid-body
 * dynamics use the textbook recursive Newton-Euler algorithm with a
 * forward-mode tangent for the gradient; the reference computes the same
 * quantities with GRiD-generated code (rbdfiles/iiwa_eepos_grid.cuh).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "model.h"
#include "oracle.h"

#ifndef GPT_REAL
#define GPT_REAL double
#define GPT_SFX f64
#endif
typedef GPT_REAL R;
#define ORC_CAT2(a, b, c) a##b##c
#define ORC_CAT(a, b, c) ORC_CAT2(a, b, c)
#define ORC(name) ORC_CAT(orc_, GPT_SFX, _##name)

#define NS 14
#define NC 7
#define NX 21
#define SS 196
#define SC 98
#define CC 49
#define GSTRIDE 245
#define CSTRIDE 294

/* ------------------------------------------------------------------------ */
/* model                                                                     */
/* ------------------------------------------------------------------------ */

static void fixed_rot(int kind, double Rm[9]) /* row-major */
{
    static const double r0[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    static const double r1[9] = {-1, 0, 0, 0, 0, 1, 0, 1, 0};
    static const double r2[9] = {1, 0, 0, 0, 0, -1, 0, 1, 0};
    memcpy(Rm, kind == 0 ? r0 : (kind == 1 ? r1 : r2), sizeof(r0));
}

typedef struct {
    R E[ORC_NJ][9];  /* child <- parent rotation, row-major: (Rf Rz(q))^T */
    R p[ORC_NJ][3];  /* child origin in parent coordinates */
} xforms_t;

typedef struct {
    R Ibar[ORC_NJ][9]; /* rotational inertia about the link origin, row-major */
    R m[ORC_NJ];
    R c[ORC_NJ][3];
} inertia_t;

static void build_inertia(inertia_t *I)
{
    for (int i = 0; i < ORC_NJ; ++i) {
        const double m = ORC_MASS[i], *c = ORC_COM[i], *t = ORC_INERTIA[i];
        double Ic[9] = {t[0], t[3], t[4], t[3], t[1], t[5], t[4], t[5], t[2]};
        double cc = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k)
                I->Ibar[i][3 * r + k] = (R)(Ic[3 * r + k] + m * ((r == k) * cc - c[r] * c[k]));
        I->m[i] = (R)m;
        for (int r = 0; r < 3; ++r) I->c[i][r] = (R)c[r];
    }
}

/* rbdfiles/iiwa_eepos_grid.cuh:1768-1853 (load_update_XImats_helpers) */
static void build_xforms(const R *q, xforms_t *X)
{
    for (int i = 0; i < ORC_NJ; ++i) {
        double Rf[9];
        fixed_rot(ORC_JOINT_R_KIND[i], Rf);
        R s = (R)sin(q[i]), cq = (R)cos(q[i]);
        /* W = Rf * Rz(q); E = W^T */
        R Rz[9] = {cq, -s, 0, s, cq, 0, 0, 0, 1};
        R W[9];
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) {
                R acc = 0;
                for (int j = 0; j < 3; ++j) acc += (R)Rf[3 * r + j] * Rz[3 * j + k];
                W[3 * r + k] = acc;
            }
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) X->E[i][3 * r + k] = W[3 * k + r];
        for (int r = 0; r < 3; ++r) X->p[i][r] = (R)ORC_JOINT_P[i][r];
    }
}

static inline void cross3(const R *a, const R *b, R *o)
{
    R t0 = a[1] * b[2] - a[2] * b[1];
    R t1 = a[2] * b[0] - a[0] * b[2];
    R t2 = a[0] * b[1] - a[1] * b[0];
    o[0] = t0; o[1] = t1; o[2] = t2;
}
static inline void mv3(const R *M, const R *v, R *o)
{
    for (int r = 0; r < 3; ++r) o[r] = M[3 * r] * v[0] + M[3 * r + 1] * v[1] + M[3 * r + 2] * v[2];
}
static inline void mtv3(const R *M, const R *v, R *o)
{
    for (int r = 0; r < 3; ++r) o[r] = M[r] * v[0] + M[3 + r] * v[1] + M[6 + r] * v[2];
}

/* motion transform parent->child: [E w; E (v - p x w)] */
static void xm_apply(const xforms_t *X, int i, const R *m, R *o)
{
    R t[3], u[3];
    mv3(X->E[i], m, o);
    cross3(X->p[i], m, t);
    for (int k = 0; k < 3; ++k) u[k] = m[3 + k] - t[k];
    mv3(X->E[i], u, o + 3);
}
/* force transform child->parent (X^T f): [E^T n + p x (E^T f); E^T f] */
static void xf_apply_T(const xforms_t *X, int i, const R *f, R *o)
{
    R a[3], b[3], t[3];
    mtv3(X->E[i], f, a);
    mtv3(X->E[i], f + 3, b);
    cross3(X->p[i], b, t);
    for (int k = 0; k < 3; ++k) { o[k] = a[k] + t[k]; o[3 + k] = b[k]; }
}
/* v x_m u */
static void crm(const R *v, const R *u, R *o)
{
    R a[3], b[3], c[3];
    cross3(v, u, a);
    cross3(v + 3, u, b);
    cross3(v, u + 3, c);
    for (int k = 0; k < 3; ++k) { o[k] = a[k]; o[3 + k] = b[k] + c[k]; }
}
/* v x_f f */
static void crf(const R *v, const R *f, R *o)
{
    R a[3], b[3], c[3];
    cross3(v, f, a);
    cross3(v + 3, f + 3, b);
    cross3(v, f + 3, c);
    for (int k = 0; k < 3; ++k) { o[k] = a[k] + b[k]; o[3 + k] = c[k]; }
}
/* spatial inertia times motion: [Ibar w + m c x v; m v - m c x w] */
static void inertia_apply(const inertia_t *I, int i, const R *v, R *o)
{
    R a[3], b[3], cw[3];
    mv3(I->Ibar[i], v, a);
    cross3(I->c[i], v + 3, b);
    cross3(I->c[i], v, cw);
    for (int k = 0; k < 3; ++k) {
        o[k] = a[k] + I->m[i] * b[k];
        o[3 + k] = I->m[i] * (v[3 + k] - cw[k]);
    }
}

/*
 * Recursive Newton-Euler inverse dynamics with a forward-mode tangent.
 * Follows the quantities of rbdfiles/iiwa_eepos_grid.cuh:2511-2740
 * (inverse_dynamics_inner) and :4558 (inverse_dynamics_gradient_inner):
 * tau = ID(q, qd, qdd), dtau = d/deps ID(q + eps dq, qd + eps dqd, qdd + eps dqdd).
 * Gravity is 0 (iiwa_eepos_plant.cuh:50-51).  dtau may be NULL.
 */
static void rnea_t(const xforms_t *X, const inertia_t *I, const R *q, const R *qd, const R *qdd,
                   const R *dq, const R *dqd, const R *dqdd, R *tau, R *dtau)
{
    (void)q;
    R v[ORC_NJ][6], a[ORC_NJ][6], f[ORC_NJ][6];
    R dv[ORC_NJ][6], da[ORC_NJ][6], df[ORC_NJ][6];
    const int tangent = (dtau != NULL);
    for (int i = 0; i < ORC_NJ; ++i) {
        R vp[6] = {0, 0, 0, 0, 0, 0}, ap[6] = {0, 0, 0, 0, 0, 0};
        R dvp[6] = {0, 0, 0, 0, 0, 0}, dap[6] = {0, 0, 0, 0, 0, 0};
        if (i > 0) {
            memcpy(vp, v[i - 1], sizeof(vp)); memcpy(ap, a[i - 1], sizeof(ap));
            memcpy(dvp, dv[i - 1], sizeof(dvp)); memcpy(dap, da[i - 1], sizeof(dap));
        }
        R Xv[6], Xa[6];
        xm_apply(X, i, vp, Xv);
        xm_apply(X, i, ap, Xa);
        R vJ[6] = {0, 0, qd[i], 0, 0, 0};
        for (int k = 0; k < 6; ++k) v[i][k] = Xv[k] + vJ[k];
        R cvj[6];
        crm(v[i], vJ, cvj);
        for (int k = 0; k < 6; ++k) a[i][k] = Xa[k] + cvj[k];
        a[i][2] += qdd[i];
        R Iv[6], Ia[6], cIv[6];
        inertia_apply(I, i, v[i], Iv);
        inertia_apply(I, i, a[i], Ia);
        crf(v[i], Iv, cIv);
        for (int k = 0; k < 6; ++k) f[i][k] = Ia[k] + cIv[k];
        if (tangent) {
            R S[6] = {0, 0, 1, 0, 0, 0};
            R Xdv[6], Xda[6], sXv[6], sXa[6];
            xm_apply(X, i, dvp, Xdv);
            xm_apply(X, i, dap, Xda);
            crm(S, Xv, sXv);
            crm(S, Xa, sXa);
            R dvJ[6] = {0, 0, dqd[i], 0, 0, 0};
            for (int k = 0; k < 6; ++k) dv[i][k] = Xdv[k] - dq[i] * sXv[k] + dvJ[k];
            R t1[6], t2[6];
            crm(dv[i], vJ, t1);
            crm(v[i], dvJ, t2);
            for (int k = 0; k < 6; ++k) da[i][k] = Xda[k] - dq[i] * sXa[k] + t1[k] + t2[k];
            da[i][2] += dqdd[i];
            R Ida[6], Idv[6], c1[6], c2[6];
            inertia_apply(I, i, da[i], Ida);
            inertia_apply(I, i, dv[i], Idv);
            crf(dv[i], Iv, c1);
            crf(v[i], Idv, c2);
            for (int k = 0; k < 6; ++k) df[i][k] = Ida[k] + c1[k] + c2[k];
        }
    }
    for (int i = ORC_NJ - 1; i >= 0; --i) {
        tau[i] = f[i][2];
        if (tangent) dtau[i] = df[i][2];
        if (i > 0) {
            R t[6];
            xf_apply_T(X, i, f[i], t);
            if (tangent) {
                R S[6] = {0, 0, 1, 0, 0, 0}, sf[6], t2[6], t3[6];
                xf_apply_T(X, i, df[i], t2);
                crf(S, f[i], sf);
                xf_apply_T(X, i, sf, t3);
                for (int k = 0; k < 6; ++k) df[i - 1][k] += t2[k] + dq[i] * t3[k];
            }
            for (int k = 0; k < 6; ++k) f[i - 1][k] += t[k];
        }
    }
}

static inertia_t g_inertia;
static int g_inertia_ready = 0;
static const inertia_t *inertia(void)
{
    if (!g_inertia_ready) { build_inertia(&g_inertia); g_inertia_ready = 1; }
    return &g_inertia;
}

void ORC(rnea)(const R *q, const R *qd, const R *qdd, R *tau)
{
    xforms_t X;
    build_xforms(q, &X);
    rnea_t(&X, inertia(), q, qd, qdd, NULL, NULL, NULL, tau, NULL);
}

/* in-place inverse of an SPD n x n (col-major) matrix via Cholesky */
static int spd_inverse(R *M, int n)
{
    R L[49 * 4];
    R Inv[49 * 4];
    memset(L, 0, sizeof(R) * n * n);
    for (int j = 0; j < n; ++j) {
        R d = M[j + n * j];
        for (int k = 0; k < j; ++k) d -= L[j + n * k] * L[j + n * k];
        if (!(d > 0)) return -1;
        R ljj = (R)sqrt(d);
        L[j + n * j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            R s = M[i + n * j];
            for (int k = 0; k < j; ++k) s -= L[i + n * k] * L[j + n * k];
            L[i + n * j] = s / ljj;
        }
    }
    for (int col = 0; col < n; ++col) {
        R y[14];
        for (int i = 0; i < n; ++i) {
            R s = (i == col) ? (R)1 : (R)0;
            for (int k = 0; k < i; ++k) s -= L[i + n * k] * y[k];
            y[i] = s / L[i + n * i];
        }
        for (int i = n - 1; i >= 0; --i) {
            R s = y[i];
            for (int k = i + 1; k < n; ++k) s -= L[k + n * i] * Inv[k + n * col];
            Inv[i + n * col] = s / L[i + n * i];
        }
    }
    memcpy(M, Inv, sizeof(R) * n * n);
    return 0;
}

/* joint-space inertia M(q) (col-major 7x7) column by column: M e_j = ID(q, 0, e_j) */
static void mass_matrix(const xforms_t *X, const R *q, R *M)
{
    R zero[ORC_NJ] = {0};
    for (int j = 0; j < ORC_NJ; ++j) {
        R e[ORC_NJ] = {0};
        e[j] = 1;
        rnea_t(X, inertia(), q, zero, e, NULL, NULL, NULL, M + ORC_NJ * j, NULL);
    }
    /* symmetrise (exact in theory; removes rounding asymmetry) */
    for (int j = 0; j < ORC_NJ; ++j)
        for (int i = j + 1; i < ORC_NJ; ++i) {
            R s = (R)0.5 * (M[i + 7 * j] + M[j + 7 * i]);
            M[i + 7 * j] = s; M[j + 7 * i] = s;
        }
}

/* rbdfiles/iiwa_eepos_grid.cuh:3753 (direct_minv_inner): M(q)^{-1}, full 7x7 col-major */
void ORC(minv)(const R *q, R *Minv)
{
    xforms_t X;
    build_xforms(q, &X);
    mass_matrix(&X, q, Minv);
    spd_inverse(Minv, ORC_NJ);
}

/* rbdfiles/iiwa_eepos_grid.cuh:4351-4395 (forward_dynamics): qdd = Minv (u - c(q,qd)) */
void ORC(fd)(const R *q, const R *qd, const R *u, R *qdd)
{
    xforms_t X;
    build_xforms(q, &X);
    R M[49], c[7], zero[7] = {0};
    mass_matrix(&X, q, M);
    spd_inverse(M, 7);
    rnea_t(&X, inertia(), q, qd, zero, NULL, NULL, NULL, c, NULL);
    for (int r = 0; r < 7; ++r) {
        R acc = 0;
        for (int k = 0; k < 7; ++k) acc += M[r + 7 * k] * (u[k] - c[k]);
        qdd[r] = acc;
    }
}

/*
 * rbdfiles/iiwa_eepos_plant.cuh:126-156 (forwardDynamicsAndGradient):
 * qdd = FD(q,qd,u); df_du (7x21 col-major) = [-Minv dID/dq, -Minv dID/dqd, Minv]
 * with dID evaluated at (q, qd, qdd).
 */
void ORC(fd_grad)(const R *q, const R *qd, const R *u, R *qdd, R *df_du)
{
    xforms_t X;
    build_xforms(q, &X);
    R M[49], c[7], zero[7] = {0};
    mass_matrix(&X, q, M);
    spd_inverse(M, 7);
    rnea_t(&X, inertia(), q, qd, zero, NULL, NULL, NULL, c, NULL);
    for (int r = 0; r < 7; ++r) {
        R acc = 0;
        for (int k = 0; k < 7; ++k) acc += M[r + 7 * k] * (u[k] - c[k]);
        qdd[r] = acc;
    }
    for (int j = 0; j < 14; ++j) {
        R dq[7] = {0}, dqd[7] = {0}, tau[7], dtau[7];
        if (j < 7) dq[j] = 1; else dqd[j - 7] = 1;
        rnea_t(&X, inertia(), q, qd, qdd, dq, dqd, zero, tau, dtau);
        for (int r = 0; r < 7; ++r) {
            R acc = 0;
            for (int k = 0; k < 7; ++k) acc += M[r + 7 * k] * dtau[k];
            df_du[7 * j + r] = -acc;
        }
    }
    for (int j = 0; j < 7; ++j)
        for (int r = 0; r < 7; ++r) df_du[98 + 7 * j + r] = M[r + 7 * j];
}

/* ------------------------------------------------------------------------ */
/* forward kinematics: rbdfiles/iiwa_eepos_grid.cuh:1857-1913, 2015-2090     */
/* ------------------------------------------------------------------------ */

/* chain of homogeneous transforms; frames[i] = T_0 ... T_i (row-major 3x4) */
static void fk_frames(const R *q, R frames[ORC_NJ][12])
{
    R T[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    for (int i = 0; i < ORC_NJ; ++i) {
        double Rf[9];
        fixed_rot(ORC_JOINT_R_KIND[i], Rf);
        R s = (R)sin(q[i]), cq = (R)cos(q[i]);
        R Rz[9] = {cq, -s, 0, s, cq, 0, 0, 0, 1};
        R W[9];
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) {
                R acc = 0;
                for (int j = 0; j < 3; ++j) acc += (R)Rf[3 * r + j] * Rz[3 * j + k];
                W[3 * r + k] = acc;
            }
        R N[12];
        for (int r = 0; r < 3; ++r) {
            for (int k = 0; k < 3; ++k)
                N[4 * r + k] = T[4 * r] * W[k] + T[4 * r + 1] * W[3 + k] + T[4 * r + 2] * W[6 + k];
            N[4 * r + 3] = T[4 * r] * (R)ORC_JOINT_P[i][0] + T[4 * r + 1] * (R)ORC_JOINT_P[i][1] +
                           T[4 * r + 2] * (R)ORC_JOINT_P[i][2] + T[4 * r + 3];
        }
        memcpy(T, N, sizeof(T));
        memcpy(frames[i], T, sizeof(T));
    }
}

/* end-effector xyz + roll/pitch/yaw (grid end_effector_positions_inner :2015-2090) */
void ORC(fk)(const R *q, R *ee)
{
    R F[ORC_NJ][12];
    fk_frames(q, F);
    const R *T = F[ORC_NJ - 1];
    ee[0] = T[3]; ee[1] = T[7]; ee[2] = T[11];
    ee[3] = (R)atan2(T[9], T[10]);
    ee[4] = (R)-atan2(T[8], sqrt(T[9] * T[9] + T[10] * T[10]));
    ee[5] = (R)atan2(T[4], T[0]);
}

/* d(ee xyz)/dq_j = z_j x (p - o_j); layout dee[6*j + {0,1,2}], rpy slots 0
 * (grid end_effector_positions_gradient_inner :2255; only xyz is consumed,
 * iiwa_eepos_plant.cuh:339) */
void ORC(fk_grad)(const R *q, R *dee)
{
    R F[ORC_NJ][12];
    fk_frames(q, F);
    const R *T = F[ORC_NJ - 1];
    R p[3] = {T[3], T[7], T[11]};
    for (int j = 0; j < ORC_NJ; ++j) {
        R z[3] = {F[j][2], F[j][6], F[j][10]};
        R d[3] = {p[0] - F[j][3], p[1] - F[j][7], p[2] - F[j][11]};
        R o[3];
        cross3(z, d, o);
        for (int k = 0; k < 3; ++k) dee[6 * j + k] = o[k];
        for (int k = 3; k < 6; ++k) dee[6 * j + k] = 0;
    }
}

/* ------------------------------------------------------------------------ */
/* integrator: integrator.cuh:25-126                                          */
/* ------------------------------------------------------------------------ */

static void step_state(int type, R dt, const R *x, const R *qdd, R *xn)
{
    for (int i = 0; i < 7; ++i) {
        if (type == 0) {
            xn[i] = x[i] + dt * x[7 + i];
            xn[7 + i] = x[7 + i] + dt * qdd[i];
        } else {
            xn[7 + i] = x[7 + i] + dt * qdd[i];
            xn[i] = x[i] + dt * xn[7 + i];
        }
    }
}

/* exec_integrator_gradient (integrator.cuh:85-126); A 14x14, B 14x7 col-major */
static void integrator_gradient(int type, R dt, const R *dqdd, R *A, R *B)
{
    for (int c = 0; c < 14; ++c)
        for (int r = 0; r < 14; ++r) {
            R val;
            if (type == 0) {
                val = (R)(r == c);
                if (r < 7 && r == c - 7) val += dt;
                if (r >= 7) val += dt * dqdd[c * 7 + r - 7];
            } else {
                int rq = r % 7;
                R dtv = (r == rq) ? dt : (R)1;
                val = (R)(r == c) + dt * (R)(r == c - 7) + dt * dqdd[c * 7 + rq] * dtv;
            }
            A[r + 14 * c] = val;
        }
    for (int c = 0; c < 7; ++c)
        for (int r = 0; r < 14; ++r) {
            R val;
            if (type == 0) {
                val = 0;
                if (r >= 7) val = dt * dqdd[(14 + c) * 7 + r - 7];
            } else {
                int rq = r % 7;
                R dtv = (r == rq) ? dt : (R)1;
                val = dt * dqdd[98 + c * 7 + rq] * dtv;
            }
            B[r + 14 * c] = val;
        }
}

/* ------------------------------------------------------------------------ */
/* tracking cost: iiwa_eepos_plant.cuh:240-405                               */
/* ------------------------------------------------------------------------ */

/* trackingcost (:240-290) at one knot; with_r selects the control term */
static R tracking_cost(const orc_params *P, const R *x, const R *u, int with_r, const R *goal)
{
    R acc = 0;
    for (int i = 0; i < 7; ++i) acc += (R)0.5 * ((R)P->qd_cost * x[7 + i] * x[7 + i]);
    if (with_r)
        for (int i = 0; i < 7; ++i) acc += (R)0.5 * ((R)P->r_cost * u[i] * u[i]);
    R ee[6];
    ORC(fk)(x, ee);
    for (int d = 0; d < 3; ++d) {
        R e = ee[d] - goal[d];
        acc += (R)0.5 * (R)P->q_ee * e * e;
    }
    return acc;
}

/* trackingCostGradientAndHessian (:295-378): Q = [q_q q_q^T, 0; 0, QD I], R = R_cost I */
static void cost_grad_hess(const orc_params *P, const R *x, const R *u, const R *goal, R *Q, R *qv,
                           R *Rm, R *rv)
{
    R ee[6], J[42];
    ORC(fk)(x, ee);
    ORC(fk_grad)(x, J);
    R e[3] = {ee[0] - goal[0], ee[1] - goal[1], ee[2] - goal[2]};
    for (int i = 0; i < 7; ++i)
        qv[i] = (R)P->q_ee * (J[6 * i] * e[0] + J[6 * i + 1] * e[1] + J[6 * i + 2] * e[2]);
    for (int i = 7; i < 14; ++i) qv[i] = (R)P->qd_cost * x[i];
    for (int i = 0; i < 14; ++i)
        for (int j = 0; j < 14; ++j)
            Q[i * 14 + j] = (i < 7 && j < 7) ? qv[i] * qv[j] : ((i == j) ? (R)P->qd_cost : (R)0);
    if (Rm) {
        for (int i = 0; i < 7; ++i) rv[i] = (R)P->r_cost * u[i];
        for (int i = 0; i < 7; ++i)
            for (int j = 0; j < 7; ++j) Rm[i * 7 + j] = (i == j) ? (R)P->r_cost : (R)0;
    }
}

/* ------------------------------------------------------------------------ */
/* KKT formation: schur.cuh:391-524                                           */
/* ------------------------------------------------------------------------ */

void ORC(form_kkt)(const orc_params *P, int N, const R *xu, const R *goal, const R *xs, R *G, R *C,
                   R *g, R *c)
{
    const R dt = (R)P->dt;
    for (int k = 0; k < N - 1; ++k) {
        const R *x = xu + NX * k, *u = x + NS, *xn = xu + NX * (k + 1);
        R qdd[7], dfdu[147], A[SS], B[SC], xp[14];
        ORC(fd_grad)(x, x + 7, u, qdd, dfdu);
        step_state(P->integrator, dt, x, qdd, xp);
        integrator_gradient(P->integrator, dt, dfdu, A, B);
        R *Qk = G + GSTRIDE * k, *Rk = Qk + SS, *qk = g + NX * k, *rk = qk + NS;
        cost_grad_hess(P, x, u, goal + 6 * k, Qk, qk, Rk, rk);
        if (k == N - 2) {
            const R *xt = P->ref_terminal ? x : xn;
            const R *gt = goal + 6 * (k + 1);
            R alias[3];
            if (P->ref_terminal) {
                /* the reference's kernel reserves 6 shared floats for the goal but copies 12
                 * (schur.cuh:413-425), so goal_{k+1} lands on Q_k's first row, which the first
                 * cost call overwrites with q_0 q_j before the terminal call reads its target
                 * (iiwa_eepos_plant.cuh:396-401): the terminal target is Q_k[0][0..2] */
                alias[0] = Qk[0];
                alias[1] = Qk[1];
                alias[2] = Qk[2];
                gt = alias;
            }
            cost_grad_hess(P, xt, NULL, gt, G + GSTRIDE * (k + 1), g + NX * (k + 1), NULL, NULL);
            for (int i = 0; i < NS; ++i) c[i] = xu[i] - xs[i];
        }
        for (int i = 0; i < SS; ++i) C[CSTRIDE * k + i] = -A[i];
        for (int i = 0; i < SC; ++i) C[CSTRIDE * k + SS + i] = -B[i];
        for (int i = 0; i < NS; ++i) c[NS * (k + 1) + i] = xn[i] - xp[i];
    }
}

/* ------------------------------------------------------------------------ */
/* Schur complement and block-Jacobi preconditioner: oldschur.cuh:518-963    */
/* ------------------------------------------------------------------------ */

/* oldschur.cuh:100-149 (mat_mat_prod), sum order kept */
static void mat_mat(R *out, const R *A, const R *B, int Ar, int Ac, int Br, int Bc, int transB)
{
    if (!transB) {
        for (int col = 0; col < Bc; ++col)
            for (int row = 0; row < Ar; ++row) {
                R res = 0;
                for (int t = 0; t < Ac; ++t) res += A[t * Ar + row] * B[col * Br + t];
                out[col * Ar + row] = res;
            }
    } else {
        for (int col = 0; col < Br; ++col)
            for (int row = 0; row < Ar; ++row) {
                R res = 0;
                for (int t = 0; t < Ac; ++t) res += A[t * Ar + row] * B[t * Br + col];
                out[col * Ar + row] = res;
            }
    }
}
/* oldschur.cuh:86-97 (mat_vec_prod) */
static void mat_vec(int rows, int cols, const R *M, const R *v, R *o)
{
    for (int r = 0; r < rows; ++r) {
        R res = 0;
        for (int c = 0; c < cols; ++c) res += M[r + c * rows] * v[c];
        o[r] = res;
    }
}
/*
 * Gauss-Jordan without pivoting on [A | I] (dim x 2dim, col-major), as
 * oldschur.cuh:214-242 (style 0: multiply by 1/pivot) and :245-332 (style 1:
 * divide by pivot).  Returns A^{-1} in the right half.
 */
static void gauss_jordan(R *M, int dim, int style)
{
    R tmp[2 * 14 + 1];
    for (int piv = 0; piv < dim; ++piv) {
        int pco = piv * dim;
        for (int i = 0; i < dim; ++i) tmp[i] = M[i + pco];
        for (int i = 0; i <= dim; ++i) tmp[dim + i] = M[piv + pco + i * dim];
        R pvInv = (R)1 / M[piv + pco];
        R pv = tmp[piv];
        for (int ind = 0; ind < dim * (dim + 1); ++ind) {
            int row = ind % dim, col = ind / dim;
            R *e = &M[pco + ind];
            if (style == 0) {
                if (row == piv) *e *= pvInv;
                else *e -= tmp[row] * pvInv * tmp[dim + col];
            } else {
                if (row == piv) *e /= pv;
                else *e -= tmp[row] / pv * tmp[dim + col];
            }
        }
    }
}
static void invert_into(const R *A, int dim, R *Ainv, int style)
{
    R M[14 * 28];
    for (int c = 0; c < dim; ++c)
        for (int r = 0; r < dim; ++r) {
            M[r + dim * c] = A[r + dim * c];
            M[r + dim * (dim + c)] = (R)(r == c);
        }
    gauss_jordan(M, dim, style);
    memcpy(Ainv, M + dim * dim, sizeof(R) * dim * dim);
}

/*
 * gato_form_schur_jacobi_inner (oldschur.cuh:518-963).  Ginv receives
 * (Q_k + rho I)^{-1} and (R_k + rho I)^{-1} in the G layout (the reference
 * overwrites G in place, schur.cuh:236-256; here it is a separate buffer).
 * Pinv off-diagonal blocks and S[0].left / S[N-1].right are zero.
 */
void ORC(form_schur)(int N, R rho, const R *G, const R *C, const R *g, const R *c, R *S, R *Pinv,
                     R *gamma, R *Ginv)
{
    memset(S, 0, sizeof(R) * 3 * SS * N);
    memset(Pinv, 0, sizeof(R) * 3 * SS * N);
    for (int k = 0; k < N; ++k) {
        if (k == 0) {
            R Q0[SS], Q0i[SS], gk[NS];
            memcpy(Q0, G, sizeof(Q0));
            for (int i = 0; i < NS; ++i) Q0[i + NS * i] += rho;
            for (int i = 0; i < SS; ++i) Pinv[SS + i] = -Q0[i];
            invert_into(Q0, NS, Q0i, 1);
            mat_vec(NS, NS, Q0i, g, gk);
            for (int i = 0; i < SS; ++i) S[SS + i] = -Q0i[i];
            for (int i = 0; i < NS; ++i) gamma[i] = -gk[i];
            if (N == 1) memcpy(Ginv, Q0i, sizeof(Q0i));
            continue;
        }
        const R *Ak = C + CSTRIDE * (k - 1), *Bk = Ak + SS;
        R Qk[SS], Qkp1[SS], Rk[CC], Qki[SS], Qkp1i[SS], Rki[CC];
        memcpy(Qk, G + GSTRIDE * (k - 1), sizeof(Qk));
        memcpy(Qkp1, G + GSTRIDE * k, sizeof(Qkp1));
        memcpy(Rk, G + GSTRIDE * (k - 1) + SS, sizeof(Rk));
        const R *qk = g + NX * (k - 1), *qkp1 = g + NX * k, *rk = g + NX * (k - 1) + NS;
        for (int i = 0; i < NS; ++i) { Qk[i + NS * i] += rho; Qkp1[i + NS * i] += rho; }
        for (int i = 0; i < NC; ++i) Rk[i + NC * i] += rho;
        invert_into(Qk, NS, Qki, 1);
        invert_into(Qkp1, NS, Qkp1i, 1);
        invert_into(Rk, NC, Rki, 1);
        memcpy(Ginv + GSTRIDE * (k - 1), Qki, sizeof(Qki));
        memcpy(Ginv + GSTRIDE * (k - 1) + SS, Rki, sizeof(Rki));
        if (k == N - 1) memcpy(Ginv + GSTRIDE * k, Qkp1i, sizeof(Qkp1i));
        R phi[SS], BRi[SC], gk[NS], t1[NS], t2[NS], theta[SS], tmp[SS], thetai[SS];
        mat_mat(phi, Ak, Qki, NS, NS, NS, NS, 0);
        mat_mat(BRi, Bk, Rki, NS, NC, NC, NC, 0);
        mat_vec(NS, NS, Qkp1i, qkp1, gk);
        for (int i = 0; i < NS; ++i) gk[i] -= c[NS * k + i];
        mat_vec(NS, NS, phi, qk, t1);
        mat_vec(NS, NC, BRi, rk, t2);
        for (int i = 0; i < NS; ++i) gk[i] += t2[i] + t1[i];
        mat_mat(theta, phi, Ak, NS, NS, NS, NS, 1);
        for (int i = 0; i < SS; ++i) theta[i] += Qkp1i[i];
        mat_mat(tmp, BRi, Bk, NS, NC, NS, NC, 1);
        for (int i = 0; i < SS; ++i) theta[i] += tmp[i];
        R *row = S + 3 * SS * k;
        for (int i = 0; i < SS; ++i) { row[i] = -phi[i]; row[SS + i] = -theta[i]; }
        invert_into(theta, NS, thetai, 0);
        for (int i = 0; i < SS; ++i) Pinv[3 * SS * k + SS + i] = -thetai[i];
        for (int i = 0; i < NS; ++i) gamma[NS * k + i] = -gk[i];
        R *prev_right = S + 3 * SS * (k - 1) + 2 * SS;
        for (int cc = 0; cc < NS; ++cc)
            for (int r = 0; r < NS; ++r) prev_right[r + NS * cc] = -phi[cc + NS * r];
    }
}

/*
 * CSC (upper triangle, == CSR lower triangle) pattern of the Schur matrix:
 * prep_csr (utils.cuh:84-118).  nnz = 196(N-1) + 105N.
 */
void ORC(csc_pattern)(int N, int32_t *col_ptr, int32_t *row_ind)
{
    const int tri = (NS + 1) * NS / 2, brow = SS + tri;
    col_ptr[0] = 0;
    for (int b = 0; b < N; ++b)
        for (int r = 0; r < NS; ++r) {
            int off = (b > 0) * tri + (b > 0) * (b - 1) * brow + (b > 0) * r * NS + (r + 1) * r / 2;
            int len = (b > 0) * NS + r + 1;
            col_ptr[b * NS + r + 1] = off + len;
            for (int cidx = 0; cidx < len; ++cidx) row_ind[off + cidx] = (b > 0) * (b - 1) * NS + cidx;
        }
}

/* values of that CSC from S (store_block_csr_lowertri, utils.cuh:55-81) */
void ORC(csc_values)(int N, const R *S, float *val)
{
    const int tri = (NS + 1) * NS / 2, brow = SS + tri;
    for (int b = 0; b < N; ++b) {
        const R *left = S + 3 * SS * b, *diag = left + SS;
        for (int r = 0; r < NS; ++r) {
            int off = (b > 0) * tri + (b > 0) * (b - 1) * brow + (b > 0) * r * NS + (r + 1) * r / 2;
            if (b > 0)
                for (int cidx = 0; cidx < NS; ++cidx) val[off + cidx] = (float)left[r + cidx * NS];
            for (int cidx = 0; cidx <= r; ++cidx)
                val[off + (b > 0) * NS + cidx] = (float)diag[r + cidx * NS];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* linear solves                                                             */
/* ------------------------------------------------------------------------ */

static void s_matvec(int N, const R *S, const R *x, R *y)
{
    for (int k = 0; k < N; ++k) {
        const R *row = S + 3 * SS * k;
        for (int r = 0; r < NS; ++r) {
            R acc = 0;
            if (k > 0)
                for (int cc = 0; cc < NS; ++cc) acc += row[r + NS * cc] * x[NS * (k - 1) + cc];
            for (int cc = 0; cc < NS; ++cc) acc += row[SS + r + NS * cc] * x[NS * k + cc];
            if (k < N - 1)
                for (int cc = 0; cc < NS; ++cc) acc += row[2 * SS + r + NS * cc] * x[NS * (k + 1) + cc];
            y[NS * k + r] = acc;
        }
    }
}
/* y = Pinv x for the block-tridiagonal Pinv (3 blocks per row).  The block-Jacobi Pinv has zero
 * off-diagonal blocks, whose terms are skipped, so its products are unchanged; the stair
 * preconditioner (form_ss) fills them. */
static void p_apply(int N, const R *Pinv, const R *x, R *y)
{
    for (int k = 0; k < N; ++k) {
        const R *d = Pinv + 3 * SS * k + SS;
        const R *lft = Pinv + 3 * SS * k, *rgt = Pinv + 3 * SS * k + 2 * SS;
        int has_l = 0, has_r = 0;
        for (int i = 0; i < SS && k > 0; ++i) has_l |= lft[i] != 0;
        for (int i = 0; i < SS && k < N - 1; ++i) has_r |= rgt[i] != 0;
        for (int r = 0; r < NS; ++r) {
            R acc = 0;
            for (int cc = 0; cc < NS; ++cc) acc += d[r + NS * cc] * x[NS * k + cc];
            if (has_l)
                for (int cc = 0; cc < NS; ++cc) acc += lft[r + NS * cc] * x[NS * (k - 1) + cc];
            if (has_r)
                for (int cc = 0; cc < NS; ++cc) acc += rgt[r + NS * cc] * x[NS * (k + 1) + cc];
            y[NS * k + r] = acc;
        }
    }
}

/*
 * Preconditioned conjugate gradient on S lambda = gamma with the block-Jacobi
 * preconditioner Pinv, warm-started from lambda.  The reference launches the
 * GPU-PCG kernel here (toplevel.cuh:135-157, 292-294); its source is not in
 * the reference tree, so this follows the published PCG recurrence with
 * FP64 dot products.  exit_mode 0: ||r||_2 <= tol ||gamma||_2;
 * exit_mode 1: |r^T Pinv r| < tol.  Returns iterations; *maxiter_exit = 1 if
 * the budget ran out.
 */
int ORC(pcg)(int N, const R *S, const R *Pinv, const R *gamma, R *lambda, int max_iter, double tol,
             int exit_mode, int *maxiter_exit)
{
    const int n = NS * N;
    R *r = malloc(sizeof(R) * n), *z = malloc(sizeof(R) * n), *p = malloc(sizeof(R) * n),
      *v = malloc(sizeof(R) * n);
    s_matvec(N, S, lambda, v);
    double eta = 0, rr = 0, gg = 0;
    for (int i = 0; i < n; ++i) { r[i] = gamma[i] - v[i]; gg += (double)gamma[i] * gamma[i]; }
    p_apply(N, Pinv, r, z);
    for (int i = 0; i < n; ++i) { p[i] = z[i]; eta += (double)r[i] * z[i]; rr += (double)r[i] * r[i]; }
    int it = 0, conv;
    conv = exit_mode == 0 ? (sqrt(rr) <= tol * sqrt(gg)) : (fabs(eta) < tol);
    while (!conv && it < max_iter) {
        s_matvec(N, S, p, v);
        double pv = 0;
        for (int i = 0; i < n; ++i) pv += (double)p[i] * v[i];
        R alpha = (R)(eta / pv);
        for (int i = 0; i < n; ++i) { lambda[i] += alpha * p[i]; r[i] -= alpha * v[i]; }
        p_apply(N, Pinv, r, z);
        double en = 0;
        rr = 0;
        for (int i = 0; i < n; ++i) { en += (double)r[i] * z[i]; rr += (double)r[i] * r[i]; }
        ++it;
        conv = exit_mode == 0 ? (sqrt(rr) <= tol * sqrt(gg)) : (fabs(en) < tol);
        if (conv) break;
        R beta = (R)(en / eta);
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        eta = en;
    }
    if (maxiter_exit) *maxiter_exit = !conv;
    free(r); free(z); free(p); free(v);
    return it;
}

/*
 * FP64 block-tridiagonal (banded, half-bandwidth 27) Cholesky solve of
 * (-S) lambda = (-gamma); the FP64 reference solution of the Schur system.
 */
int ORC(banded_cholesky)(int N, const R *S, const R *gamma, double *lambda)
{
    double *L = calloc((size_t)SS * N, sizeof(double)), *E = calloc((size_t)SS * N, sizeof(double));
    double *y = malloc(sizeof(double) * NS * N);
    int rc = 0;
    for (int k = 0; k < N && !rc; ++k) {
        double D[SS];
        for (int i = 0; i < SS; ++i) D[i] = -(double)S[3 * SS * k + SS + i];
        if (k > 0) {
            /* E_k = B_k L_{k-1}^{-T} where B_k = -S[k].left; solve X L^T = B rowwise */
            double Bk[SS];
            for (int i = 0; i < SS; ++i) Bk[i] = -(double)S[3 * SS * k + i];
            const double *Lp = L + SS * (k - 1);
            double *Ek = E + SS * k;
            for (int r = 0; r < NS; ++r)
                for (int j = 0; j < NS; ++j) {
                    double s = Bk[r + NS * j];
                    for (int t = 0; t < j; ++t) s -= Ek[r + NS * t] * Lp[j + NS * t];
                    Ek[r + NS * j] = s / Lp[j + NS * j];
                }
            for (int cc = 0; cc < NS; ++cc)
                for (int r = 0; r < NS; ++r) {
                    double s = 0;
                    for (int t = 0; t < NS; ++t) s += Ek[r + NS * t] * Ek[cc + NS * t];
                    D[r + NS * cc] -= s;
                }
        }
        double *Lk = L + SS * k;
        for (int j = 0; j < NS; ++j) {
            double d = D[j + NS * j];
            for (int t = 0; t < j; ++t) d -= Lk[j + NS * t] * Lk[j + NS * t];
            if (!(d > 0)) { rc = -1; break; }
            double ljj = sqrt(d);
            Lk[j + NS * j] = ljj;
            for (int i = j + 1; i < NS; ++i) {
                double s = D[i + NS * j];
                for (int t = 0; t < j; ++t) s -= Lk[i + NS * t] * Lk[j + NS * t];
                Lk[i + NS * j] = s / ljj;
            }
        }
    }
    if (!rc) {
        for (int k = 0; k < N; ++k) {
            const double *Lk = L + SS * k, *Ek = E + SS * k;
            for (int r = 0; r < NS; ++r) {
                double s = -(double)gamma[NS * k + r];
                if (k > 0)
                    for (int t = 0; t < NS; ++t) s -= Ek[r + NS * t] * y[NS * (k - 1) + t];
                for (int t = 0; t < r; ++t) s -= Lk[r + NS * t] * y[NS * k + t];
                y[NS * k + r] = s / Lk[r + NS * r];
            }
        }
        for (int k = N - 1; k >= 0; --k) {
            const double *Lk = L + SS * k;
            for (int r = NS - 1; r >= 0; --r) {
                double s = y[NS * k + r];
                if (k < N - 1) {
                    const double *En = E + SS * (k + 1);
                    for (int t = 0; t < NS; ++t) s -= En[t + NS * r] * lambda[NS * (k + 1) + t];
                }
                for (int t = r + 1; t < NS; ++t) s -= Lk[t + NS * r] * lambda[NS * k + t];
                lambda[NS * k + r] = s / Lk[r + NS * r];
            }
        }
    }
    free(L); free(E); free(y);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* dz recovery: oldschur.cuh:966-1105                                         */
/* ------------------------------------------------------------------------ */

void ORC(compute_dz)(int N, const R *Ginv, const R *C, const R *g, const R *lambda, R *dz)
{
    for (int k = 0; k < N; ++k) {
        /* state row */
        R s[NS], o[NS];
        if (k != N - 1) {
            const R *At = C + CSTRIDE * k;
            for (int i = 0; i < NS; ++i) {
                R res = 0;
                for (int t = 0; t < NS; ++t) res += At[i * NS + t] * lambda[NS * (k + 1) + t];
                s[i] = res;
            }
        } else {
            for (int i = 0; i < NS; ++i) s[i] = 0;
        }
        for (int i = 0; i < NS; ++i) s[i] = lambda[NS * k + i] + s[i];
        for (int i = 0; i < NS; ++i) s[i] = g[NX * k + i] - s[i];
        mat_vec(NS, NS, Ginv + GSTRIDE * k, s, o);
        for (int i = 0; i < NS; ++i) dz[NX * k + i] = o[i];
        if (k == N - 1) break;
        /* control row */
        const R *Bt = C + CSTRIDE * k + SS;
        R sc[NC], oc[NC];
        for (int i = 0; i < NC; ++i) {
            R res = 0;
            for (int t = 0; t < NS; ++t) res += Bt[i * NS + t] * lambda[NS * (k + 1) + t];
            sc[i] = res;
        }
        for (int i = 0; i < NC; ++i) sc[i] = g[NX * k + NS + i] - sc[i];
        mat_vec(NC, NC, Ginv + GSTRIDE * k + SS, sc, oc);
        for (int i = 0; i < NC; ++i) dz[NX * k + NS + i] = oc[i];
    }
}

/* ------------------------------------------------------------------------ */
/* merit: merit.cuh:16-145, integrator.cuh:187-219                            */
/* ------------------------------------------------------------------------ */

/*
 * Merit at xu + alpha dz (dz may be NULL for alpha = 0).  line_search = 1 is
 * ls_gato_compute_merit (merit.cuh:16-94): the last knot adds
 * ||x_0 + alpha dz_0 - x_s||_1; line_search = 0 is compute_merit
 * (merit.cuh:99-145): the last knot's defect term is 0.  Also returns the
 * per-knot point merits when knot_out is not NULL.
 */
R ORC(merit)(const orc_params *P, int N, const R *xu, const R *dz, R alpha, const R *goal, const R *xs,
             int line_search, R *knot_out)
{
    R total = 0;
    for (int k = 0; k < N; ++k) {
        const int last = (k == N - 1);
        const int len = last ? NS : 2 * NS + NC;
        R loc[2 * NS + NC];
        for (int i = 0; i < len; ++i) loc[i] = xu[NX * k + i] + (dz ? alpha * dz[NX * k + i] : (R)0);
        R J = tracking_cost(P, loc, loc + NS, !last, goal + 6 * k);
        R ck = 0;
        if (!last) {
            R qdd[7], xp[14];
            ORC(fd)(loc, loc + 7, loc + NS, qdd);
            step_state(P->integrator, (R)P->dt, loc, qdd, xp);
            for (int i = 0; i < NS; ++i) ck += (R)fabs(loc[NX + i] - xp[i]);
        } else if (line_search) {
            for (int i = 0; i < NS; ++i)
                ck += (R)fabs((xu[i] + (dz ? alpha * dz[i] : (R)0)) - xs[i]);
        }
        R pm = J + (R)P->mu * ck;
        if (knot_out) knot_out[k] = pm;
        total += pm;
    }
    return total;
}

/* ------------------------------------------------------------------------ */
/* QDLDL-API LDL^T (declared in ldl.c)                                        */
/* ------------------------------------------------------------------------ */
int orc_ldl_solve(int n, const int32_t *Ap, const int32_t *Ai, const float *Ax, const float *b, float *x);

/* ------------------------------------------------------------------------ */
/* SQP loop: toplevel.cuh:24-503 (wall-clock cap removed)                     */
/* ------------------------------------------------------------------------ */

int ORC(sqp_solve)(const orc_params *P, const orc_solver *SV, int N, const R *goal, R *lambda, R *xu,
                   R *rho_io, R rho_reset, orc_stats *st, int32_t *pcg_iters_out)
{
    const int nxu = NX * N - NC, n = NS * N;
    R xs[NS];
    memcpy(xs, xu, sizeof(xs)); /* toplevel.cuh:110 */
    R *G = malloc(sizeof(R) * (GSTRIDE * N)), *Cm = malloc(sizeof(R) * (CSTRIDE * N)),
      *g = malloc(sizeof(R) * (NX * N)), *c = malloc(sizeof(R) * n), *S = malloc(sizeof(R) * 3 * SS * N),
      *Pv = malloc(sizeof(R) * 3 * SS * N), *gam = malloc(sizeof(R) * n), *Gi = malloc(sizeof(R) * (GSTRIDE * N)),
      *dz = malloc(sizeof(R) * (NX * N));
    int32_t *cp = NULL, *ri = NULL;
    float *val = NULL, *bf = NULL, *xf = NULL;
    double *ld = NULL;
    const int nnz = SS * (N - 1) + 105 * N;
    if (SV->linsys == 1) {
        cp = malloc(sizeof(int32_t) * (n + 1)); ri = malloc(sizeof(int32_t) * nnz);
        val = malloc(sizeof(float) * nnz); bf = malloc(sizeof(float) * n); xf = malloc(sizeof(float) * n);
        ORC(csc_pattern)(N, cp, ri);
    } else if (SV->linsys == 2) {
        ld = malloc(sizeof(double) * n);
    }
    memset(st, 0, sizeof(*st));
    R rho = *rho_io, drho = 1, f = (R)SV->rho_factor, rmax = (R)SV->rho_max, rmin = (R)SV->rho_min;
    R merit0 = ORC(merit)(P, N, xu, NULL, 0, goal, xs, 0, NULL);
    int rc = 0;
    for (int it = 0; it < SV->sqp_max_iter; ++it) {
        ORC(form_kkt)(P, N, xu, goal, xs, G, Cm, g, c);
        ORC(form_schur)(N, rho, G, Cm, g, c, S, Pv, gam, Gi);
        if (SV->linsys == 0) {
            int mx = 0;
            int pit = ORC(pcg)(N, S, Pv, gam, lambda, SV->pcg_max_iter, SV->pcg_tol, SV->pcg_exit_mode, &mx);
            if (pcg_iters_out) pcg_iters_out[st->linsys_count] = pit;
            st->pcg_iters_total += pit;
            st->pcg_maxiter_count += mx;
        } else if (SV->linsys == 1) {
            ORC(csc_values)(N, S, val);
            for (int i = 0; i < n; ++i) bf[i] = (float)gam[i];
            if (orc_ldl_solve(n, cp, ri, val, bf, xf) < 0) rc = -1;
            for (int i = 0; i < n; ++i) lambda[i] = (R)xf[i];
        } else {
            if (ORC(banded_cholesky)(N, S, gam, ld) < 0) rc = -1;
            for (int i = 0; i < n; ++i) lambda[i] = (R)ld[i];
        }
        st->linsys_count++;
        ORC(compute_dz)(N, Gi, Cm, g, lambda, dz);
        R merits[8], minm = merit0;
        int best = 0;
        for (int p = 0; p < 8; ++p) {
            R alpha = (R)(-1.0 / (double)(1 << p));
            merits[p] = ORC(merit)(P, N, xu, dz, alpha, goal, xs, 1, NULL);
        }
        for (int i = 0; i < 8; ++i)
            if (merits[i] < minm) { minm = merits[i]; best = i; }
        if (minm == merit0) {
            drho = (drho * f > f) ? drho * f : f;
            rho = (rho * drho > rmin) ? rho * drho : rmin;
            st->sqp_iters++;
            st->ls_fail_count++;
            if (rho > rmax) { st->rho_exit = 1; rho = rho_reset; break; }
            continue;
        }
        R alpha = (R)(-1.0 / (double)(1 << best));
        drho = (drho / f < 1 / f) ? drho / f : 1 / f;
        rho = (rho * drho > rmin) ? rho * drho : rmin;
        for (int i = 0; i < nxu; ++i) xu[i] += alpha * dz[i];
        st->sqp_iters++;
        merit0 = minm;
    }
    st->merit_final = merit0;
    st->rho_final = rho;
    *rho_io = rho;
    free(G); free(Cm); free(g); free(c); free(S); free(Pv); free(gam); free(Gi); free(dz);
    free(cp); free(ri); free(val); free(bf); free(xf); free(ld);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* plant simulation and the MPC tracking loop                                */
/* ------------------------------------------------------------------------ */

/* One explicit-Euler plant step x <- x + h [qd; FD(q, qd, u)]: simple_integrator_kernel
 * (integrator.cuh:306-331), which always integrates with type 0. */
static void plant_step(R *x, const R *u, R h)
{
    R qdd[7], xn[NS];
    ORC(fd)(x, x + 7, u, qdd);
    step_state(0, h, x, qdd, xn);
    memcpy(x, xn, sizeof(xn));
}

/* Control slot applied at plant time t (s): floor(t / timestep) (integrator.cuh:380-388),
 * clamped to the last control of the horizon. */
static int control_slot(double t, double timestep, int N)
{
    unsigned co = (unsigned)(t / timestep);
    return (int)co > N - 2 ? N - 2 : (int)co;
}

/* simple_simulate (integrator.cuh:365-398): advances x_s by sim_time_us of plant time in
 * steps of sim_step (a float, as the reference's T), starting time_offset_us into the
 * horizon xu, then one final step of the remainder fmod(sim_time, sim_step). */
void ORC(simulate)(int N, R *xs, const R *xu, double timestep, double time_offset_us, double sim_time_us,
                   double sim_step)
{
    const double t0 = time_offset_us * 1e-6, sim_time = sim_time_us * 1e-6;
    const float h = (float)sim_step;
    int co = control_slot(t0, timestep, N);
    const unsigned n = (unsigned)(sim_time / (double)h);
    for (unsigned step = 0; step < n; ++step) {
        co = control_slot(t0 + (double)((float)step * h), timestep, N);
        plant_step(xs, xu + NX * co + NS, (R)h);
    }
    const R hl = (R)(float)fmod(sim_time, (double)h);
    plant_step(xs, xu + NX * co + NS, hl);
}

/* sum_{i<3} |p(q)_i - goal_i| (toplevel.cuh:674-681) */
static R tracking_error(const R *xs, const R *goal)
{
    R ee[6];
    ORC(fk)(xs, ee);
    R e = 0;
    for (int i = 0; i < 3; ++i) e += (R)fabs((double)(ee[i] - goal[i]));
    return e;
}

/* track (toplevel.cuh:507-796) with CONST_UPDATE_FREQ 1, ADD_NOISE 0: each control update
 * solves the SQP from the shifted previous solution, simulates the plant for sim_period_us
 * with the previous solution's controls, and once per timestep (SHIFT_THRESHOLD) records the
 * tracking error and shifts xu, the goal window and lambda one knot along the trajectory.
 * Trajectory rows: eePos_traj [6 S], xu_traj [21 S] (x_k, u_k per row, runme.cu:145-161).
 * xs (14) is the plant state, in/out; errors receives one entry per shift (S at most). */
int ORC(track)(const orc_params *P, const orc_solver *SV, const orc_track_cfg *TC, int N, int S, const R *eePos_traj,
               const R *xu_traj, R *xs, R *errors, orc_track_stats *ts)
{
    const int traj_len = NX * N - NC;
    const double dt = (double)(float)P->dt;
    const double thr = (double)(float)TC->shift_threshold;
    R *xu = malloc(sizeof(R) * NX * N), *xu_old = malloc(sizeof(R) * NX * N), *goal = malloc(sizeof(R) * 6 * N),
      *lambda = calloc((size_t)NS * N, sizeof(R));
    memcpy(xu, xu_traj, sizeof(R) * traj_len);      /* toplevel.cuh:550-552 */
    memcpy(xu_old, xu_traj, sizeof(R) * traj_len);
    memcpy(goal, eePos_traj, sizeof(R) * 6 * N);
    memset(ts, 0, sizeof(*ts));
    R rho = (R)1e-3;
    orc_stats st;
    int rc = 0;
    if (TC->jitter_solves > 0) { /* toplevel.cuh:581-592 */
        orc_solver jv = *SV;
        jv.pcg_tol = 1e-11;
        jv.pcg_max_iter = 10000;
        for (int j = 0; j < TC->jitter_solves && rc == 0; ++j) {
            rc = ORC(sqp_solve)(P, &jv, N, goal, lambda, xu, &rho, (R)1e-3, &st, NULL);
            memcpy(xu, xu_traj, sizeof(R) * traj_len);
        }
        rho = (R)1e-3;
    }
    double time_since = 0.0, prev_sim = 0.0;
    int shifted = 0, traj_offset = 0, step;
    for (step = 0; step < TC->max_control_updates && rc == 0; ++step) {
        if (traj_offset == S) break;
        rc = ORC(sqp_solve)(P, SV, N, goal, lambda, xu, &rho, (R)TC->rho_reset, &st, NULL);
        ts->sqp_iters_total += st.sqp_iters;
        ts->pcg_iters_total += st.pcg_iters_total;
        ts->ls_fail_total += st.ls_fail_count;
        ts->rho_exits += st.rho_exit;
        const double sim = TC->sim_period_us;
        ORC(simulate)(N, xs, xu_old, dt, prev_sim, sim, TC->sim_step);
        memcpy(xu_old, xu, sizeof(R) * traj_len);
        time_since += sim * 1e-6;
        if (!shifted && time_since > thr) {
            errors[traj_offset] = tracking_error(xs, goal);
            traj_offset++;
            /* just_shift (integrator.cuh:299-304): knot k <- knot k+1 (x_{N-1} -> x_{N-2}; u_{N-2} kept) */
            memmove(xu, xu + NX, sizeof(R) * (NX * (N - 2) + NS));
            if (traj_offset + N < S) {
                memcpy(xu + traj_len - NX, xu_traj + NX * traj_offset - NC, sizeof(R) * NX);
            } else {
                memcpy(xu + traj_len - NS, xu_traj + NX * (S - 1), sizeof(R) * 7);
                memset(xu + traj_len - 7, 0, sizeof(R) * 7);
                memset(xu + traj_len - NX, 0, sizeof(R) * NC);
            }
            memmove(goal, goal + 6, sizeof(R) * 6 * (N - 1));
            const int row = (traj_offset + N < S) ? traj_offset + N - 1 : S - 1;
            memcpy(goal + 6 * (N - 1), eePos_traj + 6 * row, sizeof(R) * 6);
            memmove(lambda, lambda + NS, sizeof(R) * NS * (N - 1));
            shifted = 1;
        }
        if (time_since > dt) {
            shifted = 0;
            time_since = fmod(time_since, dt);
        }
        memcpy(xu, xs, sizeof(R) * NS);
        prev_sim = sim;
    }
    ts->control_updates = step;
    ts->shifts = traj_offset;
    ts->final_error = tracking_error(xs, goal);
    ts->rho_final = rho;
    free(xu); free(xu_old); free(goal); free(lambda);
    return rc;
}

/* gato_form_ss_inner (oldschur.cuh:334-494): the stair ("SS") preconditioner's off-diagonal blocks,
 * from S and the block-Jacobi diagonal theta_k^{-1} already in Pinv's diagonal blocks:
 *   Pinv[k].left  = -(theta_k^{-1} S[k].left)  theta_{k-1}^{-1}          (k > 0)
 *   Pinv[k].right = -(theta_k^{-1} S[k+1].left^T) theta_{k+1}^{-1}       (k < N-1)
 * with the reference's product order.  The reference ships it without calling it. */
void ORC(form_ss)(int N, const R *S, R *Pinv)
{
    R scratch[SS], out[SS], phiT[SS];
    for (int k = 0; k < N; ++k) {
        const R *tk = Pinv + 3 * SS * k + SS;
        if (k > 0) {
            mat_mat(scratch, tk, S + 3 * SS * k, NS, NS, NS, NS, 0);
            mat_mat(out, scratch, Pinv + 3 * SS * (k - 1) + SS, NS, NS, NS, NS, 0);
            for (int i = 0; i < SS; ++i) Pinv[3 * SS * k + i] = -out[i];
        }
        if (k < N - 1) {
            const R *phi = S + 3 * SS * (k + 1);
            for (int i = 0; i < SS; ++i) phiT[(i % NS) * NS + i / NS] = phi[i];  /* load_block_bd transpose */
            mat_mat(scratch, tk, phiT, NS, NS, NS, NS, 0);
            mat_mat(out, scratch, Pinv + 3 * SS * (k + 1) + SS, NS, NS, NS, NS, 0);
            for (int i = 0; i < SS; ++i) Pinv[3 * SS * k + 2 * SS + i] = -out[i];
        }
    }
}
