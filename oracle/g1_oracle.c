/* g1_oracle.c -- FP64 CPU oracle of the batched G1 step (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference's host-compiled physics:
 *   spatial algebra          reference src/spatial.h:1-278
 *   FK + velocities          reference src/g1_core.h:29-54   (g1o_fk_vel)
 *   pure ABA (no contacts)   reference src/g1_core.h:59-105  (g1o_aba_pure)
 *   contacts + PD + ABA      reference src/g1_core.h:109-207 (g1o_aba_fused)
 *   semi-implicit Euler      reference src/g1_core.h:212-222 (g1o_integrate)
 *   host ABI                 reference src/host_lib.cpp:7-53
 *   reset + RNG              reference src/g1_kernel.cu:54-103
 * Model constants come from g1sim_b200/csrc/g1_model_data.h, generated from
 * the MJCF by g1sim_b200/model/gen_model.py.
 *
 * Build: oracle/Makefile (-O2 -ffp-contract=off so float code matches the
 * CUDA path's explicitly rounded float arithmetic bit for bit).
 */
#include "g1_oracle.h"

#include <math.h>
#include <stddef.h>
#include <string.h>

#include "../g1sim_b200/csrc/g1_model_data.h"

#define NB G1M_NB
#define NQ G1M_NQ
#define NV G1M_NV
#define NU G1M_NU
#define NC G1M_NC
#define NJ (NB - 1)
#define ANCHOR_FREE 1e30

/* ------------------------------------------------------------ algebra --- */
typedef struct { double x, y, z; } v3;
typedef struct { double m[9]; } m3; /* row-major */
typedef struct { double w, x, y, z; } quat;
typedef struct { m3 R; v3 p; } se3;
typedef struct { v3 a, l; } sv;     /* [angular; linear], body frame */
typedef struct { double m[21]; } m6s; /* lower-triangular packed 6x6 */

static v3 mk3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 scl3(double s, v3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
static double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 crs3(v3 a, v3 b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static v3 ld3(const double* p) { return mk3(p[0], p[1], p[2]); }

/* reference src/spatial.h:22-39 */
static v3 mv(const m3* A, v3 v) {
  return mk3(A->m[0] * v.x + A->m[1] * v.y + A->m[2] * v.z,
             A->m[3] * v.x + A->m[4] * v.y + A->m[5] * v.z,
             A->m[6] * v.x + A->m[7] * v.y + A->m[8] * v.z);
}
static v3 mtv(const m3* A, v3 v) {
  return mk3(A->m[0] * v.x + A->m[3] * v.y + A->m[6] * v.z,
             A->m[1] * v.x + A->m[4] * v.y + A->m[7] * v.z,
             A->m[2] * v.x + A->m[5] * v.y + A->m[8] * v.z);
}
static m3 mm(const m3* A, const m3* B) {
  m3 C;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      C.m[3 * i + j] = A->m[3 * i + 0] * B->m[0 * 3 + j] + A->m[3 * i + 1] * B->m[1 * 3 + j] +
                       A->m[3 * i + 2] * B->m[2 * 3 + j];
  return C;
}
/* A B^T, reference src/spatial.h:190-196 */
static m3 mmT(const m3* A, const m3* B) {
  m3 C;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      C.m[3 * i + j] = A->m[3 * i + 0] * B->m[3 * j + 0] + A->m[3 * i + 1] * B->m[3 * j + 1] +
                       A->m[3 * i + 2] * B->m[3 * j + 2];
  return C;
}

/* reference src/spatial.h:42-62 */
static quat qnrm(quat q) {
  double n = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  double s = 1.0 / n;
  quat r = {q.w * s, q.x * s, q.y * s, q.z * s};
  return r;
}
static quat qmul(quat a, quat b) {
  quat r = {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
            a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
  return r;
}
static m3 q2m(quat q) {
  double w = q.w, x = q.x, y = q.y, z = q.z;
  m3 R;
  R.m[0] = 1 - 2 * (y * y + z * z); R.m[1] = 2 * (x * y - w * z);     R.m[2] = 2 * (x * z + w * y);
  R.m[3] = 2 * (x * y + w * z);     R.m[4] = 1 - 2 * (x * x + z * z); R.m[5] = 2 * (y * z - w * x);
  R.m[6] = 2 * (x * z - w * y);     R.m[7] = 2 * (y * z + w * x);     R.m[8] = 1 - 2 * (x * x + y * y);
  return R;
}
/* Rodrigues, reference src/spatial.h:63-70 */
static m3 axang(v3 a, double q) {
  double c = cos(q), s = sin(q), t = 1 - c;
  m3 R;
  R.m[0] = c + t * a.x * a.x;       R.m[1] = t * a.x * a.y - s * a.z; R.m[2] = t * a.x * a.z + s * a.y;
  R.m[3] = t * a.x * a.y + s * a.z; R.m[4] = c + t * a.y * a.y;       R.m[5] = t * a.y * a.z - s * a.x;
  R.m[6] = t * a.x * a.z - s * a.y; R.m[7] = t * a.y * a.z + s * a.x; R.m[8] = c + t * a.z * a.z;
  return R;
}
/* q <- q (x) exp(w dt / 2), body-frame w; reference src/spatial.h:73-79 */
static quat qint(quat q, v3 w, double dt) {
  double angle = sqrt(dot3(w, w)) * dt;
  if (angle < 1e-12) return q;
  double s = sin(angle / 2) / (angle / dt);
  quat dq = {cos(angle / 2), s * w.x, s * w.y, s * w.z};
  return qnrm(qmul(q, dq));
}

static sv mksv(v3 a, v3 l) { sv r = {a, l}; return r; }
static sv addsv(sv u, sv w) { return mksv(add3(u.a, w.a), add3(u.l, w.l)); }
static sv subsv(sv u, sv w) { return mksv(sub3(u.a, w.a), sub3(u.l, w.l)); }
static sv sclsv(double s, sv u) { return mksv(scl3(s, u.a), scl3(s, u.l)); }
static double dotsv(sv u, sv w) { return dot3(u.a, w.a) + dot3(u.l, w.l); }

/* reference src/spatial.h:97-118 */
static sv mact_inv(const se3* X, sv m) {
  return mksv(mtv(&X->R, m.a), mtv(&X->R, sub3(m.l, crs3(X->p, m.a))));
}
static sv fact(const se3* X, sv f) {
  v3 l = mv(&X->R, f.l);
  return mksv(add3(mv(&X->R, f.a), crs3(X->p, l)), l);
}
static sv crm(sv v, sv m) {
  return mksv(crs3(v.a, m.a), add3(crs3(v.a, m.l), crs3(v.l, m.a)));
}
static sv crf(sv v, sv f) {
  return mksv(add3(crs3(v.a, f.a), crs3(v.l, f.l)), crs3(v.a, f.l));
}

/* packed symmetric 6x6: reference src/spatial.h:121-172 */
static sv m6mul(const m6s* A, sv u) {
  double x[6] = {u.a.x, u.a.y, u.a.z, u.l.x, u.l.y, u.l.z};
  double y[6] = {0, 0, 0, 0, 0, 0};
  int idx = 0;
  for (int i = 0; i < 6; ++i) {
    for (int j = 0; j < i; ++j) {
      double Aij = A->m[idx++];
      y[i] += Aij * x[j];
      y[j] += Aij * x[i];
    }
    y[i] += A->m[idx++] * x[i];
  }
  return mksv(mk3(y[0], y[1], y[2]), mk3(y[3], y[4], y[5]));
}
static void m6subouter(m6s* A, sv U, double invd) {
  double u[6] = {U.a.x, U.a.y, U.a.z, U.l.x, U.l.y, U.l.z};
  int idx = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) A->m[idx++] -= u[i] * u[j] * invd;
}
static m6s spin(double mass, v3 c, const double* Icom) {
  m6s I;
  double cx[9] = {0, -c.z, c.y, c.z, 0, -c.x, -c.y, c.x, 0};
  int idx = 0;
  for (int i = 0; i < 6; ++i) {
    for (int j = 0; j <= i; ++j) {
      double val;
      if (i < 3 && j < 3) {
        double s = 0;
        for (int k = 0; k < 3; ++k) s += cx[3 * i + k] * cx[3 * k + j];
        val = Icom[3 * i + j] - mass * s;
      } else if (i >= 3 && j < 3) {
        val = -mass * cx[3 * (i - 3) + j];
      } else {
        val = (i == j) ? mass : 0.0;
      }
      I.m[idx++] = val;
    }
  }
  return I;
}

/* child articulated inertia into the parent frame: reference src/spatial.h:174-251 */
static m3 blkJ(const m6s* I) {
  m3 r = {{I->m[0], I->m[1], I->m[3], I->m[1], I->m[2], I->m[4], I->m[3], I->m[4], I->m[5]}};
  return r;
}
static m3 blkH(const m6s* I) {
  m3 r = {{I->m[6], I->m[10], I->m[15], I->m[7], I->m[11], I->m[16], I->m[8], I->m[12], I->m[17]}};
  return r;
}
static m3 blkM(const m6s* I) {
  m3 r = {{I->m[9], I->m[13], I->m[18], I->m[13], I->m[14], I->m[19], I->m[18], I->m[19], I->m[20]}};
  return r;
}
static m3 skew_mul(v3 p, const m3* A) { /* (p x) A */
  m3 C;
  for (int j = 0; j < 3; ++j) {
    C.m[0 * 3 + j] = -p.z * A->m[1 * 3 + j] + p.y * A->m[2 * 3 + j];
    C.m[1 * 3 + j] = p.z * A->m[0 * 3 + j] - p.x * A->m[2 * 3 + j];
    C.m[2 * 3 + j] = -p.y * A->m[0 * 3 + j] + p.x * A->m[1 * 3 + j];
  }
  return C;
}
static m3 mul_skew(const m3* A, v3 p) { /* A (p x) */
  m3 C;
  for (int i = 0; i < 3; ++i) {
    C.m[i * 3 + 0] = A->m[i * 3 + 1] * p.z - A->m[i * 3 + 2] * p.y;
    C.m[i * 3 + 1] = -A->m[i * 3 + 0] * p.z + A->m[i * 3 + 2] * p.x;
    C.m[i * 3 + 2] = A->m[i * 3 + 0] * p.y - A->m[i * 3 + 1] * p.x;
  }
  return C;
}
static void psum_transform(m6s* P, const m6s* Ii, const se3* X) {
  m3 Ji = blkJ(Ii), Hi = blkH(Ii), Mi = blkM(Ii);
  m3 t, tJ, tH, tM;
  t = mm(&X->R, &Ji); tJ = mmT(&t, &X->R);
  t = mm(&X->R, &Hi); tH = mmT(&t, &X->R);
  t = mm(&X->R, &Mi); tM = mmT(&t, &X->R);
  m3 pxM = skew_mul(X->p, &tM);
  m3 HA;
  for (int i = 0; i < 9; ++i) HA.m[i] = tH.m[i] + pxM.m[i];
  m3 tHT;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) tHT.m[3 * i + j] = tH.m[3 * j + i];
  m3 pxHT = skew_mul(X->p, &tHT);
  m3 HApx = mul_skew(&HA, X->p);
  m3 JA;
  for (int i = 0; i < 9; ++i) JA.m[i] = tJ.m[i] + pxHT.m[i] - HApx.m[i];
  P->m[0] += JA.m[0];
  P->m[1] += JA.m[3]; P->m[2] += JA.m[4];
  P->m[3] += JA.m[6]; P->m[4] += JA.m[7]; P->m[5] += JA.m[8];
  P->m[6] += HA.m[0]; P->m[7] += HA.m[3]; P->m[8] += HA.m[6];
  P->m[10] += HA.m[1]; P->m[11] += HA.m[4]; P->m[12] += HA.m[7];
  P->m[15] += HA.m[2]; P->m[16] += HA.m[5]; P->m[17] += HA.m[8];
  P->m[9] += tM.m[0];
  P->m[13] += tM.m[3]; P->m[14] += tM.m[4];
  P->m[18] += tM.m[6]; P->m[19] += tM.m[7]; P->m[20] += tM.m[8];
}

/* SPD 6x6 solve by Cholesky on a packed copy: reference src/spatial.h:254-278 */
static sv m6solve(const m6s* A, sv b) {
  double L[21];
  memcpy(L, A->m, sizeof(L));
  for (int j = 0; j < 6; ++j) {
    int jj = j * (j + 1) / 2 + j;
    for (int k = 0; k < j; ++k) L[jj] -= L[j * (j + 1) / 2 + k] * L[j * (j + 1) / 2 + k];
    L[jj] = sqrt(L[jj]);
    double inv = 1.0 / L[jj];
    for (int i = j + 1; i < 6; ++i) {
      int ij = i * (i + 1) / 2 + j;
      for (int k = 0; k < j; ++k) L[ij] -= L[i * (i + 1) / 2 + k] * L[j * (j + 1) / 2 + k];
      L[ij] *= inv;
    }
  }
  double y[6] = {b.a.x, b.a.y, b.a.z, b.l.x, b.l.y, b.l.z};
  for (int i = 0; i < 6; ++i) {
    for (int k = 0; k < i; ++k) y[i] -= L[i * (i + 1) / 2 + k] * y[k];
    y[i] /= L[i * (i + 1) / 2 + i];
  }
  for (int i = 5; i >= 0; --i) {
    for (int k = i + 1; k < 6; ++k) y[i] -= L[k * (k + 1) / 2 + i] * y[k];
    y[i] /= L[i * (i + 1) / 2 + i];
  }
  return mksv(mk3(y[0], y[1], y[2]), mk3(y[3], y[4], y[5]));
}

/* ----------------------------------------------------------- physics --- */
/* per-env scratch, reference src/g1_core.h:13-23 */
typedef struct {
  se3 liMi[NB];
  m3 oR[NB];
  v3 oP[NB];
  sv v[NB];
  m6s IA[NB];
  sv pA[NB];
  sv U[NJ];
  double D[NJ], u[NJ];
  sv a[NB];
} ws_t;

static const g1o_envparams kDefaultEp = {1.0, 0.0, 1.0, 1.0};

void g1o_default_config(g1o_config* c) { /* reference src/g1_types.h:44-55 */
  c->gravity_z = -9.81;
  c->contact_kn = 2e4;
  c->contact_dn = 280;
  c->contact_kt = 1e4;
  c->contact_dt = 280;
  c->limit_kp = 200;
  c->limit_kd = 5;
  c->dt = 1e-3;
}
void g1o_default_envparams(g1o_envparams* ep) { *ep = kDefaultEp; }

static sv hinge_S(int h) {
  v3 ax = ld3(g1m_jnt_axis + 3 * h), an = ld3(g1m_jnt_anchor + 3 * h);
  return mksv(ax, crs3(an, ax));
}

/* reference src/g1_core.h:29-54 */
static void fk_vel(const double* qpos, const double* qvel, ws_t* w) {
  quat bq = {qpos[3], qpos[4], qpos[5], qpos[6]};
  w->liMi[0].R = q2m(qnrm(bq));
  w->liMi[0].p = ld3(qpos);
  w->oR[0] = w->liMi[0].R;
  w->oP[0] = w->liMi[0].p;
  w->v[0] = mksv(ld3(qvel + 3), mtv(&w->oR[0], ld3(qvel)));
  for (int i = 1; i < NB; ++i) {
    int h = i - 1, par = g1m_parent[i];
    v3 ax = ld3(g1m_jnt_axis + 3 * h), an = ld3(g1m_jnt_anchor + 3 * h);
    double q = qpos[7 + h], qd = qvel[6 + h];
    quat tq = {g1m_tree_quat[4 * i], g1m_tree_quat[4 * i + 1], g1m_tree_quat[4 * i + 2],
               g1m_tree_quat[4 * i + 3]};
    m3 RT = q2m(qnrm(tq));
    m3 RJ = axang(ax, q);
    w->liMi[i].R = mm(&RT, &RJ);
    w->liMi[i].p = add3(mv(&RT, sub3(an, mv(&RJ, an))), ld3(g1m_tree_pos + 3 * i));
    w->oR[i] = mm(&w->oR[par], &w->liMi[i].R);
    w->oP[i] = add3(mv(&w->oR[par], w->liMi[i].p), w->oP[par]);
    w->v[i] = addsv(mact_inv(&w->liMi[i], w->v[par]), sclsv(qd, hinge_S(h)));
  }
}

static m6s body_inertia(int i, const g1o_envparams* ep) {
  double m = g1m_mass[i] + (i == 0 ? ep->dmass : 0.0);
  return spin(m, ld3(g1m_com + 3 * i), g1m_inertia_com + 9 * i);
}

/* ABA backward/base/forward shared tail; reference src/g1_core.h:72-105 and :156-206 */
static void aba_forward(const double* qvel, ws_t* w, double* qacc) {
  w->a[0] = m6solve(&w->IA[0], subsv(mksv(mk3(0, 0, 0), mk3(0, 0, 0)), w->pA[0]));
  for (int i = 1; i < NB; ++i) {
    int h = i - 1, par = g1m_parent[i];
    sv Sh = hinge_S(h);
    sv c = crm(w->v[i], sclsv(qvel[6 + h], Sh));
    sv ap = addsv(mact_inv(&w->liMi[i], w->a[par]), c);
    double qdd = (w->u[h] - dotsv(w->U[h], ap)) / w->D[h];
    w->a[i] = addsv(ap, sclsv(qdd, Sh));
    qacc[6 + h] = qdd;
  }
  v3 aw = w->a[0].a;
  v3 al = mv(&w->oR[0], add3(w->a[0].l, crs3(w->v[0].a, w->v[0].l)));
  qacc[0] = al.x; qacc[1] = al.y; qacc[2] = al.z;
  qacc[3] = aw.x; qacc[4] = aw.y; qacc[5] = aw.z;
}

/* reference src/g1_core.h:59-105 */
static void aba_pure(const g1o_config* cfg, const double* qvel, const double* tau, ws_t* w,
                     double* qacc) {
  for (int i = 0; i < NB; ++i) {
    v3 c = ld3(g1m_com + 3 * i);
    w->IA[i] = body_inertia(i, &kDefaultEp);
    v3 gb = mtv(&w->oR[i], mk3(0, 0, cfg->gravity_z));
    v3 fg = scl3(g1m_mass[i], gb);
    w->pA[i] = subsv(crf(w->v[i], m6mul(&w->IA[i], w->v[i])), mksv(crs3(c, fg), fg));
  }
  {
    v3 fb = mtv(&w->oR[0], ld3(tau));
    w->pA[0] = subsv(w->pA[0], mksv(ld3(tau + 3), fb));
  }
  for (int i = NB - 1; i >= 1; --i) {
    int h = i - 1, par = g1m_parent[i];
    double qd = qvel[6 + h];
    sv Sh = hinge_S(h);
    w->U[h] = m6mul(&w->IA[i], Sh);
    w->D[h] = dotsv(Sh, w->U[h]) + g1m_armature[h];
    w->u[h] = tau[6 + h] - g1m_damping[h] * qd - dotsv(Sh, w->pA[i]);
    double invd = 1.0 / w->D[h];
    sv c = crm(w->v[i], sclsv(qd, Sh));
    m6s Ia = w->IA[i];
    m6subouter(&Ia, w->U[h], invd);
    sv pa = addsv(addsv(w->pA[i], m6mul(&Ia, c)), sclsv(w->u[h] * invd, w->U[h]));
    psum_transform(&w->IA[par], &Ia, &w->liMi[i]);
    w->pA[par] = addsv(w->pA[par], fact(&w->liMi[i], pa));
  }
  aba_forward(qvel, w, qacc);
}

/* reference src/g1_core.h:109-207, with per-env friction / base mass / gain scales */
static void aba_fused(const g1o_config* cfg, const g1o_envparams* ep, const double* qpos,
                      const double* qvel, const double* ctrl, double* anchor, ws_t* w,
                      double* qacc, double* fn_out) {
  for (int i = 0; i < NB; ++i) {
    v3 c = ld3(g1m_com + 3 * i);
    double m = g1m_mass[i] + (i == 0 ? ep->dmass : 0.0);
    w->IA[i] = body_inertia(i, ep);
    v3 gb = mtv(&w->oR[i], mk3(0, 0, cfg->gravity_z));
    v3 fg = scl3(m, gb);
    sv f = mksv(crs3(c, fg), fg);
    w->pA[i] = subsv(crf(w->v[i], m6mul(&w->IA[i], w->v[i])), f);
  }
  /* contacts: reference src/g1_core.h:123-153 */
  for (int k = 0; k < NC; ++k) {
    int b = g1m_contact_body[k];
    v3 r = ld3(g1m_contact_pos + 3 * k);
    v3 p = add3(mv(&w->oR[b], r), w->oP[b]);
    double depth = g1m_contact_radius - p.z;
    double fn = 0;
    if (depth > 0) {
      v3 vp = mv(&w->oR[b], add3(w->v[b].l, crs3(w->v[b].a, r)));
      fn = cfg->contact_kn * depth - cfg->contact_dn * vp.z;
      if (fn < 0) fn = 0;
      if (fn > 500.0) fn = 500.0;
      if (anchor[2 * k] >= ANCHOR_FREE) {
        anchor[2 * k] = p.x;
        anchor[2 * k + 1] = p.y;
      }
      double ftx = -cfg->contact_kt * (p.x - anchor[2 * k]) - cfg->contact_dt * vp.x;
      double fty = -cfg->contact_kt * (p.y - anchor[2 * k + 1]) - cfg->contact_dt * vp.y;
      double ftn = sqrt(ftx * ftx + fty * fty), fmax = ep->mu * fn;
      if (ftn > fmax) {
        double sc = fmax / (ftn + 1e-12);
        ftx *= sc;
        fty *= sc;
        anchor[2 * k] = p.x + ftx / cfg->contact_kt;
        anchor[2 * k + 1] = p.y + fty / cfg->contact_kt;
      }
      v3 fw = mk3(ftx, fty, fn);
      v3 fb = mtv(&w->oR[b], fw);
      w->pA[b] = subsv(w->pA[b], mksv(crs3(r, fb), fb));
    } else {
      anchor[2 * k] = ANCHOR_FREE;
      anchor[2 * k + 1] = ANCHOR_FREE;
    }
    if (fn_out) fn_out[k] = fn;
  }
  /* backward with PD servos, soft limits and implicit damping: reference src/g1_core.h:156-186 */
  for (int i = NB - 1; i >= 1; --i) {
    int h = i - 1, par = g1m_parent[i];
    double qd = qvel[6 + h];
    sv Sh = hinge_S(h);
    w->U[h] = m6mul(&w->IA[i], Sh);
    double q = qpos[7 + h];
    double kp = g1m_act_kp[h] * ep->kp_scale, kv = g1m_act_kv[h] * ep->kd_scale;
    double t = kp * (ctrl[h] - q) - kv * qd;
    double lim = g1m_act_frclim[h];
    if (t > lim) t = lim;
    if (t < -lim) t = -lim;
    double lo = g1m_jnt_range[2 * h], hi = g1m_jnt_range[2 * h + 1];
    double bd = kv + g1m_damping[h];
    if (q < lo) { t += cfg->limit_kp * (lo - q) - cfg->limit_kd * qd; bd += cfg->limit_kd; }
    if (q > hi) { t += cfg->limit_kp * (hi - q) - cfg->limit_kd * qd; bd += cfg->limit_kd; }
    w->D[h] = dotsv(Sh, w->U[h]) + g1m_armature[h] + cfg->dt * bd;
    w->u[h] = t - g1m_damping[h] * qd - dotsv(Sh, w->pA[i]);
    double invd = 1.0 / w->D[h];
    sv c = crm(w->v[i], sclsv(qd, Sh));
    m6s Ia = w->IA[i];
    m6subouter(&Ia, w->U[h], invd);
    sv pa = addsv(addsv(w->pA[i], m6mul(&Ia, c)), sclsv(w->u[h] * invd, w->U[h]));
    psum_transform(&w->IA[par], &Ia, &w->liMi[i]);
    w->pA[par] = addsv(w->pA[par], fact(&w->liMi[i], pa));
  }
  aba_forward(qvel, w, qacc);
}

/* reference src/g1_core.h:212-222 */
static void integrate(double dt, const double* qacc, double* qpos, double* qvel) {
  for (int i = 0; i < NV; ++i) qvel[i] += dt * qacc[i];
  qpos[0] += dt * qvel[0];
  qpos[1] += dt * qvel[1];
  qpos[2] += dt * qvel[2];
  quat q = {qpos[3], qpos[4], qpos[5], qpos[6]};
  q = qint(q, ld3(qvel + 3), dt);
  qpos[3] = q.w; qpos[4] = q.x; qpos[5] = q.y; qpos[6] = q.z;
  for (int h = 0; h < NJ; ++h) qpos[7 + h] += dt * qvel[6 + h];
}

/* reference src/g1_core.h:225-232 */
static void one_step(const g1o_config* cfg, const g1o_envparams* ep, double* qpos, double* qvel,
                     const double* ctrl, double* anchor, ws_t* w, double* fn_out) {
  double qacc[NV];
  fk_vel(qpos, qvel, w);
  aba_fused(cfg, ep, qpos, qvel, ctrl, anchor, w, qacc, fn_out);
  integrate(cfg->dt, qacc, qpos, qvel);
}

/* foot outputs from the last FK, reference src/g1_kernel.cu:128-145 */
static void foot_out(const ws_t* w, double* foot_pos, double* foot_vel) {
  if (foot_pos) {
    foot_pos[0] = w->oP[6].x; foot_pos[1] = w->oP[6].y; foot_pos[2] = w->oP[6].z;
    foot_pos[3] = w->oP[12].x; foot_pos[4] = w->oP[12].y; foot_pos[5] = w->oP[12].z;
  }
  if (foot_vel) {
    v3 vl = mv(&w->oR[6], w->v[6].l), vr = mv(&w->oR[12], w->v[12].l);
    foot_vel[0] = vl.x; foot_vel[1] = vl.y; foot_vel[2] = vl.z;
    foot_vel[3] = vr.x; foot_vel[4] = vr.y; foot_vel[5] = vr.z;
  }
}

/* ---------------------------------------------------------- host ABI --- */
int g1_sizes(int* nb, int* nq, int* nv, int* nu, int* nc) {
  *nb = NB; *nq = NQ; *nv = NV; *nu = NU; *nc = NC;
  return 8;
}

void g1_c_fk(const double* qpos, double* xpos, double* xmat) {
  ws_t w;
  double qv[NV];
  memset(qv, 0, sizeof(qv));
  fk_vel(qpos, qv, &w);
  for (int b = 0; b < NB; ++b) {
    xpos[3 * b + 0] = w.oP[b].x; xpos[3 * b + 1] = w.oP[b].y; xpos[3 * b + 2] = w.oP[b].z;
    for (int k = 0; k < 9; ++k) xmat[9 * b + k] = w.oR[b].m[k];
  }
}

void g1_c_fd(const double* qpos, const double* qvel, const double* tau, double* qacc) {
  ws_t w;
  g1o_config cfg;
  g1o_default_config(&cfg);
  fk_vel(qpos, qvel, &w);
  aba_pure(&cfg, qvel, tau, &w, qacc);
}

void g1o_step(const g1o_config* cfg, const g1o_envparams* ep, double* qpos, double* qvel,
              const double* ctrl, double* anchor, int nsub, double* fn_out, double* foot_pos,
              double* foot_vel) {
  ws_t w;
  double fn[NC];
  memset(fn, 0, sizeof(fn));
  if (!ep) ep = &kDefaultEp;
  for (int s = 0; s < nsub; ++s) one_step(cfg, ep, qpos, qvel, ctrl, anchor, &w, fn);
  if (nsub > 0) foot_out(&w, foot_pos, foot_vel);
  if (fn_out) memcpy(fn_out, fn, sizeof(fn));
}

void g1_c_step(double* qpos, double* qvel, const double* ctrl, int nsub, double dt,
               double* fn_out, double* anchor) {
  g1o_config cfg;
  g1o_default_config(&cfg);
  cfg.dt = dt;
  g1o_step(&cfg, &kDefaultEp, qpos, qvel, ctrl, anchor, nsub, fn_out, NULL, NULL);
}

/* ----------------------------------------------------------- batches --- */
void g1o_step_soa(int nenv, int nsub, const g1o_config* cfg, double* qpos, double* qvel,
                  double* anchor, const double* ctrl, const double* mu, const double* dmass,
                  const double* kp_scale, const double* kd_scale, double* foot_pos,
                  double* foot_vel, double* contact_forces) {
  for (int e = 0; e < nenv; ++e) {
    double qp[NQ], qv[NV], ct[NU], an[2 * NC], fn[NC], fp[6], fv[6];
    size_t n = (size_t)nenv;
    for (int i = 0; i < NQ; ++i) qp[i] = qpos[i * n + e];
    for (int i = 0; i < NV; ++i) qv[i] = qvel[i * n + e];
    for (int i = 0; i < NU; ++i) ct[i] = ctrl[i * n + e];
    for (int i = 0; i < 2 * NC; ++i) an[i] = anchor[i * n + e];
    g1o_envparams ep = kDefaultEp;
    if (mu) ep.mu = mu[e];
    if (dmass) ep.dmass = dmass[e];
    if (kp_scale) ep.kp_scale = kp_scale[e];
    if (kd_scale) ep.kd_scale = kd_scale[e];
    g1o_step(cfg, &ep, qp, qv, ct, an, nsub, fn, fp, fv);
    for (int i = 0; i < NQ; ++i) qpos[i * n + e] = qp[i];
    for (int i = 0; i < NV; ++i) qvel[i * n + e] = qv[i];
    for (int i = 0; i < 2 * NC; ++i) anchor[i * n + e] = an[i];
    if (foot_pos) for (int i = 0; i < 6; ++i) foot_pos[i * n + e] = fp[i];
    if (foot_vel) for (int i = 0; i < 6; ++i) foot_vel[i * n + e] = fv[i];
    if (contact_forces) for (int i = 0; i < NC; ++i) contact_forces[i * n + e] = fn[i];
  }
}

/* ------------------------------------------------------ branch margins --- */
/* Distance of one substep from every branch of the discontinuous model,
 * normalised by the size of FP32 rounding at that branch: contact touchdown
 * (depth 0, 1e-6 m), normal-force clamps (0 and 500 N, 1e-2 N), stick/slip
 * (|ft| = mu fn, 1e-2 N + 1e-6 relative), soft joint limits (1e-6 rad) and
 * the servo torque clamp (1e-3 N m).  A value below 1 means an FP32 step may
 * legitimately take the other branch (reference src/g1_core.h:129-150,
 * :168-174). */
static double branch_margin(const g1o_config* cfg, const g1o_envparams* ep, const double* qpos,
                            const double* qvel, const double* ctrl, const double* anchor_in) {
  ws_t w;
  double anchor[2 * NC];
  memcpy(anchor, anchor_in, sizeof(anchor));
  fk_vel(qpos, qvel, &w);
  double m = 1e300;
#define MARGIN(x) do { double _x = (x); if (_x < m) m = _x; } while (0)
  for (int k = 0; k < NC; ++k) {
    int b = g1m_contact_body[k];
    v3 r = ld3(g1m_contact_pos + 3 * k);
    v3 p = add3(mv(&w.oR[b], r), w.oP[b]);
    double depth = g1m_contact_radius - p.z;
    MARGIN(fabs(depth) / 1e-6);
    if (depth <= 0) continue;
    v3 vp = mv(&w.oR[b], add3(w.v[b].l, crs3(w.v[b].a, r)));
    double fn = cfg->contact_kn * depth - cfg->contact_dn * vp.z;
    MARGIN(fabs(fn) / 1e-2);
    MARGIN(fabs(fn - 500.0) / 1e-2);
    if (fn < 0) fn = 0;
    if (fn > 500.0) fn = 500.0;
    double ax = anchor[2 * k] >= ANCHOR_FREE ? p.x : anchor[2 * k];
    double ay = anchor[2 * k + 1] >= ANCHOR_FREE ? p.y : anchor[2 * k + 1];
    double ftx = -cfg->contact_kt * (p.x - ax) - cfg->contact_dt * vp.x;
    double fty = -cfg->contact_kt * (p.y - ay) - cfg->contact_dt * vp.y;
    double ftn = sqrt(ftx * ftx + fty * fty), fmax = ep->mu * fn;
    MARGIN(fabs(ftn - fmax) / (1e-2 + 1e-6 * (ftn > fmax ? ftn : fmax)));
  }
  for (int h = 0; h < NJ; ++h) {
    double q = qpos[7 + h], qd = qvel[6 + h];
    MARGIN(fabs(q - g1m_jnt_range[2 * h]) / 1e-6);
    MARGIN(fabs(q - g1m_jnt_range[2 * h + 1]) / 1e-6);
    double kp = g1m_act_kp[h] * ep->kp_scale, kv = g1m_act_kv[h] * ep->kd_scale;
    double t = kp * (ctrl[h] - q) - kv * qd;
    MARGIN(fabs(fabs(t) - g1m_act_frclim[h]) / 1e-3);
  }
#undef MARGIN
  return m;
}

void g1o_branch_margin_soa(int nenv, const g1o_config* cfg, const double* qpos,
                           const double* qvel, const double* anchor, const double* ctrl,
                           const double* mu, const double* dmass, double* margin) {
  size_t n = (size_t)nenv;
  for (int e = 0; e < nenv; ++e) {
    double qp[NQ], qv[NV], ct[NU], an[2 * NC];
    for (int i = 0; i < NQ; ++i) qp[i] = qpos[i * n + e];
    for (int i = 0; i < NV; ++i) qv[i] = qvel[i * n + e];
    for (int i = 0; i < NU; ++i) ct[i] = ctrl[i * n + e];
    for (int i = 0; i < 2 * NC; ++i) an[i] = anchor[i * n + e];
    g1o_envparams ep = kDefaultEp;
    if (mu) ep.mu = mu[e];
    if (dmass) ep.dmass = dmass[e];
    margin[e] = branch_margin(cfg, &ep, qp, qv, ct, an);
  }
}

/* --------------------------------------------------------- RNG, reset --- */
/* 32-bit xorshift-multiply integer hash (C. Wellons' "lowbias32"), the
 * reference's g1_hash (src/g1_kernel.cu:54-58). */
unsigned g1o_hash(unsigned x) {
  x ^= x >> 16; x *= 0x7feb352du;
  x ^= x >> 15; x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

/* reference g1_urand (src/g1_kernel.cu:59-62), in float */
static float ref_urand(unsigned* s) {
  *s = g1o_hash(*s + 0x9E3779B9u);
  return (float)(*s) * 2.3283064365386963e-10f;
}

/* reference src/g1_kernel.cu:85-103: float arithmetic, one rounding per op */
void g1o_reset_done_soa(int nenv, double* qpos, double* qvel, double* anchor,
                        const uint8_t* done, unsigned seed, float noise, float drop) {
  size_t n = (size_t)nenv;
  for (int e = 0; e < nenv; ++e) {
    if (!done[e]) continue;
    unsigned s = g1o_hash(seed ^ (unsigned)(e + 1));
    for (int i = 0; i < NQ; ++i) {
      float v = (float)g1m_qpos_stand[i];
      if (i == 2) v = v + drop;
      if (i >= 7) {
        /* v += noise*(2u-1) as one fused multiply-add: the reference's
         * compilers contract it (nvcc -fmad=true default); 2u-1 is exact */
        float u = ref_urand(&s);
        float r = 2.0f * u - 1.0f;
        v = fmaf(noise, r, v);
      }
      qpos[i * n + e] = v;
    }
    for (int i = 0; i < NV; ++i) qvel[i * n + e] = 0;
    for (int i = 0; i < 2 * NC; ++i) anchor[i * n + e] = (double)1e30f;
  }
}

/* Counter-based uniform in [0,1) with 24 random bits (exact in float). */
float g1o_uniform(unsigned seed, unsigned stream, unsigned counter) {
  unsigned h = g1o_hash(seed ^ g1o_hash(stream * 0x9E3779B9u + 0x7F4A7C15u));
  h = g1o_hash(h ^ (counter * 0x85EBCA6Bu + 0xC2B2AE35u));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

static float draw_target(unsigned seed, int e, int step, int j, float frac) {
  float u = g1o_uniform(seed, (unsigned)e, (unsigned)step * 64u + (unsigned)j);
  float r = 2.0f * u - 1.0f; /* exact */
  float lo = (float)g1m_jnt_range[2 * j], hi = (float)g1m_jnt_range[2 * j + 1];
  float span = frac * (hi - lo);
  float d = r * span;
  return (float)g1m_qpos_stand[7 + j] + d;
}

void g1o_draw_targets(int nenv, unsigned seed, int step, float target_frac, float* ctrl_f) {
  for (int j = 0; j < NU; ++j)
    for (int e = 0; e < nenv; ++e)
      ctrl_f[(size_t)j * nenv + e] = draw_target(seed, e, step, j, target_frac);
}

void g1o_rollout_soa(int nenv, int npolicy, int decim, const g1o_config* cfg,
                     const g1o_rollout_params* rp, double* qpos, double* qvel, double* anchor,
                     double* ctrl, const double* mu, const double* dmass, int* reset_count) {
  size_t n = (size_t)nenv;
  for (int e = 0; e < nenv; ++e) {
    double qp[NQ], qv[NV], ct[NU], an[2 * NC];
    for (int i = 0; i < NQ; ++i) qp[i] = qpos[i * n + e];
    for (int i = 0; i < NV; ++i) qv[i] = qvel[i * n + e];
    for (int i = 0; i < NU; ++i) ct[i] = ctrl[i * n + e];
    for (int i = 0; i < 2 * NC; ++i) an[i] = anchor[i * n + e];
    g1o_envparams ep = kDefaultEp;
    if (mu) ep.mu = mu[e];
    if (dmass) ep.dmass = dmass[e];
    for (int k = 0; k < npolicy; ++k) {
      int step = rp->step0 + k;
      if (rp->redraw)
        for (int j = 0; j < NU; ++j) ct[j] = draw_target(rp->seed, e, step, j, rp->target_frac);
      g1o_step(cfg, &ep, qp, qv, ct, an, decim, NULL, NULL, NULL);
      if ((float)qp[2] < rp->reset_z) {
        float u = g1o_uniform(rp->seed ^ 0x5bd1e995u, (unsigned)e, (unsigned)step);
        float z0 = rp->z0_lo + u * (rp->z0_hi - rp->z0_lo);
        for (int i = 0; i < NQ; ++i) qp[i] = (float)g1m_qpos_stand[i];
        qp[2] = z0;
        for (int i = 0; i < NV; ++i) qv[i] = 0;
        for (int i = 0; i < 2 * NC; ++i) an[i] = (double)1e30f;
        if (reset_count) reset_count[e] += 1;
      }
    }
    for (int i = 0; i < NQ; ++i) qpos[i * n + e] = qp[i];
    for (int i = 0; i < NV; ++i) qvel[i * n + e] = qv[i];
    for (int i = 0; i < NU; ++i) ctrl[i * n + e] = ct[i];
    for (int i = 0; i < 2 * NC; ++i) anchor[i * n + e] = an[i];
  }
}
