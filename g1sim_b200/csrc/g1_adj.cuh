// g1_adj.cuh -- reverse-mode adjoint of one G1 substep, written for the
// G1's structure (the chain phases of g1_phys.cuh) and any real type R
// (float for the product, double for the validation build).
//
// The step x' = f(x, u, kp_scale, kd_scale) (x = qpos 36, qvel 35, anchor 16)
// is the g1_phys.cuh step -- FK, contacts, PD servo with implicit damping
// and ABA, semi-implicit Euler (reference src/g1_core.h:29-232) -- in plain
// R arithmetic.  Its vector-Jacobian product is derived by hand:
//
//   ABA solves  Mt(q) nu_dot = tau(q, qd, u) - b(x) + J(q)^T f(x)
//   with Mt = M + diag(armature + dt * implicit damping), nu = (w_body,
//   v_body, qd), nu_dot = (a0, qdd).  For an adjoint nu_dot_bar of nu_dot,
//     mu = Mt^-1 nu_dot_bar            (one more ABA sweep with the primal's
//                                       factors U / D, 1 / D and the base LDL)
//     theta_bar += d/dtheta [ mu . (tau + J^T f - Mt nu_dot - b) ]
//   at fixed mu and nu_dot.  The bracket is -Psi(-mu) plus the servo terms,
//     Psi(psi) = sum_i psi_i . (I_i at_i + v_i x* I_i v_i - W_ext,i),
//   the inverse-dynamics residual of the body accelerations at_i = a_i -
//   (0, g_i) weighted by the bodies' velocities psi_i under the generalised
//   velocity -mu (psi_i = X_i psi_p + S_i mu'_i, which is the ABA forward
//   recursion of the mu solve itself).  Psi is reversed body by body from
//   the leaves to the root: 6-vector adjoints of psi_i, at_i and v_i move to
//   the parent through X_i^T (a force transform), and each hinge angle picks
//   up -ybar . (S_i x y_i) for y in (psi, X_i at_p, v_i); the contact
//   wrench W_ext depends on the foot's world pose and twist and on the
//   anchors, and is reversed sphere by sphere; the legs' world pose is
//   reversed up the chain to the base pose.  No 6x6 articulated inertia is
//   ever differentiated.
//
// Switches (contact touchdown, normal-force clamp, fresh anchor, stick /
// slip, torque clamp, soft limits) take the primal's branch: the
// derivative is one-sided at a switch.
//
// A per-env tape (slot-major storage of R, shared memory on the device) holds
// the primal's per-body and per-hinge values that the reverse pass reads.
#pragma once
#include <math.h>

#include "g1_model_derived.h"

#if defined(__CUDACC__)
#define GA_HD __host__ __device__ __forceinline__
#define GA_CE __host__ __device__ constexpr
#else
#define GA_HD inline
#endif

namespace g1b::adj {

constexpr int kNB = G1M_NB, kNJ = G1M_NB - 1, kNQ = G1M_NQ, kNV = G1M_NV, kNU = G1M_NU, kNC = G1M_NC;
constexpr int kState = kNQ + kNV + 2 * kNC;  // 87
constexpr int kQV = kNQ;                       // qvel offset in x
constexpr int kAN = kNQ + kNV;                 // anchor offset in x

// ------------------------------------------------------------ model
template <class R>
struct BodyA {
  R T[9];       // tree rotation parent <- body (row-major)
  R p[3];       // body origin in the parent frame
  R J[6], H[9]; // rigid spatial inertia at the origin (J xx yy zz xy xz yz, H = m [c]x)
  R m;
  R kp, kv, lim, lo, hi, arm, damp;
  int axis, ident;
};
template <class R>
struct ModelA {
  BodyA<R> b[kNB];
  R stand[kNQ];
  R cpos[3 * kNC];
  R com0[3], icom0[6];
  R radius, mu0;
};
template <class R>
constexpr ModelA<R> make_model() {
  ModelA<R> M{};
  for (int i = 0; i < kNB; ++i) {
    BodyA<R>& b = M.b[i];
    for (int k = 0; k < 9; ++k) b.T[k] = (R)g1m_tree_rot[9 * i + k];
    for (int k = 0; k < 3; ++k) b.p[k] = (R)g1m_tree_pos[3 * i + k];
    for (int k = 0; k < 6; ++k) b.J[k] = (R)g1m_sp_inertia[16 * i + k];
    for (int k = 0; k < 9; ++k) b.H[k] = (R)g1m_sp_inertia[16 * i + 6 + k];
    b.m = (R)g1m_sp_inertia[16 * i + 15];
    b.ident = g1m_tree_ident[i];
    if (i > 0) {
      const int h = i - 1;
      b.kp = (R)g1m_act_kp[h];
      b.kv = (R)g1m_act_kv[h];
      b.lim = (R)g1m_act_frclim[h];
      b.lo = (R)g1m_jnt_range[2 * h];
      b.hi = (R)g1m_jnt_range[2 * h + 1];
      b.arm = (R)g1m_armature[h];
      b.damp = (R)g1m_damping[h];
      b.axis = g1m_axis_idx[h];
    }
  }
  for (int k = 0; k < kNQ; ++k) M.stand[k] = (R)g1m_qpos_stand[k];
  for (int k = 0; k < 3 * kNC; ++k) M.cpos[k] = (R)g1m_contact_pos[k];
  for (int k = 0; k < 3; ++k) M.com0[k] = (R)g1m_com[k];
  M.icom0[0] = (R)g1m_inertia_com[0];
  M.icom0[1] = (R)g1m_inertia_com[4];
  M.icom0[2] = (R)g1m_inertia_com[8];
  M.icom0[3] = (R)g1m_inertia_com[1];
  M.icom0[4] = (R)g1m_inertia_com[2];
  M.icom0[5] = (R)g1m_inertia_com[5];
  M.radius = (R)g1m_contact_radius;
  M.mu0 = (R)g1m_contact_mu;
  return M;
}
#if defined(__CUDACC__)
static __constant__ ModelA<float> c_adj_f = make_model<float>();
static __constant__ ModelA<double> c_adj_d = make_model<double>();
#endif
static constexpr ModelA<float> k_adj_f = make_model<float>();
static constexpr ModelA<double> k_adj_d = make_model<double>();
template <class R>
GA_HD const ModelA<R>& model();
template <>
GA_HD const ModelA<float>& model<float>() {
#if defined(__CUDA_ARCH__)
  return c_adj_f;
#else
  return k_adj_f;
#endif
}
template <>
GA_HD const ModelA<double>& model<double>() {
#if defined(__CUDA_ARCH__)
  return c_adj_d;
#else
  return k_adj_d;
#endif
}
template <class R>
GA_HD const BodyA<R>& body(int i) { return model<R>().b[i]; }

template <class R>
struct Cfg {
  R gz, kn, dn, kt, dtc, lkp, lkd, dt;
};
// Per-env parameters: friction, base-mass offset, servo gain scales.
template <class R>
struct Par {
  R mu, dmass, kps, kds;
};

// ------------------------------------------------------------ algebra
template <class R>
struct V3 {
  R x, y, z;
};
template <class R>
GA_HD R& at(V3<R>& v, int i) { return i == 0 ? v.x : i == 1 ? v.y : v.z; }
template <class R>
GA_HD R cat(const V3<R>& v, int i) { return i == 0 ? v.x : i == 1 ? v.y : v.z; }
template <class R>
GA_HD V3<R> v3(R x, R y, R z) { return V3<R>{x, y, z}; }
template <class R>
GA_HD V3<R> operator+(const V3<R>& a, const V3<R>& b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class R>
GA_HD V3<R> operator-(const V3<R>& a, const V3<R>& b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class R>
GA_HD V3<R> operator-(const V3<R>& a) { return v3(-a.x, -a.y, -a.z); }
template <class R>
GA_HD V3<R> operator*(R s, const V3<R>& a) { return v3(s * a.x, s * a.y, s * a.z); }
template <class R>
GA_HD V3<R>& operator+=(V3<R>& a, const V3<R>& b) {
  a.x += b.x;
  a.y += b.y;
  a.z += b.z;
  return a;
}
template <class R>
GA_HD R dot(const V3<R>& a, const V3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R>
GA_HD V3<R> cross(const V3<R>& a, const V3<R>& b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class R>
GA_HD V3<R> zero3() { return v3(R(0), R(0), R(0)); }

// Row-major 3x3.
template <class R>
struct M3 {
  R m[9];
};
template <class R>
GA_HD V3<R> mul(const M3<R>& A, const V3<R>& x) {
  return v3(A.m[0] * x.x + A.m[1] * x.y + A.m[2] * x.z, A.m[3] * x.x + A.m[4] * x.y + A.m[5] * x.z,
            A.m[6] * x.x + A.m[7] * x.y + A.m[8] * x.z);
}
template <class R>
GA_HD V3<R> mulT(const M3<R>& A, const V3<R>& x) {
  return v3(A.m[0] * x.x + A.m[3] * x.y + A.m[6] * x.z, A.m[1] * x.x + A.m[4] * x.y + A.m[7] * x.z,
            A.m[2] * x.x + A.m[5] * x.y + A.m[8] * x.z);
}
// A += a b^T
template <class R>
GA_HD void add_outer(M3<R>& A, const V3<R>& a, const V3<R>& b) {
  A.m[0] += a.x * b.x; A.m[1] += a.x * b.y; A.m[2] += a.x * b.z;
  A.m[3] += a.y * b.x; A.m[4] += a.y * b.y; A.m[5] += a.y * b.z;
  A.m[6] += a.z * b.x; A.m[7] += a.z * b.y; A.m[8] += a.z * b.z;
}

// Spatial 6-vector [angular; linear] (motion or force).
template <class R>
struct SV {
  V3<R> w, l;
};
template <class R>
GA_HD SV<R> sv(const V3<R>& w, const V3<R>& l) { return SV<R>{w, l}; }
template <class R>
GA_HD SV<R> sv0() { return SV<R>{zero3<R>(), zero3<R>()}; }
template <class R>
GA_HD SV<R> operator+(const SV<R>& a, const SV<R>& b) { return sv(a.w + b.w, a.l + b.l); }
template <class R>
GA_HD SV<R> operator-(const SV<R>& a, const SV<R>& b) { return sv(a.w - b.w, a.l - b.l); }
template <class R>
GA_HD SV<R>& operator+=(SV<R>& a, const SV<R>& b) {
  a.w += b.w;
  a.l += b.l;
  return a;
}
template <class R>
GA_HD R dot(const SV<R>& a, const SV<R>& b) { return dot(a.w, b.w) + dot(a.l, b.l); }
// motion cross product m x n
template <class R>
GA_HD SV<R> crm(const SV<R>& m, const SV<R>& n) { return sv(cross(m.w, n.w), cross(m.w, n.l) + cross(m.l, n.w)); }
// force cross product m x* f
template <class R>
GA_HD SV<R> crf(const SV<R>& m, const SV<R>& f) { return sv(cross(m.w, f.w) + cross(m.l, f.l), cross(m.w, f.l)); }

// ----------------------------------------- joint and tree rotations
// A(q) rotates about basis axis AX: coordinates i1 = AX+1, i2 = AX+2 (mod 3)
// mix as [x_i1'; x_i2'] = [[c, -s], [s, c]] [x_i1; x_i2].
template <int AX, class R>
GA_HD V3<R> rotA(const V3<R>& x, R c, R s) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  V3<R> r = x;
  at(r, i1) = c * cat(x, i1) - s * cat(x, i2);
  at(r, i2) = s * cat(x, i1) + c * cat(x, i2);
  return r;
}
template <int AX, class R>
GA_HD V3<R> rotAT(const V3<R>& x, R c, R s) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  V3<R> r = x;
  at(r, i1) = c * cat(x, i1) + s * cat(x, i2);
  at(r, i2) = c * cat(x, i2) - s * cat(x, i1);
  return r;
}
template <class R>
GA_HD V3<R> rotT(const BodyA<R>& b, const V3<R>& x) {
  if (b.ident) return x;
  return v3(b.T[0] * x.x + b.T[1] * x.y + b.T[2] * x.z, b.T[3] * x.x + b.T[4] * x.y + b.T[5] * x.z,
            b.T[6] * x.x + b.T[7] * x.y + b.T[8] * x.z);
}
template <class R>
GA_HD V3<R> rotTT(const BodyA<R>& b, const V3<R>& x) {
  if (b.ident) return x;
  return v3(b.T[0] * x.x + b.T[3] * x.y + b.T[6] * x.z, b.T[1] * x.x + b.T[4] * x.y + b.T[7] * x.z,
            b.T[2] * x.x + b.T[5] * x.y + b.T[8] * x.z);
}
template <class R>
GA_HD V3<R> pvec(const BodyA<R>& b) { return v3(b.p[0], b.p[1], b.p[2]); }

// Motion vector parent -> child frame: X = (E = T A, p), w' = E^T w,
// v' = E^T (v - p x w).
template <int AX, class R>
GA_HD SV<R> mot_in(const BodyA<R>& b, const SV<R>& m, R c, R s) {
  return sv(rotAT<AX>(rotTT(b, m.w), c, s), rotAT<AX>(rotTT(b, m.l - cross(pvec(b), m.w)), c, s));
}
// Force (or motion adjoint) child -> parent: X^T f = (E f.w + p x E f.l, E f.l).
template <int AX, class R>
GA_HD SV<R> frc_out(const BodyA<R>& b, const SV<R>& f, R c, R s) {
  const V3<R> l = rotT(b, rotA<AX>(f.l, c, s));
  return sv(rotT(b, rotA<AX>(f.w, c, s)) + cross(pvec(b), l), l);
}
// S x m for S = (e_AX, 0): (e x m.w, e x m.l)
template <int AX, class R>
GA_HD V3<R> ecross(const V3<R>& m) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  V3<R> r = zero3<R>();
  at(r, i1) = -cat(m, i2);
  at(r, i2) = cat(m, i1);
  return r;
}
// ybar . (S x m)
template <int AX, class R>
GA_HD R dot_scross(const SV<R>& ybar, const SV<R>& m) {
  return dot(ybar.w, ecross<AX>(m.w)) + dot(ybar.l, ecross<AX>(m.l));
}

// ---------------------------------------------------- rigid inertias
// [[J, H], [H^T, m 1]] in [angular; linear] order; J symmetric (xx yy zz xy xz yz).
template <class R>
struct RB {
  R J[6], H[9], m;
};
template <class R>
GA_HD RB<R> rigid(int i, R dmass) {
  RB<R> r;
  const BodyA<R>& b = body<R>(i);
  if (i == 0 && dmass != R(0)) {  // pelvis with a mass offset, COM and its inertia unchanged
    const ModelA<R>& M = model<R>();
    const R cx = M.com0[0], cy = M.com0[1], cz = M.com0[2], m = b.m + dmass;
    r.J[0] = M.icom0[0] + m * (cy * cy + cz * cz);
    r.J[1] = M.icom0[1] + m * (cx * cx + cz * cz);
    r.J[2] = M.icom0[2] + m * (cx * cx + cy * cy);
    r.J[3] = M.icom0[3] - m * (cx * cy);
    r.J[4] = M.icom0[4] - m * (cx * cz);
    r.J[5] = M.icom0[5] - m * (cy * cz);
    r.H[0] = R(0);    r.H[1] = -m * cz; r.H[2] = m * cy;
    r.H[3] = m * cz;  r.H[4] = R(0);    r.H[5] = -m * cx;
    r.H[6] = -m * cy; r.H[7] = m * cx;  r.H[8] = R(0);
    r.m = m;
    return r;
  }
  for (int k = 0; k < 6; ++k) r.J[k] = b.J[k];
  for (int k = 0; k < 9; ++k) r.H[k] = b.H[k];
  r.m = b.m;
  return r;
}
template <class R>
GA_HD V3<R> symv(const R* J, const V3<R>& x) {
  return v3(J[0] * x.x + J[3] * x.y + J[4] * x.z, J[3] * x.x + J[1] * x.y + J[5] * x.z,
            J[4] * x.x + J[5] * x.y + J[2] * x.z);
}
template <class R>
GA_HD SV<R> imul(const RB<R>& I, const SV<R>& x) {
  const R* H = I.H;
  const V3<R> Hl = v3(H[0] * x.l.x + H[1] * x.l.y + H[2] * x.l.z, H[3] * x.l.x + H[4] * x.l.y + H[5] * x.l.z,
                      H[6] * x.l.x + H[7] * x.l.y + H[8] * x.l.z);
  const V3<R> HTw = v3(H[0] * x.w.x + H[3] * x.w.y + H[6] * x.w.z, H[1] * x.w.x + H[4] * x.w.y + H[7] * x.w.z,
                       H[2] * x.w.x + H[5] * x.w.y + H[8] * x.w.z);
  return sv(symv(I.J, x.w) + Hl, HTw + I.m * x.l);
}

// Articulated inertia [[J, H], [H^T, M]] (J, M symmetric).
template <class R>
struct AI {
  R J[6], H[9], M[6];
};
GA_HD constexpr int sidx(int r, int c) {
  return r == c ? r : ((r == 0 && c == 1) || (r == 1 && c == 0)) ? 3 : ((r == 0 && c == 2) || (r == 2 && c == 0)) ? 4 : 5;
}
template <class R>
GA_HD AI<R> ai_of(const RB<R>& I) {
  AI<R> A;
  for (int k = 0; k < 6; ++k) A.J[k] = I.J[k];
  for (int k = 0; k < 9; ++k) A.H[k] = I.H[k];
  A.M[0] = A.M[1] = A.M[2] = I.m;
  A.M[3] = A.M[4] = A.M[5] = R(0);
  return A;
}
template <class R>
GA_HD void ai_add(AI<R>& A, const AI<R>& B) {
  for (int k = 0; k < 6; ++k) {
    A.J[k] += B.J[k];
    A.M[k] += B.M[k];
  }
  for (int k = 0; k < 9; ++k) A.H[k] += B.H[k];
}

// A S A^T for symmetric S under the joint rotation about AX.
template <int AX, class R>
GA_HD void rotA_sym(R* S, R c, R s) {
  constexpr int k = AX, i = (AX + 1) % 3, j = (AX + 2) % 3;
  const R sii = S[sidx(i, i)], sjj = S[sidx(j, j)], sij = S[sidx(i, j)];
  const R sik = S[sidx(i, k)], sjk = S[sidx(j, k)];
  const R bii = c * sii - s * sij, bij = c * sij - s * sjj;
  const R bji = s * sii + c * sij, bjj = s * sij + c * sjj;
  S[sidx(i, k)] = c * sik - s * sjk;
  S[sidx(j, k)] = s * sik + c * sjk;
  S[sidx(i, i)] = c * bii - s * bij;
  S[sidx(j, j)] = s * bji + c * bjj;
  S[sidx(i, j)] = s * bii + c * bij;
}
template <int AX, class R>
GA_HD void rotA_gen(R* H, R c, R s) {
  constexpr int i = (AX + 1) % 3, j = (AX + 2) % 3;
  for (int col = 0; col < 3; ++col) {
    const R a = H[3 * i + col], b = H[3 * j + col];
    H[3 * i + col] = c * a - s * b;
    H[3 * j + col] = s * a + c * b;
  }
  for (int row = 0; row < 3; ++row) {
    const R a = H[3 * row + i], b = H[3 * row + j];
    H[3 * row + i] = c * a - s * b;
    H[3 * row + j] = s * a + c * b;
  }
}
template <class R>
GA_HD void rotT_sym(const BodyA<R>& b, R* S) {
  R B[9];
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c)
      B[3 * a + c] = b.T[3 * a] * S[sidx(0, c)] + b.T[3 * a + 1] * S[sidx(1, c)] + b.T[3 * a + 2] * S[sidx(2, c)];
  R r[6];
  for (int a = 0; a < 3; ++a)
    for (int c = a; c < 3; ++c)
      r[sidx(a, c)] = B[3 * a] * b.T[3 * c] + B[3 * a + 1] * b.T[3 * c + 1] + B[3 * a + 2] * b.T[3 * c + 2];
  for (int k = 0; k < 6; ++k) S[k] = r[k];
}
template <class R>
GA_HD void rotT_gen(const BodyA<R>& b, R* H) {
  R B[9];
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c) B[3 * a + c] = b.T[3 * a] * H[c] + b.T[3 * a + 1] * H[3 + c] + b.T[3 * a + 2] * H[6 + c];
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c)
      H[3 * a + c] = B[3 * a] * b.T[3 * c] + B[3 * a + 1] * b.T[3 * c + 1] + B[3 * a + 2] * b.T[3 * c + 2];
}
// acc += X^T Ia X (child articulated inertia moved into the parent frame).
template <int AX, class R>
GA_HD void ai_to_parent_add(const BodyA<R>& b, AI<R>& acc, AI<R> Ia, R c, R s) {
  rotA_sym<AX>(Ia.J, c, s);
  rotA_gen<AX>(Ia.H, c, s);
  rotA_sym<AX>(Ia.M, c, s);
  if (!b.ident) {
    rotT_sym(b, Ia.J);
    rotT_gen(b, Ia.H);
    rotT_sym(b, Ia.M);
  }
  const V3<R> p = pvec(b);
  R Hn[9];
  for (int col = 0; col < 3; ++col) {  // H' = H + [p]x M
    const V3<R> pm = cross(p, v3(Ia.M[sidx(0, col)], Ia.M[sidx(1, col)], Ia.M[sidx(2, col)]));
    Hn[col] = Ia.H[col] + pm.x;
    Hn[3 + col] = Ia.H[3 + col] + pm.y;
    Hn[6 + col] = Ia.H[6 + col] + pm.z;
  }
  // J' = J + [p]x H^T - H' [p]x
  V3<R> pHT[3], HnP[3];
  for (int cc = 0; cc < 3; ++cc) pHT[cc] = cross(p, v3(Ia.H[3 * cc], Ia.H[3 * cc + 1], Ia.H[3 * cc + 2]));
  for (int r = 0; r < 3; ++r) HnP[r] = cross(p, v3(Hn[3 * r], Hn[3 * r + 1], Hn[3 * r + 2]));
  for (int r = 0; r < 3; ++r)
    for (int cc = r; cc < 3; ++cc) acc.J[sidx(r, cc)] += Ia.J[sidx(r, cc)] + cat(pHT[cc], r) + cat(HnP[r], cc);
  for (int k = 0; k < 9; ++k) acc.H[k] += Hn[k];
  for (int k = 0; k < 6; ++k) acc.M[k] += Ia.M[k];
}

// ------------------------------------------------------------- tape
// Per-env storage, slot k at p[k * STRIDE].
template <class R, int STRIDE>
struct Tape {
  R* p;
  GA_HD R get(int k) const { return p[k * STRIDE]; }
  GA_HD void put(int k, R v) { p[k * STRIDE] = v; }
  GA_HD void add(int k, R v) { p[k * STRIDE] += v; }
};
// body b: twist w (3), v (3), gravity g (3), acceleration a (6), psi (6)
constexpr int kSB = 21;
GA_HD constexpr int tb(int b, int k) { return kSB * b + k; }
enum { kBw = 0, kBv = 3, kBg = 6, kBa = 9, kBpsi = 15 };
// hinge body i (1..29): cos, sin, U/D (6), 1/D, u/D, qdd, branch flags,
// y (nu_dot_bar, then u/D of the mu solve, then mu), qbar, qdbar
constexpr int kSH = 15;
constexpr int kTH0 = kSB * kNB;
GA_HD constexpr int th(int i, int k) { return kTH0 + kSH * (i - 1) + k; }
enum { kHc = 0, kHs = 1, kHW = 2, kHinvD = 8, kHuD = 9, kHqdd = 10, kHflag = 11, kHy = 12, kHqb = 13, kHqdb = 14 };
// foot f: world rotation (9), world position (3), contact wrench W_ext (6), sphere flags
constexpr int kSF = 19;
constexpr int kTF0 = kTH0 + kSH * kNJ;
GA_HD constexpr int tf(int f, int k) { return kTF0 + kSF * f + k; }
enum { kFR = 0, kFP = 9, kFW = 12, kFflag = 18 };
// base: LDL^T of the base articulated inertia (strict lower L 15, 1/d 6)
constexpr int kTL0 = kTF0 + kSF * 2;
constexpr int kTapeSlots = kTL0 + 21;

template <class R, class Tp>
GA_HD void put3(Tp& tp, int k, const V3<R>& v) {
  tp.put(k, v.x);
  tp.put(k + 1, v.y);
  tp.put(k + 2, v.z);
}
template <class R, class Tp>
GA_HD V3<R> get3(const Tp& tp, int k) { return v3(tp.get(k), tp.get(k + 1), tp.get(k + 2)); }
template <class R, class Tp>
GA_HD void put6(Tp& tp, int k, const SV<R>& v) {
  put3(tp, k, v.w);
  put3(tp, k + 3, v.l);
}
template <class R, class Tp>
GA_HD SV<R> get6(const Tp& tp, int k) { return sv(get3<R>(tp, k), get3<R>(tp, k + 3)); }

// chains: 0 left leg 1-6, 1 right leg 7-12, 2 waist 13-15, 3 left arm 16-22,
// 4 right arm 23-29 (legs and waist hang off the pelvis, arms off body 15)
GA_HD constexpr int chain_first(int c) { return c == 0 ? 1 : c == 1 ? 7 : c == 2 ? 13 : c == 3 ? 16 : 23; }
GA_HD constexpr int chain_last(int c) { return c == 0 ? 6 : c == 1 ? 12 : c == 2 ? 15 : c == 3 ? 22 : 29; }
GA_HD constexpr int chain_parent(int c) { return c < 3 ? 0 : 15; }

// ---------------------------------------------------- base kinematics
template <class R>
struct Base {
  R pos[3], quat[4], vw[3], wb[3];
};
template <class R>
GA_HD void quat_rot(const R* q, M3<R>& M) {  // rotation of a unit quaternion (w, x, y, z)
  const R w = q[0], x = q[1], y = q[2], z = q[3];
  M.m[0] = R(1) - R(2) * (y * y + z * z); M.m[1] = R(2) * (x * y - w * z); M.m[2] = R(2) * (x * z + w * y);
  M.m[3] = R(2) * (x * y + w * z); M.m[4] = R(1) - R(2) * (x * x + z * z); M.m[5] = R(2) * (y * z - w * x);
  M.m[6] = R(2) * (x * z - w * y); M.m[7] = R(2) * (y * z + w * x); M.m[8] = R(1) - R(2) * (x * x + y * y);
}
// unit quaternion, its norm and rotation from the stored (not exactly unit) one
template <class R>
GA_HD void base_frame(const Base<R>& st, R* qn, R& qnorm, M3<R>& R0) {
  qnorm = sqrt(st.quat[0] * st.quat[0] + st.quat[1] * st.quat[1] + st.quat[2] * st.quat[2] + st.quat[3] * st.quat[3]);
  const R inv = R(1) / qnorm;
  for (int k = 0; k < 4; ++k) qn[k] = st.quat[k] * inv;
  quat_rot(qn, R0);
}

// ============================================================== primal
// Accessors: X reads (and with kWrite writes) the 87 state entries of the
// env (hinge angles, rates, anchors); U reads the 29 targets.
template <int AX, bool kLeg, class R, class Tp, class X>
GA_HD void fk_body(int i, const X& x, V3<R>& w, V3<R>& v, V3<R>& g, M3<R>& Rw, V3<R>& Pw, Tp& tp) {
  const BodyA<R>& b = body<R>(i);
  const R q = x.get(6 + i), qd = x.get(kQV + 5 + i);
  const R s = sin(q), c = cos(q);
  tp.put(th(i, kHc), c);
  tp.put(th(i, kHs), s);
  const SV<R> m = mot_in<AX>(b, sv(w, v), c, s);
  w = m.w;
  at(w, AX) += qd;
  v = m.l;
  g = rotAT<AX>(rotTT(b, g), c, s);
  put3(tp, tb(i, kBw), w);
  put3(tp, tb(i, kBv), v);
  put3(tp, tb(i, kBg), g);
  if constexpr (kLeg) {  // world pose: P_i = P_p + R_p p ; R_i = R_p T A
    Pw = Pw + mul(Rw, pvec(b));
    M3<R> E;  // E = T A : columns of T rotated
    for (int a = 0; a < 3; ++a) {
      const V3<R> row = rotAT<AX>(v3(b.ident ? R(a == 0) : b.T[3 * a], b.ident ? R(a == 1) : b.T[3 * a + 1],
                                     b.ident ? R(a == 2) : b.T[3 * a + 2]),
                                  c, s);  // row a of T A = (A^T T^T e_a)^T
      E.m[3 * a] = row.x;
      E.m[3 * a + 1] = row.y;
      E.m[3 * a + 2] = row.z;
    }
    M3<R> Rn;
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc)
        Rn.m[3 * r + cc] = Rw.m[3 * r] * E.m[cc] + Rw.m[3 * r + 1] * E.m[3 + cc] + Rw.m[3 * r + 2] * E.m[6 + cc];
    Rw = Rn;
  }
}
template <bool kLeg, class R, class Tp, class X>
GA_HD void fk_chain(int c, const X& x, M3<R>& Rw, V3<R>& Pw, Tp& tp) {
  const int p = chain_parent(c);
  V3<R> w = get3<R>(tp, tb(p, kBw)), v = get3<R>(tp, tb(p, kBv)), g = get3<R>(tp, tb(p, kBg));
  for (int i = chain_first(c); i <= chain_last(c); ++i) {
    switch (body<R>(i).axis) {
      case 0: fk_body<0, kLeg>(i, x, w, v, g, Rw, Pw, tp); break;
      case 1: fk_body<1, kLeg>(i, x, w, v, g, Rw, Pw, tp); break;
      default: fk_body<2, kLeg>(i, x, w, v, g, Rw, Pw, tp); break;
    }
  }
}

// Sphere contact flags (4 bits per sphere k of a foot, in a small integer):
// bit 0 in contact, bit 1 fresh anchor, bit 2 slip, bit 3 normal force in
// its linear range (0 < fn_raw < 500).
enum { kCin = 1, kCfresh = 2, kCslip = 4, kClin = 8 };

// Contacts of foot f (spheres 4f .. 4f+3) from the foot's world pose and
// twist (reference src/g1_core.h:123-153); stores the body-frame contact
// wrench W_ext and the flags; with kWrite updates the anchors in x.
template <bool kWrite, class R, class Tp, class X>
GA_HD void foot_contacts(int f, const M3<R>& Rw, const V3<R>& Pw, X& x, const Cfg<R>& cfg, R mu, Tp& tp) {
  const int ib = f == 0 ? 6 : 12;
  const V3<R> w = get3<R>(tp, tb(ib, kBw)), v = get3<R>(tp, tb(ib, kBv));
  const ModelA<R>& M = model<R>();
  V3<R> F = zero3<R>(), Tq = zero3<R>();
  int flags = 0;
  for (int j = 0; j < 4; ++j) {
    const int k = 4 * f + j;
    const V3<R> r = v3(M.cpos[3 * k], M.cpos[3 * k + 1], M.cpos[3 * k + 2]);
    const V3<R> rw = mul(Rw, r);
    const V3<R> pc = Pw + rw;
    const V3<R> vp = mul(Rw, v + cross(w, r));
    const R depth = M.radius - pc.z;
    const R fr = cfg.kn * depth - cfg.dn * vp.z;
    const R fn = fr < R(0) ? R(0) : (fr > R(500) ? R(500) : fr);
    R ax = x.get(kAN + 2 * k), ay = x.get(kAN + 2 * k + 1);
    const bool fresh = ax >= R(1e29);
    if (fresh) {
      ax = pc.x;
      ay = pc.y;
    }
    R ftx = -cfg.kt * (pc.x - ax) - cfg.dtc * vp.x;
    R fty = -cfg.kt * (pc.y - ay) - cfg.dtc * vp.y;
    const R ftn = sqrt(ftx * ftx + fty * fty), fmax = mu * fn;
    const bool slip = ftn > fmax;
    if (slip) {
      const R scl = fmax / (ftn + R(1e-12));
      ftx *= scl;
      fty *= scl;
      ax = pc.x + ftx / cfg.kt;
      ay = pc.y + fty / cfg.kt;
    }
    const bool in = depth > R(0);
    if (in) {
      const V3<R> fk = v3(ftx, fty, fn);
      F += fk;
      Tq += cross(rw, fk);
    }
    if constexpr (kWrite) {
      x.put(kAN + 2 * k, in ? ax : R(1e30));
      x.put(kAN + 2 * k + 1, in ? ay : R(1e30));
    }
    flags |= ((in ? kCin : 0) | (fresh ? kCfresh : 0) | (slip ? kCslip : 0) | ((fr > R(0) && fr < R(500)) ? kClin : 0))
             << (4 * j);
  }
  put3(tp, tf(f, kFW), mulT(Rw, Tq));
  put3(tp, tf(f, kFW + 3), mulT(Rw, F));
  tp.put(tf(f, kFflag), (R)flags);
  for (int k = 0; k < 9; ++k) tp.put(tf(f, kFR + k), Rw.m[k]);
  put3(tp, tf(f, kFP), Pw);
}

// rigid-body bias with gravity: v x* (I v) - I (0, g)
template <class R>
GA_HD SV<R> bias(const RB<R>& I, const SV<R>& v, const V3<R>& g) {
  return crf(v, imul(I, v)) - imul(I, sv(zero3<R>(), g));
}

// Servo torque with soft limits (reference src/g1_core.h:166-177).  Flags:
// bit 0 torque clamped, bit 1 below the lower limit, bit 2 above the upper.
template <class R>
GA_HD R servo(const BodyA<R>& b, R q, R qd, R u, const Par<R>& par, const Cfg<R>& cfg, R& bd, int& flags) {
  const R kp = b.kp * par.kps, kv = b.kv * par.kds;
  const R t0 = kp * (u - q) - kv * qd;
  R t = t0 < -b.lim ? -b.lim : (t0 > b.lim ? b.lim : t0);
  flags = (t0 < -b.lim || t0 > b.lim) ? 1 : 0;
  bd = kv + b.damp;
  if (q < b.lo) {
    t += cfg.lkp * (b.lo - q) - cfg.lkd * qd;
    bd += cfg.lkd;
    flags |= 2;
  }
  if (q > b.hi) {
    t += cfg.lkp * (b.hi - q) - cfg.lkd * qd;
    bd += cfg.lkd;
    flags |= 4;
  }
  return t - b.damp * qd;
}

// One hinge of the ABA backward pass: (IA, pA) of body i -> projection into
// the parent, added to (accI, accP).
template <int AX, class R, class Tp, class X, class UA>
GA_HD void aba_bwd_body(int i, const AI<R>& IA, const SV<R>& pA, AI<R>& accI, SV<R>& accP, const X& x, const UA& u,
                        const Par<R>& par, const Cfg<R>& cfg, Tp& tp) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const BodyA<R>& b = body<R>(i);
  const R c = tp.get(th(i, kHc)), s = tp.get(th(i, kHs));
  const R q = x.get(6 + i), qd = x.get(kQV + 5 + i);
  SV<R> U;
  U.w = v3(IA.J[sidx(0, AX)], IA.J[sidx(1, AX)], IA.J[sidx(2, AX)]);
  U.l = v3(IA.H[3 * AX], IA.H[3 * AX + 1], IA.H[3 * AX + 2]);
  R bd;
  int flags;
  const R tau = servo(b, q, qd, u.get(i - 1), par, cfg, bd, flags);
  const R D = cat(U.w, AX) + b.arm + cfg.dt * bd;
  const R uu = tau - cat(pA.w, AX);
  const R invD = R(1) / D;
  const SV<R> W = sv(invD * U.w, invD * U.l);
  const R uD = uu * invD;
  put6(tp, th(i, kHW), W);
  tp.put(th(i, kHinvD), invD);
  tp.put(th(i, kHuD), uD);
  tp.put(th(i, kHflag), (R)flags);
  AI<R> Ia;
  for (int a = 0; a < 3; ++a)
    for (int bb = a; bb < 3; ++bb) {
      Ia.J[sidx(a, bb)] = IA.J[sidx(a, bb)] - cat(U.w, a) * cat(W.w, bb);
      Ia.M[sidx(a, bb)] = IA.M[sidx(a, bb)] - cat(U.l, a) * cat(W.l, bb);
    }
  for (int a = 0; a < 3; ++a)
    for (int bb = 0; bb < 3; ++bb) Ia.H[3 * a + bb] = IA.H[3 * a + bb] - cat(U.w, a) * cat(W.l, bb);
  // velocity product c = v x (S qd): four non-zeros
  const V3<R> w = get3<R>(tp, tb(i, kBw)), v = get3<R>(tp, tb(i, kBv));
  const R c0 = qd * cat(w, i2), c1 = -(qd * cat(w, i1)), c2 = qd * cat(v, i2), c3 = -(qd * cat(v, i1));
  SV<R> pa;
  for (int a = 0; a < 3; ++a) {
    at(pa.w, a) = cat(pA.w, a) + Ia.J[sidx(a, i1)] * c0 + Ia.J[sidx(a, i2)] * c1 + Ia.H[3 * a + i1] * c2 +
                  Ia.H[3 * a + i2] * c3 + uD * cat(U.w, a);
    at(pa.l, a) = cat(pA.l, a) + Ia.H[3 * i1 + a] * c0 + Ia.H[3 * i2 + a] * c1 + Ia.M[sidx(a, i1)] * c2 +
                  Ia.M[sidx(a, i2)] * c3 + uD * cat(U.l, a);
  }
  ai_to_parent_add<AX>(b, accI, Ia, c, s);
  accP += frc_out<AX>(b, pa, c, s);
}

// Backward pass over chain c from (IA, pA) of its last body; returns the
// chain's projection into its parent.
template <class R, class Tp, class X, class UA>
GA_HD void aba_bwd_chain(int c, AI<R> IA, SV<R> pA, AI<R>& outI, SV<R>& outP, const X& x, const UA& u, const Par<R>& par,
                         const Cfg<R>& cfg, Tp& tp) {
  const int first = chain_first(c);
  for (int i = chain_last(c); i >= first; --i) {
    AI<R> IAp;
    SV<R> pAp = sv0<R>();
    if (i > first) {
      const RB<R> I = rigid<R>(i - 1, R(0));
      IAp = ai_of(I);
      pAp = bias(I, get6<R>(tp, tb(i - 1, kBw)), get3<R>(tp, tb(i - 1, kBg)));
    } else {
      for (int k = 0; k < 6; ++k) IAp.J[k] = IAp.M[k] = R(0);
      for (int k = 0; k < 9; ++k) IAp.H[k] = R(0);
    }
    switch (body<R>(i).axis) {
      case 0: aba_bwd_body<0>(i, IA, pA, IAp, pAp, x, u, par, cfg, tp); break;
      case 1: aba_bwd_body<1>(i, IA, pA, IAp, pAp, x, u, par, cfg, tp); break;
      default: aba_bwd_body<2>(i, IA, pA, IAp, pAp, x, u, par, cfg, tp); break;
    }
    IA = IAp;
    pA = pAp;
  }
  outI = IA;
  outP = pA;
}

// LDL^T of the base articulated inertia, kept on the tape (reference
// src/spatial.h:254-278 factors the same matrix by Cholesky).
template <class R, class Tp>
GA_HD void ldl_factor(const AI<R>& A, Tp& tp) {
  R m[6][6];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      m[a][b] = A.J[sidx(a, b)];
      m[3 + a][3 + b] = A.M[sidx(a, b)];
      m[a][3 + b] = A.H[3 * a + b];
      m[3 + b][a] = A.H[3 * a + b];
    }
  R L[6][6], d[6];
  for (int j = 0; j < 6; ++j) {
    R dj = m[j][j];
    for (int k = 0; k < j; ++k) dj -= L[j][k] * L[j][k] * d[k];
    d[j] = dj;
    const R id = R(1) / dj;
    tp.put(kTL0 + 15 + j, id);
    for (int i = j + 1; i < 6; ++i) {
      R xx = m[i][j];
      for (int k = 0; k < j; ++k) xx -= L[i][k] * L[j][k] * d[k];
      L[i][j] = xx * id;
    }
  }
  int n = 0;
  for (int i = 1; i < 6; ++i)
    for (int j = 0; j < i; ++j) tp.put(kTL0 + n++, L[i][j]);
}
template <class R, class Tp>
GA_HD SV<R> ldl_solve(const SV<R>& rhs, const Tp& tp) {
  R y[6] = {rhs.w.x, rhs.w.y, rhs.w.z, rhs.l.x, rhs.l.y, rhs.l.z};
  int n = 0;
  for (int i = 1; i < 6; ++i)
    for (int k = 0; k < i; ++k) y[i] -= tp.get(kTL0 + n++) * y[k];
  for (int i = 0; i < 6; ++i) y[i] *= tp.get(kTL0 + 15 + i);
  for (int i = 5; i >= 0; --i)
    for (int k = i + 1; k < 6; ++k) y[i] -= tp.get(kTL0 + (k * (k - 1)) / 2 + i) * y[k];
  return sv(v3(y[0], y[1], y[2]), v3(y[3], y[4], y[5]));
}

// Forward pass of one hinge: a_i = X a_p + c_i, qdd, a_i += qdd S; with
// kWrite the hinge's semi-implicit Euler update.
template <int AX, bool kWrite, class R, class Tp, class X>
GA_HD void aba_fwd_body(int i, SV<R>& a, X& x, R dt, Tp& tp) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const BodyA<R>& b = body<R>(i);
  const R c = tp.get(th(i, kHc)), s = tp.get(th(i, kHs));
  const R qd = x.get(kQV + 5 + i);
  const V3<R> w = get3<R>(tp, tb(i, kBw)), v = get3<R>(tp, tb(i, kBv));
  SV<R> an = mot_in<AX>(b, a, c, s);
  at(an.w, i1) += qd * cat(w, i2);
  at(an.w, i2) += -(qd * cat(w, i1));
  at(an.l, i1) += qd * cat(v, i2);
  at(an.l, i2) += -(qd * cat(v, i1));
  const SV<R> W = get6<R>(tp, th(i, kHW));
  const R qdd = tp.get(th(i, kHuD)) - dot(W, an);
  at(an.w, AX) += qdd;
  a = an;
  tp.put(th(i, kHqdd), qdd);
  put6(tp, tb(i, kBa), an);
  if constexpr (kWrite) {
    const R qd1 = qd + dt * qdd;
    x.put(kQV + 5 + i, qd1);
    x.put(6 + i, x.get(6 + i) + dt * qd1);
  }
}
template <bool kWrite, class R, class Tp, class X>
GA_HD void aba_fwd_chain(int c, X& x, R dt, Tp& tp) {
  SV<R> a = get6<R>(tp, tb(chain_parent(c), kBa));
  for (int i = chain_first(c); i <= chain_last(c); ++i) {
    switch (body<R>(i).axis) {
      case 0: aba_fwd_body<0, kWrite>(i, a, x, dt, tp); break;
      case 1: aba_fwd_body<1, kWrite>(i, a, x, dt, tp); break;
      default: aba_fwd_body<2, kWrite>(i, a, x, dt, tp); break;
    }
  }
}

// One substep.  st: base state (in / out with kWrite); x: hinge state and
// anchors (read; written with kWrite); u: targets.  Fills the tape.
template <bool kWrite, class R, class Tp, class X, class UA>
GA_HD void primal(Base<R>& st, X& x, const UA& u, const Par<R>& par, const Cfg<R>& cfg, Tp& tp) {
  R qn[4], qnorm;
  M3<R> R0;
  base_frame(st, qn, qnorm, R0);
  const V3<R> w0 = v3(st.wb[0], st.wb[1], st.wb[2]);
  const V3<R> v0 = mulT(R0, v3(st.vw[0], st.vw[1], st.vw[2]));
  const V3<R> g0 = cfg.gz * v3(R0.m[6], R0.m[7], R0.m[8]);
  put3(tp, tb(0, kBw), w0);
  put3(tp, tb(0, kBv), v0);
  put3(tp, tb(0, kBg), g0);
  // FK: waist, arms, then the legs with their world pose and contacts
  M3<R> Rd = R0;
  V3<R> Pd = zero3<R>();
  for (int c = 2; c < 5; ++c) fk_chain<false>(c, x, Rd, Pd, tp);
  for (int f = 0; f < 2; ++f) {
    M3<R> Rw = R0;
    V3<R> Pw = v3(st.pos[0], st.pos[1], st.pos[2]);
    fk_chain<true>(f, x, Rw, Pw, tp);
    foot_contacts<kWrite>(f, Rw, Pw, x, cfg, par.mu, tp);
  }
  // ABA backward: arms into the torso, waist into the pelvis, legs into the pelvis
  AI<R> acc15;
  SV<R> p15;
  {
    const RB<R> I15 = rigid<R>(15, R(0));
    acc15 = ai_of(I15);
    p15 = bias(I15, get6<R>(tp, tb(15, kBw)), get3<R>(tp, tb(15, kBg)));
  }
  for (int c = 3; c < 5; ++c) {
    const int last = chain_last(c);
    const RB<R> I = rigid<R>(last, R(0));
    AI<R> ci;
    SV<R> cp;
    aba_bwd_chain(c, ai_of(I), bias(I, get6<R>(tp, tb(last, kBw)), get3<R>(tp, tb(last, kBg))), ci, cp, x, u, par,
                  cfg, tp);
    ai_add(acc15, ci);
    p15 += cp;
  }
  const RB<R> I0 = rigid<R>(0, par.dmass);
  AI<R> acc0 = ai_of(I0);
  SV<R> p0 = bias(I0, sv(w0, v0), g0);
  {
    AI<R> ci;
    SV<R> cp;
    aba_bwd_chain(2, acc15, p15, ci, cp, x, u, par, cfg, tp);
    ai_add(acc0, ci);
    p0 += cp;
  }
  for (int f = 0; f < 2; ++f) {
    const int last = chain_last(f);
    const RB<R> I = rigid<R>(last, R(0));
    const SV<R> pA = bias(I, get6<R>(tp, tb(last, kBw)), get3<R>(tp, tb(last, kBg))) - get6<R>(tp, tf(f, kFW));
    AI<R> ci;
    SV<R> cp;
    aba_bwd_chain(f, ai_of(I), pA, ci, cp, x, u, par, cfg, tp);
    ai_add(acc0, ci);
    p0 += cp;
  }
  ldl_factor(acc0, tp);
  const SV<R> a0 = ldl_solve(sv(-p0.w, -p0.l), tp);
  put6(tp, tb(0, kBa), a0);
  // forward: waist first (the arms start from the torso's acceleration)
  aba_fwd_chain<kWrite>(2, x, cfg.dt, tp);
  aba_fwd_chain<kWrite>(3, x, cfg.dt, tp);
  aba_fwd_chain<kWrite>(4, x, cfg.dt, tp);
  aba_fwd_chain<kWrite>(0, x, cfg.dt, tp);
  aba_fwd_chain<kWrite>(1, x, cfg.dt, tp);
  if constexpr (kWrite) {  // base (reference src/g1_core.h:203-206, 215-220)
    const R dt = cfg.dt;
    const V3<R> al = mul(R0, a0.l + cross(w0, v0));
    for (int k = 0; k < 3; ++k) st.vw[k] += dt * cat(al, k);
    for (int k = 0; k < 3; ++k) st.wb[k] += dt * cat(a0.w, k);
    for (int k = 0; k < 3; ++k) st.pos[k] += dt * st.vw[k];
    const R wx = st.wb[0], wy = st.wb[1], wz = st.wb[2];
    const R wn = sqrt(wx * wx + wy * wy + wz * wz);
    if (wn * dt >= R(1e-12)) {
      const R sh = sin(R(0.5) * wn * dt), ch = cos(R(0.5) * wn * dt);
      const R k = sh / wn;
      const R d[4] = {ch, k * wx, k * wy, k * wz};
      const R* q = st.quat;
      R r[4];
      r[0] = q[0] * d[0] - q[1] * d[1] - q[2] * d[2] - q[3] * d[3];
      r[1] = q[0] * d[1] + q[1] * d[0] + q[2] * d[3] - q[3] * d[2];
      r[2] = q[0] * d[2] - q[1] * d[3] + q[2] * d[0] + q[3] * d[1];
      r[3] = q[0] * d[3] + q[1] * d[2] - q[2] * d[1] + q[3] * d[0];
      const R n = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
      const R inv = R(1) / n;
      for (int j = 0; j < 4; ++j) st.quat[j] = r[j] * inv;
    }
  }
}

// ============================================================= reverse
// Accumulated adjoints of the base state (body-frame twist kept apart
// until the end) and of the base rotation.
template <class R>
struct BaseBar {
  V3<R> pos, vw, wb, w0, v0;  // w0, v0: adjoint of the body-frame base twist
  R quat[4];
  M3<R> R0;
};

// mu solve, backward over one chain: p of the last body is zero (no
// children); returns the projection into the parent.
template <int AX, class R, class Tp>
GA_HD void mus_bwd_body(int i, SV<R>& p, Tp& tp) {
  const BodyA<R>& b = body<R>(i);
  const R c = tp.get(th(i, kHc)), s = tp.get(th(i, kHs));
  const SV<R> W = get6<R>(tp, th(i, kHW));
  const R uu = tp.get(th(i, kHy)) - cat(p.w, AX);
  tp.put(th(i, kHy), uu * tp.get(th(i, kHinvD)));  // u / D
  p = frc_out<AX>(b, p + sv(uu * W.w, uu * W.l), c, s);
}
template <class R, class Tp>
GA_HD SV<R> mus_bwd_chain(int c, Tp& tp) {
  SV<R> p = sv0<R>();
  for (int i = chain_last(c); i >= chain_first(c); --i) {
    switch (body<R>(i).axis) {
      case 0: mus_bwd_body<0>(i, p, tp); break;
      case 1: mus_bwd_body<1>(i, p, tp); break;
      default: mus_bwd_body<2>(i, p, tp); break;
    }
  }
  return p;
}
template <class R, class Tp>
GA_HD SV<R> mus_bwd_chain_from(int c, SV<R> p, Tp& tp) {  // chain whose last body already carries p
  for (int i = chain_last(c); i >= chain_first(c); --i) {
    switch (body<R>(i).axis) {
      case 0: mus_bwd_body<0>(i, p, tp); break;
      case 1: mus_bwd_body<1>(i, p, tp); break;
      default: mus_bwd_body<2>(i, p, tp); break;
    }
  }
  return p;
}
// mu solve, forward: a_i = X a_p, mu_i = u/D - W . a_i, a_i += mu_i S;
// psi_i = -a_i is stored (the bodies' velocities under -mu), mu_i in y.
template <int AX, class R, class Tp>
GA_HD void mus_fwd_body(int i, SV<R>& a, Tp& tp) {
  const BodyA<R>& b = body<R>(i);
  const R c = tp.get(th(i, kHc)), s = tp.get(th(i, kHs));
  SV<R> an = mot_in<AX>(b, a, c, s);
  const R mu = tp.get(th(i, kHy)) - dot(get6<R>(tp, th(i, kHW)), an);
  at(an.w, AX) += mu;
  a = an;
  tp.put(th(i, kHy), mu);
  put6(tp, tb(i, kBpsi), sv(-an.w, -an.l));
}
template <class R, class Tp>
GA_HD void mus_fwd_chain(int c, Tp& tp) {
  const SV<R> psi = get6<R>(tp, tb(chain_parent(c), kBpsi));
  SV<R> a = sv(-psi.w, -psi.l);
  for (int i = chain_first(c); i <= chain_last(c); ++i) {
    switch (body<R>(i).axis) {
      case 0: mus_fwd_body<0>(i, a, tp); break;
      case 1: mus_fwd_body<1>(i, a, tp); break;
      default: mus_fwd_body<2>(i, a, tp); break;
    }
  }
}

// Adjoints carried up a chain of the Psi reverse: of psi (P), of the
// gravity-offset acceleration at (A) and of the twist v (V); for the legs
// also of the world pose (Rb, Pb) with the running world rotation Rw.
template <class R>
struct Up {
  SV<R> P, A, V;
  M3<R> Rb, Rw;
  V3<R> Pb;
};

// Body i's own term of Psi: psi . (I at + v x* I v - W_ext).
template <class R, class Tp>
GA_HD void psi_own(int i, R dmass, const SV<R>& Wext, Up<R>& up, const Tp& tp) {
  const RB<R> I = rigid<R>(i, i == 0 ? dmass : R(0));
  const SV<R> v = get6<R>(tp, tb(i, kBw));
  const SV<R> psi = get6<R>(tp, tb(i, kBpsi));
  const SV<R> at_ = get6<R>(tp, tb(i, kBa)) - sv(zero3<R>(), get3<R>(tp, tb(i, kBg)));
  const SV<R> Iv = imul(I, v);
  up.P += imul(I, at_) + crf(v, Iv) - Wext;
  up.A += imul(I, psi);
  up.V += imul(I, crm(psi, v)) - crf(psi, Iv);
}

// Servo terms of hinge i with mu_i: q, qd, target and gain-scale adjoints,
// and the implicit-damping term of the kd scale.
template <class R, class Tp, class X, class UA, class UB>
GA_HD void servo_rev(int i, const X& x, const UA& u, UB& ubar, const Par<R>& par, const Cfg<R>& cfg, R& qb, R& qdb,
                     R& kpb, R& kdb, const Tp& tp) {
  const BodyA<R>& b = body<R>(i);
  const R mu = tp.get(th(i, kHy));
  const int flags = (int)tp.get(th(i, kHflag));
  const R q = x.get(6 + i), qd = x.get(kQV + 5 + i), uu = u.get(i - 1);
  R ub = R(0);
  if (!(flags & 1)) {
    const R kp = b.kp * par.kps, kv = b.kv * par.kds;
    qb -= mu * kp;
    qdb -= mu * kv;
    ub = mu * kp;
    kpb += mu * b.kp * (uu - q);
    kdb -= mu * b.kv * qd;
  }
  if (flags & 6) {
    qb -= mu * cfg.lkp;
    qdb -= mu * cfg.lkd;
  }
  qdb -= mu * b.damp;
  kdb -= mu * cfg.dt * b.kv * tp.get(th(i, kHqdd));
  ubar.put(i - 1, ub);
}

// Reverse of hinge i (body i -> parent): Psi terms, world pose (legs),
// servo terms; the adjoints in `up` move to the parent's frame.
template <int AX, bool kLeg, class R, class Tp, class X, class UA, class UB>
GA_HD void psi_rev_body(int i, Up<R>& up, const X& x, const UA& u, UB& ubar, const Par<R>& par, const Cfg<R>& cfg,
                        R& kpb, R& kdb, Tp& tp) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const BodyA<R>& b = body<R>(i);
  const R c = tp.get(th(i, kHc)), s = tp.get(th(i, kHs));
  const R qd = x.get(kQV + 5 + i);
  const SV<R> v = get6<R>(tp, tb(i, kBw));
  const SV<R> psi = get6<R>(tp, tb(i, kBpsi));
  R qb = R(0), qdb = R(0);
  // psi_i = X psi_p + S mu'_i
  qb -= dot_scross<AX>(up.P, psi);
  // at_i = X at_p + S qdd + v x (S qd)
  SV<R> Xap = get6<R>(tp, tb(i, kBa)) - sv(zero3<R>(), get3<R>(tp, tb(i, kBg)));
  at(Xap.w, AX) -= tp.get(th(i, kHqdd));
  at(Xap.w, i1) -= qd * cat(v.w, i2);
  at(Xap.w, i2) += qd * cat(v.w, i1);
  at(Xap.l, i1) -= qd * cat(v.l, i2);
  at(Xap.l, i2) += qd * cat(v.l, i1);
  qb -= dot_scross<AX>(up.A, Xap);
  // v x (S qd): vbar += qd (e x Abar), qdbar += Abar . (v x e)
  up.V.w += qd * ecross<AX>(up.A.w);
  up.V.l += qd * ecross<AX>(up.A.l);
  qdb -= dot(up.A.w, ecross<AX>(v.w)) + dot(up.A.l, ecross<AX>(v.l));
  // v_i = X v_p + S qd
  qdb += cat(up.V.w, AX);
  qb -= dot_scross<AX>(up.V, v);
  up.P = frc_out<AX>(b, up.P, c, s);
  up.A = frc_out<AX>(b, up.A, c, s);
  up.V = frc_out<AX>(b, up.V, c, s);
  if constexpr (kLeg) {  // R_i = R_p E, P_i = P_p + R_p p
    for (int a = 0; a < 3; ++a)
      qb += up.Rb.m[3 * a + i1] * up.Rw.m[3 * a + i2] - up.Rb.m[3 * a + i2] * up.Rw.m[3 * a + i1];
    M3<R> E;  // E = T A
    for (int a = 0; a < 3; ++a) {
      const V3<R> row = rotAT<AX>(v3(b.ident ? R(a == 0) : b.T[3 * a], b.ident ? R(a == 1) : b.T[3 * a + 1],
                                     b.ident ? R(a == 2) : b.T[3 * a + 2]),
                                  c, s);
      E.m[3 * a] = row.x;
      E.m[3 * a + 1] = row.y;
      E.m[3 * a + 2] = row.z;
    }
    M3<R> Rb, Rp;  // Rb_p = Rb_i E^T + Pb p^T ;  R_p = R_i E^T
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) {
        Rb.m[3 * r + cc] = up.Rb.m[3 * r] * E.m[3 * cc] + up.Rb.m[3 * r + 1] * E.m[3 * cc + 1] +
                           up.Rb.m[3 * r + 2] * E.m[3 * cc + 2];
        Rp.m[3 * r + cc] = up.Rw.m[3 * r] * E.m[3 * cc] + up.Rw.m[3 * r + 1] * E.m[3 * cc + 1] +
                           up.Rw.m[3 * r + 2] * E.m[3 * cc + 2];
      }
    add_outer(Rb, up.Pb, pvec(b));
    up.Rb = Rb;
    up.Rw = Rp;
  }
  servo_rev(i, x, u, ubar, par, cfg, qb, qdb, kpb, kdb, tp);
  tp.add(th(i, kHqb), qb);
  tp.add(th(i, kHqdb), qdb);
}

// Reverse of the contacts of foot f.  Seeds: Wbar = adjoint of the
// body-frame contact wrench, and the adjoints of the output anchors (read
// from and replaced in lam by the adjoints of the input anchors).
// Produces the adjoints of the foot's body twist (added to up.V) and world
// pose (up.Rb, up.Pb).
template <class R, class Tp, class X, class L>
GA_HD void contacts_rev(int f, const SV<R>& Wbar, Up<R>& up, const X& x, L& lam, const Cfg<R>& cfg, R mu,
                        const Tp& tp) {
  const int ib = f == 0 ? 6 : 12;
  const V3<R> w = get3<R>(tp, tb(ib, kBw)), v = get3<R>(tp, tb(ib, kBv));
  M3<R> Rw;
  for (int k = 0; k < 9; ++k) Rw.m[k] = tp.get(tf(f, kFR + k));
  const V3<R> Pw = get3<R>(tp, tf(f, kFP));
  const ModelA<R>& M = model<R>();
  const int flags = (int)tp.get(tf(f, kFflag));
  // W = (R^T Tq, R^T F): adjoints of Tq, F in the world frame, and of R
  const V3<R> Tqb = mul(Rw, Wbar.w), Fb = mul(Rw, Wbar.l);
  V3<R> Tq = zero3<R>(), F = zero3<R>();
  M3<R> Rb = up.Rb;
  V3<R> Pb = up.Pb, wb = zero3<R>(), vb = zero3<R>();
  for (int j = 0; j < 4; ++j) {
    const int k = 4 * f + j;
    const int fl = (flags >> (4 * j)) & 15;
    R abx = lam.get(kAN + 2 * k), aby = lam.get(kAN + 2 * k + 1);  // adjoint of the output anchor
    R ainx = R(0), ainy = R(0);
    if (fl & kCin) {
      // recompute the sphere's forces along the primal's branches
      const V3<R> r = v3(M.cpos[3 * k], M.cpos[3 * k + 1], M.cpos[3 * k + 2]);
      const V3<R> rw = mul(Rw, r);
      const V3<R> pc = Pw + rw;
      const V3<R> vb_ = v + cross(w, r);
      const V3<R> vp = mul(Rw, vb_);
      const R depth = M.radius - pc.z;
      const R fr = cfg.kn * depth - cfg.dn * vp.z;
      const R fn = fr < R(0) ? R(0) : (fr > R(500) ? R(500) : fr);
      const R ax = (fl & kCfresh) ? pc.x : x.get(kAN + 2 * k), ay = (fl & kCfresh) ? pc.y : x.get(kAN + 2 * k + 1);
      const R t0x = -cfg.kt * (pc.x - ax) - cfg.dtc * vp.x, t0y = -cfg.kt * (pc.y - ay) - cfg.dtc * vp.y;
      const R ftn = sqrt(t0x * t0x + t0y * t0y);
      R ftx = t0x, fty = t0y;
      R scl = R(1);
      if (fl & kCslip) {
        scl = mu * fn / (ftn + R(1e-12));
        ftx *= scl;
        fty *= scl;
      }
      const V3<R> fk = v3(ftx, fty, fn);
      F += fk;
      Tq += cross(rw, fk);
      // adjoint of the sphere force from W: F += f, Tq += rw x f
      V3<R> fb = Fb + cross(Tqb, rw);
      V3<R> rwb = cross(fk, Tqb);
      V3<R> pcb = zero3<R>(), vpb = zero3<R>();
      R fnb = fb.z, t0bx, t0by, abx2 = R(0), aby2 = R(0);  // ab2: adjoint of the anchor a used in d
      if (fl & kCslip) {  // a_out = pc + ft / kt ; ft = t0 * scl
        pcb.x += abx;
        pcb.y += aby;
        const R ftbx = fb.x + abx / cfg.kt, ftby = fb.y + aby / cfg.kt;
        const R den = ftn + R(1e-12);
        const R sb = ftbx * t0x + ftby * t0y;  // adjoint of scl
        fnb += sb * mu / den;
        const R dsn = -mu * fn / (den * den) * (ftn > R(0) ? R(1) / ftn : R(0));  // d scl / d t0 = dsn * t0
        t0bx = scl * ftbx + sb * dsn * t0x;
        t0by = scl * ftby + sb * dsn * t0y;
      } else {  // a_out = a ; ft = t0
        abx2 += abx;
        aby2 += aby;
        t0bx = fb.x;
        t0by = fb.y;
      }
      // t0 = -kt (pc - a) - dtc vp
      pcb.x -= cfg.kt * t0bx;
      pcb.y -= cfg.kt * t0by;
      abx2 += cfg.kt * t0bx;
      aby2 += cfg.kt * t0by;
      vpb.x -= cfg.dtc * t0bx;
      vpb.y -= cfg.dtc * t0by;
      if (fl & kCfresh) {
        pcb.x += abx2;
        pcb.y += aby2;
      } else {
        ainx = abx2;
        ainy = aby2;
      }
      // fn = clamp(kn depth - dn vp.z), depth = radius - pc.z
      if (fl & kClin) {
        pcb.z -= cfg.kn * fnb;
        vpb.z -= cfg.dn * fnb;
      }
      // pc = P + R r ; vp = R (v + w x r) ; rw = R r
      Pb += pcb;
      add_outer(Rb, pcb + rwb, r);
      const V3<R> vbb = mulT(Rw, vpb);
      vb += vbb;
      wb += cross(r, vbb);
      add_outer(Rb, vpb, vb_);
    }
    lam.put(kAN + 2 * k, ainx);
    lam.put(kAN + 2 * k + 1, ainy);
  }
  add_outer(Rb, Tq, Wbar.w);
  add_outer(Rb, F, Wbar.l);
  up.Rb = Rb;
  up.Pb = Pb;
  up.V.w += wb;
  up.V.l += vb;
}

template <bool kLeg, class R, class Tp, class X, class UA, class UB>
GA_HD void psi_rev_chain(int c, Up<R>& up, const X& x, const UA& u, UB& ubar, const Par<R>& par, const Cfg<R>& cfg,
                         R& kpb, R& kdb, Tp& tp) {
  const int first = chain_first(c);
  for (int i = chain_last(c); i >= first; --i) {
    switch (body<R>(i).axis) {
      case 0: psi_rev_body<0, kLeg>(i, up, x, u, ubar, par, cfg, kpb, kdb, tp); break;
      case 1: psi_rev_body<1, kLeg>(i, up, x, u, ubar, par, cfg, kpb, kdb, tp); break;
      default: psi_rev_body<2, kLeg>(i, up, x, u, ubar, par, cfg, kpb, kdb, tp); break;
    }
    if (i > first) psi_own(i - 1, R(0), sv0<R>(), up, tp);
  }
}

template <class R>
GA_HD void up_zero(Up<R>& up) {
  up.P = up.A = up.V = sv0<R>();
  for (int k = 0; k < 9; ++k) up.Rb.m[k] = up.Rw.m[k] = R(0);
  up.Pb = zero3<R>();
}

// Vector-Jacobian product of one substep.  The tape must hold the primal
// of this substep (primal<false> from the same x, u).  lam: on entry the
// adjoint of x' (87 entries), on return the adjoint of x; ubar (29) gets
// the adjoint of the targets; kpb, kdb accumulate the gain-scale adjoints.
template <class R, class Tp, class X, class UA, class L, class UB>
GA_HD void reverse(const Base<R>& st, const X& x, const UA& u, L& lam, UB& ubar, const Par<R>& par,
                   const Cfg<R>& cfg, R& kpb, R& kdb, Tp& tp) {
  const R dt = cfg.dt;
  R qn[4], qnorm;
  M3<R> R0;
  base_frame(st, qn, qnorm, R0);
  const V3<R> w0 = v3(st.wb[0], st.wb[1], st.wb[2]);
  const V3<R> vw = v3(st.vw[0], st.vw[1], st.vw[2]);
  const V3<R> v0 = mulT(R0, vw);
  const SV<R> a0 = get6<R>(tp, tb(0, kBa));
  BaseBar<R> bb;
  for (int k = 0; k < 9; ++k) bb.R0.m[k] = R(0);
  bb.w0 = bb.v0 = zero3<R>();
  // ---- integrator
  bb.pos = v3(lam.get(0), lam.get(1), lam.get(2));
  const V3<R> vw1b = v3(lam.get(kQV), lam.get(kQV + 1), lam.get(kQV + 2)) + dt * bb.pos;
  V3<R> wb1b = v3(lam.get(kQV + 3), lam.get(kQV + 4), lam.get(kQV + 5));
  const V3<R> z = a0.l + cross(w0, v0);
  const V3<R> vw1 = vw + dt * mul(R0, z);
  (void)vw1;
  const V3<R> wb1 = w0 + dt * a0.w;
  {
    const R qb[4] = {lam.get(3), lam.get(4), lam.get(5), lam.get(6)};
    const R wn = sqrt(dot(wb1, wb1));
    if (wn * dt >= R(1e-12)) {
      const R h = R(0.5) * dt, xx = wn * h;
      const R sh = sin(xx), ch = cos(xx);
      const R k = sh / wn;
      const R d[4] = {ch, k * wb1.x, k * wb1.y, k * wb1.z};
      const R* q = st.quat;
      R r[4];
      r[0] = q[0] * d[0] - q[1] * d[1] - q[2] * d[2] - q[3] * d[3];
      r[1] = q[0] * d[1] + q[1] * d[0] + q[2] * d[3] - q[3] * d[2];
      r[2] = q[0] * d[2] - q[1] * d[3] + q[2] * d[0] + q[3] * d[1];
      r[3] = q[0] * d[3] + q[1] * d[2] - q[2] * d[1] + q[3] * d[0];
      const R rn = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
      R o[4];
      for (int j = 0; j < 4; ++j) o[j] = r[j] / rn;
      const R od = o[0] * qb[0] + o[1] * qb[1] + o[2] * qb[2] + o[3] * qb[3];
      R rb[4];
      for (int j = 0; j < 4; ++j) rb[j] = (qb[j] - o[j] * od) / rn;
      bb.quat[0] = rb[0] * d[0] + rb[1] * d[1] + rb[2] * d[2] + rb[3] * d[3];
      bb.quat[1] = -rb[0] * d[1] + rb[1] * d[0] - rb[2] * d[3] + rb[3] * d[2];
      bb.quat[2] = -rb[0] * d[2] + rb[1] * d[3] + rb[2] * d[0] - rb[3] * d[1];
      bb.quat[3] = -rb[0] * d[3] - rb[1] * d[2] + rb[2] * d[1] + rb[3] * d[0];
      R db[4];
      db[0] = rb[0] * q[0] + rb[1] * q[1] + rb[2] * q[2] + rb[3] * q[3];
      db[1] = -rb[0] * q[1] + rb[1] * q[0] + rb[2] * q[3] - rb[3] * q[2];
      db[2] = -rb[0] * q[2] - rb[1] * q[3] + rb[2] * q[0] + rb[3] * q[1];
      db[3] = -rb[0] * q[3] + rb[1] * q[2] - rb[2] * q[1] + rb[3] * q[0];
      // d = (cos(n h), h sinc(n h) w): dd/dw = (-h^2 sinc w^T ; h sinc I + h^3 f w w^T)
      R sinc, fx;
      if (xx < R(0.25)) {
        const R x2 = xx * xx;
        sinc = R(1) - x2 / R(6) + x2 * x2 / R(120) - x2 * x2 * x2 / R(5040);
        fx = -R(1) / R(3) + x2 / R(30) - x2 * x2 / R(840) + x2 * x2 * x2 / R(45360);
      } else {
        sinc = sh / xx;
        fx = (xx * ch - sh) / (xx * xx * xx);
      }
      const V3<R> dv = v3(db[1], db[2], db[3]);
      wb1b += (-h * h * sinc * db[0] + h * h * h * fx * dot(wb1, dv)) * wb1 + (h * sinc) * dv;
    } else {
      for (int j = 0; j < 4; ++j) bb.quat[j] = qb[j];
    }
  }
  bb.wb = wb1b;
  const SV<R> ya = sv(dt * wb1b, dt * mulT(R0, vw1b));  // adjoint of a0
  bb.vw = vw1b;
  bb.w0 += cross(v0, ya.l);
  bb.v0 += cross(ya.l, w0);
  add_outer(bb.R0, dt * vw1b, z);
  for (int i = 1; i <= kNJ; ++i) {
    const R qb = lam.get(6 + i);
    const R qd1b = lam.get(kQV + 5 + i) + dt * qb;
    tp.put(th(i, kHqb), qb);
    tp.put(th(i, kHqdb), qd1b);
    tp.put(th(i, kHy), dt * qd1b);
  }
  // ---- mu = Mt^-1 y
  {
    SV<R> p15 = sv0<R>();
    p15 += mus_bwd_chain<R>(3, tp);
    p15 += mus_bwd_chain<R>(4, tp);
    SV<R> p0 = mus_bwd_chain_from<R>(2, p15, tp);
    p0 += mus_bwd_chain<R>(0, tp);
    p0 += mus_bwd_chain<R>(1, tp);
    const SV<R> m0 = ldl_solve(ya - p0, tp);
    put6(tp, tb(0, kBpsi), sv(-m0.w, -m0.l));
    mus_fwd_chain<R>(2, tp);
    mus_fwd_chain<R>(3, tp);
    mus_fwd_chain<R>(4, tp);
    mus_fwd_chain<R>(0, tp);
    mus_fwd_chain<R>(1, tp);
  }
  // ---- Psi(-mu) reversed, servo terms, contacts, leg world pose
  Up<R> up15;
  up_zero(up15);
  psi_own(15, R(0), sv0<R>(), up15, tp);
  for (int c = 3; c < 5; ++c) {
    Up<R> up;
    up_zero(up);
    psi_own(chain_last(c), R(0), sv0<R>(), up, tp);
    psi_rev_chain<false>(c, up, x, u, ubar, par, cfg, kpb, kdb, tp);
    up15.P += up.P;
    up15.A += up.A;
    up15.V += up.V;
  }
  Up<R> up0;
  up_zero(up0);
  psi_rev_chain<false>(2, up15, x, u, ubar, par, cfg, kpb, kdb, tp);
  up0.P += up15.P;
  up0.A += up15.A;
  up0.V += up15.V;
  for (int f = 0; f < 2; ++f) {
    Up<R> up;
    up_zero(up);
    const int last = chain_last(f);
    const SV<R> Wext = get6<R>(tp, tf(f, kFW));
    psi_own(last, R(0), Wext, up, tp);
    const SV<R> psi = get6<R>(tp, tb(last, kBpsi));
    for (int k = 0; k < 9; ++k) up.Rw.m[k] = tp.get(tf(f, kFR + k));
    contacts_rev(f, sv(-psi.w, -psi.l), up, x, lam, cfg, par.mu, tp);
    psi_rev_chain<true>(f, up, x, u, ubar, par, cfg, kpb, kdb, tp);
    up0.P += up.P;
    up0.A += up.A;
    up0.V += up.V;
    for (int k = 0; k < 9; ++k) bb.R0.m[k] += up.Rb.m[k];
    bb.pos += up.Pb;
  }
  psi_own(0, par.dmass, sv0<R>(), up0, tp);
  // base: at_0 = a0 - (0, g0), g0 = gz R0[2][:] ; v_0 = (wb, R0^T vw)
  for (int k = 0; k < 3; ++k) bb.R0.m[6 + k] -= cfg.gz * cat(up0.A.l, k);
  bb.w0 += up0.V.w;
  bb.v0 += up0.V.l;
  // ---- base twist and rotation to the state
  bb.wb += bb.w0;
  bb.vw += mul(R0, bb.v0);
  add_outer(bb.R0, vw, bb.v0);
  {
    const M3<R>& G = bb.R0;
    const R w = qn[0], xq = qn[1], y = qn[2], zq = qn[3];
    R qnb[4];
    qnb[0] = R(2) * (-zq * G.m[1] + y * G.m[2] + zq * G.m[3] - xq * G.m[5] - y * G.m[6] + xq * G.m[7]);
    qnb[1] = R(2) * (y * G.m[1] + zq * G.m[2] + y * G.m[3] - R(2) * xq * G.m[4] - w * G.m[5] + zq * G.m[6] +
                     w * G.m[7] - R(2) * xq * G.m[8]);
    qnb[2] = R(2) * (-R(2) * y * G.m[0] + xq * G.m[1] + w * G.m[2] + xq * G.m[3] + zq * G.m[5] - w * G.m[6] +
                     zq * G.m[7] - R(2) * y * G.m[8]);
    qnb[3] = R(2) * (-R(2) * zq * G.m[0] - w * G.m[1] + xq * G.m[2] + w * G.m[3] - R(2) * zq * G.m[4] + y * G.m[5] +
                     xq * G.m[6] + y * G.m[7]);
    const R od = qn[0] * qnb[0] + qn[1] * qnb[1] + qn[2] * qnb[2] + qn[3] * qnb[3];
    for (int j = 0; j < 4; ++j) bb.quat[j] += (qnb[j] - qn[j] * od) / qnorm;
  }
  // ---- write the adjoint of x
  for (int k = 0; k < 3; ++k) lam.put(k, cat(bb.pos, k));
  for (int k = 0; k < 4; ++k) lam.put(3 + k, bb.quat[k]);
  for (int k = 0; k < 3; ++k) lam.put(kQV + k, cat(bb.vw, k));
  for (int k = 0; k < 3; ++k) lam.put(kQV + 3 + k, cat(bb.wb, k));
  for (int i = 1; i <= kNJ; ++i) {
    lam.put(6 + i, tp.get(th(i, kHqb)));
    lam.put(kQV + 5 + i, tp.get(th(i, kHqdb)));
  }
}

}  // namespace g1b::adj
