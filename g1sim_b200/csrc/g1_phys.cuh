// g1_phys.cuh -- FP32 G1 step specialised at compile time on the G1 tree.
//
// One environment per thread.  The step is the reference's
//   FK + velocities          (reference src/g1_core.h:29-54)
//   contacts, PD, ABA        (reference src/g1_core.h:109-207)
//   semi-implicit Euler      (reference src/g1_core.h:212-222)
// re-derived for the G1's structure instead of a generic tree walk:
//   * every hinge axis is +x, +y or +z and every joint anchor is the body
//     origin, so S = [e_ax; 0]: U = IA S is a column of IA, S^T f picks one
//     component, the joint rotation mixes two coordinates with (cos, sin);
//   * tree rotations, tree offsets and rigid-body spatial inertias are
//     compile-time constants (no per-step quat_to_mat / spatial_inertia);
//   * the tree is 5 serial chains (left leg 1-6, right leg 7-12, waist 13-15,
//     left arm 16-22, right arm 23-29) hanging off the pelvis (0) and the
//     torso (15), so the backward pass keeps ONE running articulated inertia
//     per chain plus accumulators at the two branch bodies;
//   * articulated inertias are kept as blocks J (sym), H (3x3), M (sym),
//     transformed child->parent by the axis rotation (2-plane mix), the
//     constant tree rotation and the constant offset;
//   * contacts run right after each foot's FK and add a world-frame wrench.
// Per-hinge values that the forward pass needs (cos/sin, velocity-product
// term c, U, u, 1/D) live in a Scratch (shared memory on the device).
//
// The header compiles as host code too (G1_HD) so that the same arithmetic
// can be examined on the CPU; the product only runs it on the device.
#pragma once
#include <math.h>

#include "g1_model_derived.h"

#if defined(__CUDACC__)
#define G1_HD __host__ __device__ __forceinline__
#define G1_CE __host__ __device__ constexpr
#else
#define G1_HD inline
#define G1_CE constexpr
#endif

namespace g1b {

constexpr int kNB = G1M_NB, kNJ = G1M_NB - 1, kNQ = G1M_NQ, kNV = G1M_NV, kNU = G1M_NU;
constexpr int kNC = G1M_NC;
constexpr float kAnchorFree = 1e30f;

// ------------------------------------------------------------ model access
// constexpr accessors: ONLY for constant expressions (if constexpr, constexpr
// locals).  In device code a constexpr function reading these host tables with
// a run-time argument would read host memory; run-time reads go through the
// float mirrors below (tree_rot, spi).
// consteval: a run-time call is a compile error, on the host and the device.
#if defined(__cpp_consteval)
#define G1_CONSTEVAL consteval
#else
#define G1_CONSTEVAL constexpr
#endif
G1_CONSTEVAL int parent_of(int i) { return g1m_parent[i]; }
G1_CONSTEVAL int axis_of(int i) { return g1m_axis_idx[i - 1]; }
G1_CONSTEVAL bool tree_ident(int i) { return g1m_tree_ident[i] != 0; }
G1_CONSTEVAL float tree_pos(int i, int k) { return (float)g1m_tree_pos[3 * i + k]; }
G1_CONSTEVAL float spi_c(int i, int k) { return (float)g1m_sp_inertia[16 * i + k]; }
G1_CE float f_of(double x) { return (float)x; }

// Float copies of the tables that device code indexes at run time (the
// constexpr double tables are only usable in constant expressions there).
template <int N>
struct FTab {
  float v[N];
};
template <int N>
constexpr FTab<N> ftab(const double* src) {
  FTab<N> t{};
#pragma unroll
  for (int i = 0; i < N; ++i) t.v[i] = (float)src[i];
  return t;
}
#if defined(__CUDACC__)
static __constant__ FTab<G1M_NQ> c_stand = ftab<G1M_NQ>(g1m_qpos_stand);
static __constant__ FTab<3 * G1M_NC> c_contact_pos = ftab<3 * G1M_NC>(g1m_contact_pos);
static __constant__ FTab<9 * G1M_NB> c_tree_rot = ftab<9 * G1M_NB>(g1m_tree_rot);
static __constant__ FTab<16 * G1M_NB> c_spi = ftab<16 * G1M_NB>(g1m_sp_inertia);
#endif
// run-time accessors (constant-bank loads on the device)
G1_HD float tree_rot(int i, int r, int c) {
#if defined(__CUDA_ARCH__)
  return c_tree_rot.v[9 * i + 3 * r + c];
#else
  return (float)g1m_tree_rot[9 * i + 3 * r + c];
#endif
}
G1_HD float spi(int i, int k) {
#if defined(__CUDA_ARCH__)
  return c_spi.v[16 * i + k];
#else
  return (float)g1m_sp_inertia[16 * i + k];
#endif
}
G1_HD float stand_at(int i) {
#if defined(__CUDA_ARCH__)
  return c_stand.v[i];
#else
  return (float)g1m_qpos_stand[i];
#endif
}
G1_HD float contact_pos_at(int i) {
#if defined(__CUDA_ARCH__)
  return c_contact_pos.v[i];
#else
  return (float)g1m_contact_pos[i];
#endif
}

// Per-step configuration (mirrors the reference G1Config, src/g1_types.h:33-42).
struct StepConfig {
  float gravity_z, contact_kn, contact_dn, contact_kt, contact_dt, limit_kp, limit_kd, dt;
};

// ----------------------------------------------------------------- algebra
struct V3 {
  float v[3];
};
G1_HD V3 mk3(float x, float y, float z) { return V3{{x, y, z}}; }
G1_HD V3 add(const V3& a, const V3& b) { return mk3(a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2]); }
G1_HD V3 sub(const V3& a, const V3& b) { return mk3(a.v[0] - b.v[0], a.v[1] - b.v[1], a.v[2] - b.v[2]); }
G1_HD V3 scl(float s, const V3& a) { return mk3(s * a.v[0], s * a.v[1], s * a.v[2]); }
G1_HD V3 crs(const V3& a, const V3& b) {
  return mk3(a.v[1] * b.v[2] - a.v[2] * b.v[1], a.v[2] * b.v[0] - a.v[0] * b.v[2],
             a.v[0] * b.v[1] - a.v[1] * b.v[0]);
}
G1_HD float dot(const V3& a, const V3& b) { return a.v[0] * b.v[0] + a.v[1] * b.v[1] + a.v[2] * b.v[2]; }

// 3x3 row-major
struct M3 {
  float m[9];
};
G1_HD V3 mv(const M3& A, const V3& x) {
  return mk3(A.m[0] * x.v[0] + A.m[1] * x.v[1] + A.m[2] * x.v[2],
             A.m[3] * x.v[0] + A.m[4] * x.v[1] + A.m[5] * x.v[2],
             A.m[6] * x.v[0] + A.m[7] * x.v[1] + A.m[8] * x.v[2]);
}
G1_HD V3 mtv(const M3& A, const V3& x) {
  return mk3(A.m[0] * x.v[0] + A.m[3] * x.v[1] + A.m[6] * x.v[2],
             A.m[1] * x.v[0] + A.m[4] * x.v[1] + A.m[7] * x.v[2],
             A.m[2] * x.v[0] + A.m[5] * x.v[1] + A.m[8] * x.v[2]);
}

// Symmetric 3x3: s[0..5] = xx, yy, zz, xy, xz, yz.
struct S3 {
  float s[6];
};
// pure helper called with run-time indices: must be a device function too
G1_CE int sidx(int r, int c) {
  return r == c ? r : ((r == 0 && c == 1) || (r == 1 && c == 0)) ? 3 : ((r == 0 && c == 2) || (r == 2 && c == 0)) ? 4 : 5;
}

// Articulated / rigid spatial inertia [[J, H], [H^T, M]] in [angular; linear] order.
struct AI {
  S3 J;
  M3 H;
  S3 M;
};

struct SV {
  V3 a, l;
};

// ------------------------------------------------- joint axis rotation (A)
// A rotates by q about basis axis AX: it mixes coordinates i=(AX+1)%3 and
// j=(AX+2)%3 as [x_i'; x_j'] = [[c, -s], [s, c]] [x_i; x_j].
template <int AX>
G1_HD V3 rotA(const V3& x, float c, float s) {
  constexpr int i = (AX + 1) % 3, j = (AX + 2) % 3;
  V3 r = x;
  r.v[i] = c * x.v[i] - s * x.v[j];
  r.v[j] = s * x.v[i] + c * x.v[j];
  return r;
}
template <int AX>
G1_HD V3 rotAT(const V3& x, float c, float s) {
  constexpr int i = (AX + 1) % 3, j = (AX + 2) % 3;
  V3 r = x;
  r.v[i] = c * x.v[i] + s * x.v[j];
  r.v[j] = c * x.v[j] - s * x.v[i];
  return r;
}
// A S A^T for symmetric S (rows then columns of the (i, j) plane).
template <int AX>
G1_HD S3 rotA_sym(const S3& S, float c, float s) {
  constexpr int k = AX, i = (AX + 1) % 3, j = (AX + 2) % 3;
  const float sii = S.s[sidx(i, i)], sjj = S.s[sidx(j, j)], sij = S.s[sidx(i, j)];
  const float sik = S.s[sidx(i, k)], sjk = S.s[sidx(j, k)];
  // B = A S, rows i and j
  const float bii = c * sii - s * sij, bij = c * sij - s * sjj;
  const float bji = s * sii + c * sij, bjj = s * sij + c * sjj;
  S3 r;
  r.s[sidx(k, k)] = S.s[sidx(k, k)];
  r.s[sidx(i, k)] = c * sik - s * sjk;
  r.s[sidx(j, k)] = s * sik + c * sjk;
  r.s[sidx(i, i)] = c * bii - s * bij;
  r.s[sidx(j, j)] = s * bji + c * bjj;
  r.s[sidx(i, j)] = s * bii + c * bij;
  return r;
}
// A H A^T for general H.
template <int AX>
G1_HD M3 rotA_gen(const M3& H, float c, float s) {
  constexpr int i = (AX + 1) % 3, j = (AX + 2) % 3;
  M3 B = H;  // B = A H: rows
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    B.m[3 * i + col] = c * H.m[3 * i + col] - s * H.m[3 * j + col];
    B.m[3 * j + col] = s * H.m[3 * i + col] + c * H.m[3 * j + col];
  }
  M3 r = B;  // r = B A^T: columns
#pragma unroll
  for (int row = 0; row < 3; ++row) {
    r.m[3 * row + i] = c * B.m[3 * row + i] - s * B.m[3 * row + j];
    r.m[3 * row + j] = s * B.m[3 * row + i] + c * B.m[3 * row + j];
  }
  return r;
}

// ------------------------------------------- constant tree rotation (T)
template <int I>
G1_HD V3 rotT(const V3& x) {
  if constexpr (tree_ident(I)) {
    return x;
  } else {
    V3 r;
#pragma unroll
    for (int a = 0; a < 3; ++a)
      r.v[a] = tree_rot(I, a, 0) * x.v[0] + tree_rot(I, a, 1) * x.v[1] + tree_rot(I, a, 2) * x.v[2];
    return r;
  }
}
template <int I>
G1_HD V3 rotTT(const V3& x) {
  if constexpr (tree_ident(I)) {
    return x;
  } else {
    V3 r;
#pragma unroll
    for (int a = 0; a < 3; ++a)
      r.v[a] = tree_rot(I, 0, a) * x.v[0] + tree_rot(I, 1, a) * x.v[1] + tree_rot(I, 2, a) * x.v[2];
    return r;
  }
}
template <int I>
G1_HD S3 rotT_sym(const S3& S) {
  if constexpr (tree_ident(I)) {
    return S;
  } else {
    float F[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        F[3 * a + b] = S.s[sidx(a, b)];
    float B[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        B[3 * a + b] = tree_rot(I, a, 0) * F[b] + tree_rot(I, a, 1) * F[3 + b] + tree_rot(I, a, 2) * F[6 + b];
    S3 r;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b)
        r.s[sidx(a, b)] = B[3 * a + 0] * tree_rot(I, b, 0) + B[3 * a + 1] * tree_rot(I, b, 1) +
                          B[3 * a + 2] * tree_rot(I, b, 2);
    return r;
  }
}
template <int I>
G1_HD M3 rotT_gen(const M3& H) {
  if constexpr (tree_ident(I)) {
    return H;
  } else {
    float B[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        B[3 * a + b] = tree_rot(I, a, 0) * H.m[b] + tree_rot(I, a, 1) * H.m[3 + b] + tree_rot(I, a, 2) * H.m[6 + b];
    M3 r;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        r.m[3 * a + b] = B[3 * a + 0] * tree_rot(I, b, 0) + B[3 * a + 1] * tree_rot(I, b, 1) +
                         B[3 * a + 2] * tree_rot(I, b, 2);
    return r;
  }
}

// ----------------------------------------- constant offset p (tree_pos)
// p x v, term by term so that the zero components of p drop out.
template <int I, int R>
G1_HD float pcross_c(const V3& x) {
  constexpr int a = (R + 1) % 3, b = (R + 2) % 3;
  constexpr float pa = tree_pos(I, a), pb = tree_pos(I, b);
  if constexpr (pa != 0.0f && pb != 0.0f) return pa * x.v[b] - pb * x.v[a];
  else if constexpr (pa != 0.0f) return pa * x.v[b];
  else if constexpr (pb != 0.0f) return -(pb * x.v[a]);
  else return 0.0f;
}
template <int I>
G1_HD V3 pcross(const V3& x) {
  return mk3(pcross_c<I, 0>(x), pcross_c<I, 1>(x), pcross_c<I, 2>(x));
}
template <int I>
G1_CONSTEVAL bool p_zero() {
  return tree_pos(I, 0) == 0.0f && tree_pos(I, 1) == 0.0f && tree_pos(I, 2) == 0.0f;
}

// --------------------------------------------------- rigid-body inertias
template <int I>
G1_HD AI body_inertia() {
  AI r;
#pragma unroll
  for (int k = 0; k < 6; ++k) r.J.s[k] = spi(I, k);
#pragma unroll
  for (int k = 0; k < 9; ++k) r.H.m[k] = spi(I, 6 + k);
  const float m = spi(I, 15);
  r.M.s[0] = r.M.s[1] = r.M.s[2] = m;
  r.M.s[3] = r.M.s[4] = r.M.s[5] = 0.0f;
  return r;
}

// Pelvis inertia with a per-env mass offset (COM and rotational inertia
// about the COM unchanged): J = Icom + m [c]x [c]x^T, H = m [c]x, M = m 1.
G1_HD AI pelvis_inertia(float dmass) {
  constexpr float m0 = spi_c(0, 15);
  constexpr float cx = (float)g1m_com[0], cy = (float)g1m_com[1], cz = (float)g1m_com[2];
  const float m = m0 + dmass;
  AI r;
  // Icom part of J = J0 - m0 [c]x[c]x^T, done in double at compile time
  constexpr float icxx = (float)(g1m_inertia_com[0]), icyy = (float)(g1m_inertia_com[4]);
  constexpr float iczz = (float)(g1m_inertia_com[8]), icxy = (float)(g1m_inertia_com[1]);
  constexpr float icxz = (float)(g1m_inertia_com[2]), icyz = (float)(g1m_inertia_com[5]);
  // [c]x [c]x^T = (c.c) 1 - c c^T
  r.J.s[0] = icxx + m * (cy * cy + cz * cz);
  r.J.s[1] = icyy + m * (cx * cx + cz * cz);
  r.J.s[2] = iczz + m * (cx * cx + cy * cy);
  r.J.s[3] = icxy - m * (cx * cy);
  r.J.s[4] = icxz - m * (cx * cz);
  r.J.s[5] = icyz - m * (cy * cz);
  r.H.m[0] = 0.0f;     r.H.m[1] = -m * cz; r.H.m[2] = m * cy;
  r.H.m[3] = m * cz;   r.H.m[4] = 0.0f;    r.H.m[5] = -m * cx;
  r.H.m[6] = -m * cy;  r.H.m[7] = m * cx;  r.H.m[8] = 0.0f;
  r.M.s[0] = r.M.s[1] = r.M.s[2] = m;
  r.M.s[3] = r.M.s[4] = r.M.s[5] = 0.0f;
  return r;
}

// I v for a spatial inertia
G1_HD SV ai_mul(const AI& I, const SV& x) {
  SV r;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    r.a.v[a] = I.J.s[sidx(a, 0)] * x.a.v[0] + I.J.s[sidx(a, 1)] * x.a.v[1] + I.J.s[sidx(a, 2)] * x.a.v[2] +
               I.H.m[3 * a + 0] * x.l.v[0] + I.H.m[3 * a + 1] * x.l.v[1] + I.H.m[3 * a + 2] * x.l.v[2];
    r.l.v[a] = I.H.m[a] * x.a.v[0] + I.H.m[3 + a] * x.a.v[1] + I.H.m[6 + a] * x.a.v[2] +
               I.M.s[sidx(a, 0)] * x.l.v[0] + I.M.s[sidx(a, 1)] * x.l.v[1] + I.M.s[sidx(a, 2)] * x.l.v[2];
  }
  return r;
}

// Rigid-body bias force with gravity (reference src/g1_core.h:113-120):
//   pA = v x* (I v) - [c x (m g_b); m g_b],  [c x (m g); m g] = [H g; m g].
template <int I>
G1_HD SV bias_force(const AI& In, const V3& w, const V3& v, const V3& g) {
  SV x{w, v};
  SV h = ai_mul(In, x);
  const float m = In.M.s[0];
  SV r;
  V3 hg = mk3(In.H.m[0] * g.v[0] + In.H.m[1] * g.v[1] + In.H.m[2] * g.v[2],
              In.H.m[3] * g.v[0] + In.H.m[4] * g.v[1] + In.H.m[5] * g.v[2],
              In.H.m[6] * g.v[0] + In.H.m[7] * g.v[1] + In.H.m[8] * g.v[2]);
  r.a = sub(add(crs(w, h.a), crs(v, h.l)), hg);
  r.l = sub(crs(w, h.l), scl(m, g));
  return r;
}

// ---------------------------------------------------------------- scratch
// Per-hinge slots: 0-1 cos/sin, 2-5 velocity-product term c (4 non-zeros),
// 6-11 bias force pA (FK -> backward) then U (backward -> forward),
// 12 u, 13 1/D.  Slots 406-411: pelvis bias force.
constexpr int kSlotsPerHinge = 14;
constexpr int kSlotPelvis = kNJ * kSlotsPerHinge;
constexpr int kNumSlots = kSlotPelvis + 6;
template <int I, int K>
G1_CONSTEVAL int slot() { return (I - 1) * kSlotsPerHinge + K; }

// ----------------------------------------------------------- env data
struct EnvState {
  float pos[3], quat[4], q[kNJ];
  float vw[3], wb[3], qd[kNJ];
};
// One env's arrays that stay in memory during a step (SoA, element i of the
// env at p[i * stride]): PD targets read once per hinge, contact anchors read
// and written by the contacts, last-substep outputs (nullable).
struct EnvIO {
  const float* ctrl;
  float* anchor;
  float* foot_pos;
  float* foot_vel;
  float* cf;
  size_t stride;
};
struct EnvParams {
  float mu, dmass, kp_scale, kd_scale;
};

// Running FK values of one body: body-frame twist, gravity, world pose (legs only).
struct FKNode {
  V3 w, v, g;
  M3 R;
  V3 P;
};

// ------------------------------------------------------------- FK pass
// reference src/g1_core.h:29-54 (+ bias init :113-120 and c of :180)
template <int I, bool kWorld, class Scr>
G1_HD void fk_body(FKNode& n, const EnvState& st, Scr& scr) {
  constexpr int AX = axis_of(I);
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const float q = st.q[I - 1], qd = st.qd[I - 1];
  float s, c;
  sincosf(q, &s, &c);
  scr.template put<slot<I, 0>()>(c);
  scr.template put<slot<I, 1>()>(s);
  // parent -> child: x_c = A^T T^T x_p ;  v.l uses v_p - p x w_p
  V3 t = n.v;
  if constexpr (!p_zero<I>()) t = sub(n.v, pcross<I>(n.w));
  V3 w = rotAT<AX>(rotTT<I>(n.w), c, s);
  V3 v = rotAT<AX>(rotTT<I>(t), c, s);
  V3 g = rotAT<AX>(rotTT<I>(n.g), c, s);
  w.v[AX] += qd;
  if constexpr (kWorld) {
    // R_i = R_p T A ; P_i = P_p + R_p p
    M3 RT;
    if constexpr (tree_ident(I)) {
      RT = n.R;
    } else {
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
          RT.m[3 * a + b] = n.R.m[3 * a + 0] * tree_rot(I, 0, b) + n.R.m[3 * a + 1] * tree_rot(I, 1, b) +
                            n.R.m[3 * a + 2] * tree_rot(I, 2, b);
    }
    M3 R = RT;  // columns i1, i2 mixed: R = RT A
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      R.m[3 * a + i1] = c * RT.m[3 * a + i1] + s * RT.m[3 * a + i2];
      R.m[3 * a + i2] = c * RT.m[3 * a + i2] - s * RT.m[3 * a + i1];
    }
    constexpr float p0 = tree_pos(I, 0), p1 = tree_pos(I, 1), p2 = tree_pos(I, 2);
    V3 pw = mk3(0.f, 0.f, 0.f);
#pragma unroll
    for (int a = 0; a < 3; ++a) pw.v[a] = n.R.m[3 * a + 0] * p0 + n.R.m[3 * a + 1] * p1 + n.R.m[3 * a + 2] * p2;
    n.P = add(n.P, pw);
    n.R = R;
  }
  n.w = w;
  n.v = v;
  n.g = g;
  // velocity-product term c = v x_m (qd S) = [qd (w x e_ax); qd (v x e_ax)]
  scr.template put<slot<I, 2>()>(qd * w.v[i2]);
  scr.template put<slot<I, 3>()>(-(qd * w.v[i1]));
  scr.template put<slot<I, 4>()>(qd * v.v[i2]);
  scr.template put<slot<I, 5>()>(-(qd * v.v[i1]));
}

template <int I, class Scr>
G1_HD void store_bias(const SV& pA, Scr& scr) {
  scr.template put<slot<I, 6>()>(pA.a.v[0]);
  scr.template put<slot<I, 7>()>(pA.a.v[1]);
  scr.template put<slot<I, 8>()>(pA.a.v[2]);
  scr.template put<slot<I, 9>()>(pA.l.v[0]);
  scr.template put<slot<I, 10>()>(pA.l.v[1]);
  scr.template put<slot<I, 11>()>(pA.l.v[2]);
}
template <int I, class Scr>
G1_HD SV load_bias(Scr& scr) {
  SV r;
  if constexpr (I == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) r.a.v[k] = scr.get(kSlotPelvis + k);
#pragma unroll
    for (int k = 0; k < 3; ++k) r.l.v[k] = scr.get(kSlotPelvis + 3 + k);
  } else {
    r.a = mk3(scr.template get<slot<I, 6>()>(), scr.template get<slot<I, 7>()>(), scr.template get<slot<I, 8>()>());
    r.l = mk3(scr.template get<slot<I, 9>()>(), scr.template get<slot<I, 10>()>(), scr.template get<slot<I, 11>()>());
  }
  return r;
}

// FK of a serial chain FIRST..LAST (each body's parent is the previous one,
// the first body's parent is the node passed in); stores biases.
template <int I, int LAST, bool kWorld, class Scr>
G1_HD void fk_chain(FKNode& n, const EnvState& st, Scr& scr) {
  fk_body<I, kWorld>(n, st, scr);
  if constexpr (I != 0) store_bias<I>(bias_force<I>(body_inertia<I>(), n.w, n.v, n.g), scr);
  if constexpr (I < LAST) fk_chain<I + 1, LAST, kWorld>(n, st, scr);
}

// --------------------------------------------------------------- contacts
// Eight spheres, four on each foot (reference src/g1_core.h:123-153).  The
// world wrench about the foot origin is accumulated and rotated to the body
// frame once.
template <int K0>
G1_HD void foot_contacts(const FKNode& n, const EnvIO& io, bool last, const StepConfig& cfg, float mu,
                         SV& pA_foot) {
  float* anchor = io.anchor;
  const size_t sd = io.stride;
  const V3 ww = mv(n.R, n.w);  // world angular velocity
  const V3 vo = mv(n.R, n.v);  // world velocity of the foot origin
  V3 F = mk3(0.f, 0.f, 0.f), Tq = mk3(0.f, 0.f, 0.f);
  constexpr float radius = (float)g1m_contact_radius;
  const float inv_kt = 1.0f / cfg.contact_kt;
#pragma unroll
  for (int k = K0; k < K0 + 4; ++k) {
    const V3 r = mk3(contact_pos_at(3 * k), contact_pos_at(3 * k + 1), contact_pos_at(3 * k + 2));
    const V3 rw = mv(n.R, r);
    const float px = n.P.v[0] + rw.v[0], py = n.P.v[1] + rw.v[1], pz = n.P.v[2] + rw.v[2];
    const float depth = radius - pz;
    const bool in = depth > 0.0f;
    const V3 vp = add(vo, crs(ww, rw));
    float fn = cfg.contact_kn * depth - cfg.contact_dn * vp.v[2];
    fn = fminf(fmaxf(fn, 0.0f), 500.0f);
    float ax = anchor[(2 * k) * sd], ay = anchor[(2 * k + 1) * sd];
    const bool fresh = ax >= kAnchorFree;
    ax = fresh ? px : ax;
    ay = fresh ? py : ay;
    float ftx = -cfg.contact_kt * (px - ax) - cfg.contact_dt * vp.v[0];
    float fty = -cfg.contact_kt * (py - ay) - cfg.contact_dt * vp.v[1];
    const float ftn = sqrtf(ftx * ftx + fty * fty), fmax = mu * fn;
    if (ftn > fmax) {
      const float sc = fmax / (ftn + 1e-12f);
      ftx *= sc;
      fty *= sc;
      ax = px + ftx * inv_kt;
      ay = py + fty * inv_kt;
    }
    if (in) {
      anchor[(2 * k) * sd] = ax;
      anchor[(2 * k + 1) * sd] = ay;
      const V3 f = mk3(ftx, fty, fn);
      F = add(F, f);
      Tq = add(Tq, crs(rw, f));
    } else {
      fn = 0.0f;
      anchor[(2 * k) * sd] = kAnchorFree;
      anchor[(2 * k + 1) * sd] = kAnchorFree;
    }
    if (last && io.cf) io.cf[k * sd] = fn;
  }
  pA_foot.a = sub(pA_foot.a, mtv(n.R, Tq));
  pA_foot.l = sub(pA_foot.l, mtv(n.R, F));
}

// --------------------------------------------------------- backward pass
// Transform child articulated inertia Ia (child frame) into the parent frame
// and add it: X* Ia X^-1 with X = (R = T A, p).  Blocks after rotation
// (J2, H2, M2) and then the offset P = [p]x:
//   H' = H2 + P M2 ;  J' = J2 + P H2^T - H' P ;  M' = M2.
template <int I>
G1_HD void ai_to_parent_add(AI& acc, const AI& Ia, float c, float s) {
  constexpr int AX = axis_of(I);
  S3 J = rotT_sym<I>(rotA_sym<AX>(Ia.J, c, s));
  M3 H = rotT_gen<I>(rotA_gen<AX>(Ia.H, c, s));
  S3 M = rotT_sym<I>(rotA_sym<AX>(Ia.M, c, s));
  if constexpr (!p_zero<I>()) {
    float Mf[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) Mf[3 * a + b] = M.s[sidx(a, b)];
    // H' = H + P M : (P M)[r][col] = (p x M[:,col])_r
    M3 Hn = H;
#pragma unroll
    for (int col = 0; col < 3; ++col) {
      V3 mc = mk3(Mf[col], Mf[3 + col], Mf[6 + col]);
      V3 pm = pcross<I>(mc);
#pragma unroll
      for (int r = 0; r < 3; ++r) Hn.m[3 * r + col] = H.m[3 * r + col] + pm.v[r];
    }
    // J' = J + P H^T - H' P ; (P H^T)[r][c] = (p x H[c,:]^T)_r ; (H' P)[r][c] = -(p x H'[r,:]^T)_c
    V3 pHT[3], HnP[3];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) pHT[cc] = pcross<I>(mk3(H.m[3 * cc], H.m[3 * cc + 1], H.m[3 * cc + 2]));
#pragma unroll
    for (int r = 0; r < 3; ++r) HnP[r] = pcross<I>(mk3(Hn.m[3 * r], Hn.m[3 * r + 1], Hn.m[3 * r + 2]));
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int cc = r; cc < 3; ++cc) {
        // (P H^T)[r][cc] = pHT[cc].v[r] ; (H' P)[r][cc] = -HnP[r].v[cc]
        acc.J.s[sidx(r, cc)] += J.s[sidx(r, cc)] + pHT[cc].v[r] + HnP[r].v[cc];
      }
#pragma unroll
    for (int k = 0; k < 9; ++k) acc.H.m[k] += Hn.m[k];
  } else {
#pragma unroll
    for (int k = 0; k < 6; ++k) acc.J.s[k] += J.s[k];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc.H.m[k] += H.m[k];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) acc.M.s[k] += M.s[k];
}

// force child -> parent: [R f.a + p x (R f.l); R f.l]
template <int I>
G1_HD SV f_to_parent(const SV& f, float c, float s) {
  constexpr int AX = axis_of(I);
  SV r;
  r.l = rotT<I>(rotA<AX>(f.l, c, s));
  r.a = rotT<I>(rotA<AX>(f.a, c, s));
  if constexpr (!p_zero<I>()) r.a = add(r.a, pcross<I>(r.l));
  return r;
}

// One hinge of the backward pass with PD servo, soft limits and implicit
// damping (reference src/g1_core.h:156-186).  IA, pA are body I's
// articulated inertia and bias; adds the projected values into (accI, accP).
template <int I, class Scr>
G1_HD void bwd_body(const AI& IA, const SV& pA, AI& accI, SV& accP, const EnvState& st,
                    const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr) {
  constexpr int h = I - 1, AX = axis_of(I);
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const float c = scr.template get<slot<I, 0>()>(), s = scr.template get<slot<I, 1>()>();
  // U = IA S: column AX of J, row AX of H
  SV U;
#pragma unroll
  for (int a = 0; a < 3; ++a) U.a.v[a] = IA.J.s[sidx(a, AX)];
#pragma unroll
  for (int a = 0; a < 3; ++a) U.l.v[a] = IA.H.m[3 * AX + a];
  const float q = st.q[h], qd = st.qd[h];
  constexpr float kp0 = f_of(g1m_act_kp[h]), kv0 = f_of(g1m_act_kv[h]);
  constexpr float lim = f_of(g1m_act_frclim[h]);
  constexpr float lo = f_of(g1m_jnt_range[2 * h]), hi = f_of(g1m_jnt_range[2 * h + 1]);
  constexpr float arm = f_of(g1m_armature[h]), damp = f_of(g1m_damping[h]);
  const float kp = kp0 * ep.kp_scale, kv = kv0 * ep.kd_scale;
  float t = kp * (io.ctrl[h * io.stride] - q) - kv * qd;
  t = fminf(fmaxf(t, -lim), lim);
  float b = kv + damp;
  if (q < lo) {
    t += cfg.limit_kp * (lo - q) - cfg.limit_kd * qd;
    b += cfg.limit_kd;
  }
  if (q > hi) {
    t += cfg.limit_kp * (hi - q) - cfg.limit_kd * qd;
    b += cfg.limit_kd;
  }
  const float D = U.a.v[AX] + arm + cfg.dt * b;
  float u = t - pA.a.v[AX];
  if constexpr (damp != 0.0f) u -= damp * qd;
  const float invD = 1.0f / D;
  // c (velocity-product term): angular comps i1, i2 and linear comps i1, i2
  SV cv;
  cv.a.v[AX] = 0.0f;
  cv.a.v[i1] = scr.template get<slot<I, 2>()>();
  cv.a.v[i2] = scr.template get<slot<I, 3>()>();
  cv.l.v[AX] = 0.0f;
  cv.l.v[i1] = scr.template get<slot<I, 4>()>();
  cv.l.v[i2] = scr.template get<slot<I, 5>()>();
  // Ia = IA - U U^T / D
  SV W;
  W.a = scl(invD, U.a);
  W.l = scl(invD, U.l);
  AI Ia;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int bb = a; bb < 3; ++bb) {
      Ia.J.s[sidx(a, bb)] = IA.J.s[sidx(a, bb)] - U.a.v[a] * W.a.v[bb];
      Ia.M.s[sidx(a, bb)] = IA.M.s[sidx(a, bb)] - U.l.v[a] * W.l.v[bb];
    }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) Ia.H.m[3 * a + bb] = IA.H.m[3 * a + bb] - U.a.v[a] * W.l.v[bb];
  // pa = pA + Ia c + (u / D) U   (c has zero AX components)
  SV pa;
  const float uD = u * invD;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    pa.a.v[a] = pA.a.v[a] + Ia.J.s[sidx(a, i1)] * cv.a.v[i1] + Ia.J.s[sidx(a, i2)] * cv.a.v[i2] +
                Ia.H.m[3 * a + i1] * cv.l.v[i1] + Ia.H.m[3 * a + i2] * cv.l.v[i2] + uD * U.a.v[a];
    pa.l.v[a] = pA.l.v[a] + Ia.H.m[3 * i1 + a] * cv.a.v[i1] + Ia.H.m[3 * i2 + a] * cv.a.v[i2] +
                Ia.M.s[sidx(a, i1)] * cv.l.v[i1] + Ia.M.s[sidx(a, i2)] * cv.l.v[i2] + uD * U.l.v[a];
  }
  // keep U, u, 1/D for the forward pass (in the bias slots)
  scr.template put<slot<I, 6>()>(U.a.v[0]);
  scr.template put<slot<I, 7>()>(U.a.v[1]);
  scr.template put<slot<I, 8>()>(U.a.v[2]);
  scr.template put<slot<I, 9>()>(U.l.v[0]);
  scr.template put<slot<I, 10>()>(U.l.v[1]);
  scr.template put<slot<I, 11>()>(U.l.v[2]);
  scr.template put<slot<I, 12>()>(u);
  scr.template put<slot<I, 13>()>(invD);
  ai_to_parent_add<I>(accI, Ia, c, s);
  const SV fp = f_to_parent<I>(pa, c, s);
  accP.a = add(accP.a, fp.a);
  accP.l = add(accP.l, fp.l);
}

// Backward pass over the serial chain FIRST..LAST (LAST -> FIRST); the
// chain's first body adds into (accI, accP) of its parent.
template <int FIRST, int I, class Scr>
G1_HD void bwd_chain(AI& IA, SV& pA, AI& accI, SV& accP, const EnvState& st, const EnvIO& io,
                     const EnvParams& ep, const StepConfig& cfg, Scr& scr) {
  if constexpr (I == FIRST) {
    bwd_body<I>(IA, pA, accI, accP, st, io, ep, cfg, scr);
  } else {
    AI IAp = body_inertia<I - 1>();
    SV pAp = load_bias<I - 1>(scr);
    bwd_body<I>(IA, pA, IAp, pAp, st, io, ep, cfg, scr);
    bwd_chain<FIRST, I - 1>(IAp, pAp, accI, accP, st, io, ep, cfg, scr);
  }
}

template <int FIRST, int LAST, class Scr>
G1_HD void bwd_chain_from_leaf(AI& accI, SV& accP, const EnvState& st, const EnvIO& io,
                               const EnvParams& ep, const StepConfig& cfg, Scr& scr) {
  AI IA = body_inertia<LAST>();
  SV pA = load_bias<LAST>(scr);
  bwd_chain<FIRST, LAST>(IA, pA, accI, accP, st, io, ep, cfg, scr);
}

// ---------------------------------------------------------- base solve
// IA0 a0 = -pA0, 6x6 SPD, LDL^T in [angular; linear] order (the reference
// uses a packed Cholesky, src/spatial.h:254-278; same system).
G1_HD SV base_solve(const AI& A, const SV& pA) {
  float m[6][6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      m[a][b] = A.J.s[sidx(a, b)];
      m[3 + a][3 + b] = A.M.s[sidx(a, b)];
      m[a][3 + b] = A.H.m[3 * a + b];
      m[3 + b][a] = A.H.m[3 * a + b];
    }
  float L[6][6], d[6], id[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    float dj = m[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) dj -= L[j][k] * L[j][k] * d[k];
    d[j] = dj;
    id[j] = 1.0f / dj;
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
      float x = m[i][j];
#pragma unroll
      for (int k = 0; k < j; ++k) x -= L[i][k] * L[j][k] * d[k];
      L[i][j] = x * id[j];
    }
  }
  float y[6] = {-pA.a.v[0], -pA.a.v[1], -pA.a.v[2], -pA.l.v[0], -pA.l.v[1], -pA.l.v[2]};
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int k = 0; k < i; ++k) y[i] -= L[i][k] * y[k];
#pragma unroll
  for (int i = 0; i < 6; ++i) y[i] *= id[i];
#pragma unroll
  for (int i = 5; i >= 0; --i)
#pragma unroll
    for (int k = i + 1; k < 6; ++k) y[i] -= L[k][i] * y[k];
  SV r;
  r.a = mk3(y[0], y[1], y[2]);
  r.l = mk3(y[3], y[4], y[5]);
  return r;
}

// --------------------------------------------------------- forward pass
// a_i = X^-1 a_p + c_i ; qdd = (u - U.a_i) / D ; a_i += qdd S  (reference
// src/g1_core.h:190-201), fused with the hinge's semi-implicit Euler update.
template <int I, class Scr>
G1_HD void fwd_body(SV& a, EnvState& st, float dt, Scr& scr) {
  constexpr int h = I - 1, AX = axis_of(I);
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const float c = scr.template get<slot<I, 0>()>(), s = scr.template get<slot<I, 1>()>();
  V3 t = a.l;
  if constexpr (!p_zero<I>()) t = sub(a.l, pcross<I>(a.a));
  SV an;
  an.a = rotAT<AX>(rotTT<I>(a.a), c, s);
  an.l = rotAT<AX>(rotTT<I>(t), c, s);
  an.a.v[i1] += scr.template get<slot<I, 2>()>();
  an.a.v[i2] += scr.template get<slot<I, 3>()>();
  an.l.v[i1] += scr.template get<slot<I, 4>()>();
  an.l.v[i2] += scr.template get<slot<I, 5>()>();
  const float Ua0 = scr.template get<slot<I, 6>()>(), Ua1 = scr.template get<slot<I, 7>()>();
  const float Ua2 = scr.template get<slot<I, 8>()>(), Ul0 = scr.template get<slot<I, 9>()>();
  const float Ul1 = scr.template get<slot<I, 10>()>(), Ul2 = scr.template get<slot<I, 11>()>();
  const float u = scr.template get<slot<I, 12>()>(), invD = scr.template get<slot<I, 13>()>();
  const float Ua = Ua0 * an.a.v[0] + Ua1 * an.a.v[1] + Ua2 * an.a.v[2] + Ul0 * an.l.v[0] +
                   Ul1 * an.l.v[1] + Ul2 * an.l.v[2];
  const float qdd = (u - Ua) * invD;
  an.a.v[AX] += qdd;
  a = an;
  // semi-implicit Euler (reference src/g1_core.h:214,221)
  st.qd[h] += dt * qdd;
  st.q[h] += dt * st.qd[h];
}

template <int I, int LAST, class Scr>
G1_HD void fwd_chain(SV a, EnvState& st, float dt, Scr& scr) {
  fwd_body<I>(a, st, dt, scr);
  if constexpr (I < LAST) fwd_chain<I + 1, LAST>(a, st, dt, scr);
}

// ----------------------------------------------------------- quaternions
G1_HD void quat_to_rot(const float* q, M3& R) {
  const float w = q[0], x = q[1], y = q[2], z = q[3];
  R.m[0] = 1.f - 2.f * (y * y + z * z); R.m[1] = 2.f * (x * y - w * z);       R.m[2] = 2.f * (x * z + w * y);
  R.m[3] = 2.f * (x * y + w * z);       R.m[4] = 1.f - 2.f * (x * x + z * z); R.m[5] = 2.f * (y * z - w * x);
  R.m[6] = 2.f * (x * z - w * y);       R.m[7] = 2.f * (y * z + w * x);       R.m[8] = 1.f - 2.f * (x * x + y * y);
}
G1_HD void quat_normalized(const float* q, float* r) {
  const float n = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const float inv = 1.0f / n;
#pragma unroll
  for (int k = 0; k < 4; ++k) r[k] = q[k] * inv;
}

// ----------------------------------------------------------------- step
// Base frame quantities from the state: rotation, body twist, body gravity.
G1_HD void base_node(const EnvState& st, const StepConfig& cfg, FKNode& base) {
  float qn[4];
  quat_normalized(st.quat, qn);
  quat_to_rot(qn, base.R);
  base.P = mk3(st.pos[0], st.pos[1], st.pos[2]);
  base.w = mk3(st.wb[0], st.wb[1], st.wb[2]);
  base.v = mtv(base.R, mk3(st.vw[0], st.vw[1], st.vw[2]));
  base.g = mk3(base.R.m[6] * cfg.gravity_z, base.R.m[7] * cfg.gravity_z, base.R.m[8] * cfg.gravity_z);
}

template <int FOOT_BODY, int K0>
G1_HD void foot_outputs(const FKNode& n, const EnvIO& io, bool last) {
  if (!last) return;
  constexpr int o = K0 == 0 ? 0 : 3;
  if (io.foot_pos)
#pragma unroll
    for (int k = 0; k < 3; ++k) io.foot_pos[(o + k) * io.stride] = n.P.v[k];
  if (io.foot_vel) {
    const V3 fv = mv(n.R, n.v);
#pragma unroll
    for (int k = 0; k < 3; ++k) io.foot_vel[(o + k) * io.stride] = fv.v[k];
  }
}

// One substep: FK -> contacts -> PD + ABA -> integrate (reference
// src/g1_core.h:225-232).  With last set, the foot kinematics of this
// substep's FK (before integration) and the contact normal forces are
// written to io's outputs.
template <class Scr>
G1_HD void step(EnvState& st, const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr,
                bool last) {
  // ---- FK + bias forces + contacts, chain by chain
  {
    FKNode base;
    base_node(st, cfg, base);
    {
      const SV pA0 = bias_force<0>(pelvis_inertia(ep.dmass), base.w, base.v, base.g);
#pragma unroll
      for (int k = 0; k < 3; ++k) scr.put(kSlotPelvis + k, pA0.a.v[k]);
#pragma unroll
      for (int k = 0; k < 3; ++k) scr.put(kSlotPelvis + 3 + k, pA0.l.v[k]);
    }
    {
      FKNode n = base;
      fk_chain<1, 6, true>(n, st, scr);
      SV pA6 = load_bias<6>(scr);
      foot_contacts<0>(n, io, last, cfg, ep.mu, pA6);
      store_bias<6>(pA6, scr);
      foot_outputs<6, 0>(n, io, last);
    }
    {
      FKNode n = base;
      fk_chain<7, 12, true>(n, st, scr);
      SV pA12 = load_bias<12>(scr);
      foot_contacts<4>(n, io, last, cfg, ep.mu, pA12);
      store_bias<12>(pA12, scr);
      foot_outputs<12, 4>(n, io, last);
    }
    FKNode torso = base;
    fk_chain<13, 15, false>(torso, st, scr);
    {
      FKNode n = torso;
      fk_chain<16, 22, false>(n, st, scr);
    }
    {
      FKNode n = torso;
      fk_chain<23, 29, false>(n, st, scr);
    }
  }
  // ---- backward: arms into the torso, waist into the pelvis, then legs
  AI acc0;
  SV accP0;
  {
    AI acc15 = body_inertia<15>();
    SV accP15 = load_bias<15>(scr);
    bwd_chain_from_leaf<16, 22>(acc15, accP15, st, io, ep, cfg, scr);
    bwd_chain_from_leaf<23, 29>(acc15, accP15, st, io, ep, cfg, scr);
    acc0 = pelvis_inertia(ep.dmass);
    accP0 = load_bias<0>(scr);
    AI IA14 = body_inertia<14>();
    SV pA14 = load_bias<14>(scr);
    bwd_body<15>(acc15, accP15, IA14, pA14, st, io, ep, cfg, scr);
    AI IA13 = body_inertia<13>();
    SV pA13 = load_bias<13>(scr);
    bwd_body<14>(IA14, pA14, IA13, pA13, st, io, ep, cfg, scr);
    bwd_body<13>(IA13, pA13, acc0, accP0, st, io, ep, cfg, scr);
  }
  bwd_chain_from_leaf<1, 6>(acc0, accP0, st, io, ep, cfg, scr);
  bwd_chain_from_leaf<7, 12>(acc0, accP0, st, io, ep, cfg, scr);
  // ---- base acceleration and forward pass (fused with integration)
  const SV a0 = base_solve(acc0, accP0);
  const float dt = cfg.dt;
  // base: MuJoCo free-joint qacc (world linear incl. w x v, body angular);
  // uses the pre-integration base frame, rebuilt from the unchanged state
  {
    FKNode base;
    base_node(st, cfg, base);
    const V3 al = mv(base.R, add(a0.l, crs(base.w, base.v)));
#pragma unroll
    for (int k = 0; k < 3; ++k) st.vw[k] += dt * al.v[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) st.wb[k] += dt * a0.a.v[k];
  }
  fwd_chain<1, 6>(a0, st, dt, scr);
  fwd_chain<7, 12>(a0, st, dt, scr);
  {
    SV a = a0;
    fwd_body<13>(a, st, dt, scr);
    fwd_body<14>(a, st, dt, scr);
    fwd_body<15>(a, st, dt, scr);
    fwd_chain<16, 22>(a, st, dt, scr);
    fwd_chain<23, 29>(a, st, dt, scr);
  }
  // ---- base position and orientation (semi-implicit Euler)
  {
#pragma unroll
    for (int k = 0; k < 3; ++k) st.pos[k] += dt * st.vw[k];
    // q <- q (x) exp(w dt / 2), renormalised (reference src/spatial.h:73-79)
    const float wx = st.wb[0], wy = st.wb[1], wz = st.wb[2];
    const float wn = sqrtf(wx * wx + wy * wy + wz * wz);
    const float angle = wn * dt;
    if (angle >= 1e-12f) {
      float sh, ch;
      sincosf(0.5f * angle, &sh, &ch);
      const float k = sh / wn;
      const float dq[4] = {ch, k * wx, k * wy, k * wz};
      const float* a = st.quat;
      float r[4];
      r[0] = a[0] * dq[0] - a[1] * dq[1] - a[2] * dq[2] - a[3] * dq[3];
      r[1] = a[0] * dq[1] + a[1] * dq[0] + a[2] * dq[3] - a[3] * dq[2];
      r[2] = a[0] * dq[2] - a[1] * dq[3] + a[2] * dq[0] + a[3] * dq[1];
      r[3] = a[0] * dq[3] + a[1] * dq[2] - a[2] * dq[1] + a[3] * dq[0];
      quat_normalized(r, st.quat);
    }
  }
}

}  // namespace g1b
