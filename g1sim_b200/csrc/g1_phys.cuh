// g1_phys.cuh -- FP32 G1 step for one environment per thread.
//
// The step is the reference's
//   FK + velocities          (reference src/g1_core.h:29-54)
//   contacts, PD, ABA        (reference src/g1_core.h:109-207)
//   semi-implicit Euler      (reference src/g1_core.h:212-222)
// re-derived for the G1's structure instead of a generic tree walk:
//   * every hinge axis is +x, +y or +z and every joint anchor is the body
//     origin, so S = [e_ax; 0]: U = IA S is a column of IA, S^T f picks one
//     component, the joint rotation mixes two coordinates with (cos, sin);
//     each per-hinge routine exists in three axis-specialised copies and is
//     dispatched by a warp-uniform switch (all threads of a warp process the
//     same hinge);
//   * tree rotations, tree offsets, rigid-body spatial inertias and servo
//     parameters are precomputed per body in a constant table (no per-step
//     quat_to_mat / spatial_inertia);
//   * the tree is 5 serial chains (left leg 1-6, right leg 7-12, waist 13-15,
//     left arm 16-22, right arm 23-29) hanging off the pelvis (0) and the
//     torso (15); each phase loops over a chain's hinges, so the backward
//     pass keeps ONE running articulated inertia per chain plus accumulators
//     at the two branch bodies, and the code stays small enough for the
//     instruction cache;
//   * articulated inertias are kept as blocks J (sym), H (3x3), M (sym),
//     moved child->parent by the axis rotation (2-plane mix), the tree
//     rotation and the offset;
//   * contacts run right after each foot's FK and add a world-frame wrench.
// Per-hinge values the later passes need (joint angle and rate, cos/sin,
// velocity-product term c, bias force then U, u, 1/D) live in a Scratch
// (shared memory on the device).
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

// Per-step configuration (mirrors the reference G1Config, src/g1_types.h:33-42).
struct StepConfig {
  float gravity_z, contact_kn, contact_dn, contact_kt, contact_dt, limit_kp, limit_kd, dt;
};

// ------------------------------------------------------------ model table
// Everything one body contributes, in float.  Built at compile time from the
// generated double tables; on the device it lives in constant memory and is
// indexed by a warp-uniform body index.
struct BodyC {
  float T[9];        // tree rotation (parent <- body, before the joint), row-major
  float p[3];        // body origin in the parent frame
  float J[6], H[9];  // rigid spatial inertia at the origin: J (xx yy zz xy xz yz), H = m [c]x
  float m;
  float kp, kv, lim, lo, hi, arm, damp;  // servo and joint (hinges only)
  int axis, ident;
  // extended precision for the leg world-pose chain: p = p + p_lo, and the
  // tree rotation as a rotation about y by an angle with cos / sin = hi + lo
  float p_lo[3];
  float ty_c, ty_c_lo, ty_s, ty_s_lo;
};
struct ModelC {
  BodyC b[kNB];
  float stand[kNQ];
  float contact_pos[3 * kNC];
  float com0[3], icom0[6];  // pelvis COM and rotational inertia about it
};
constexpr ModelC make_model() {
  ModelC M{};
  for (int i = 0; i < kNB; ++i) {
    BodyC& b = M.b[i];
    for (int k = 0; k < 9; ++k) b.T[k] = (float)g1m_tree_rot[9 * i + k];
    for (int k = 0; k < 3; ++k) b.p[k] = (float)g1m_tree_pos[3 * i + k];
    for (int k = 0; k < 6; ++k) b.J[k] = (float)g1m_sp_inertia[16 * i + k];
    for (int k = 0; k < 9; ++k) b.H[k] = (float)g1m_sp_inertia[16 * i + 6 + k];
    b.m = (float)g1m_sp_inertia[16 * i + 15];
    b.ident = g1m_tree_ident[i];
    for (int k = 0; k < 3; ++k) b.p_lo[k] = (float)(g1m_tree_pos[3 * i + k] - (double)b.p[k]);
    b.ty_c = (float)g1m_tree_ycs[2 * i];
    b.ty_c_lo = (float)(g1m_tree_ycs[2 * i] - (double)b.ty_c);
    b.ty_s = (float)g1m_tree_ycs[2 * i + 1];
    b.ty_s_lo = (float)(g1m_tree_ycs[2 * i + 1] - (double)b.ty_s);
    if (i > 0) {
      const int h = i - 1;
      b.kp = (float)g1m_act_kp[h];
      b.kv = (float)g1m_act_kv[h];
      b.lim = (float)g1m_act_frclim[h];
      b.lo = (float)g1m_jnt_range[2 * h];
      b.hi = (float)g1m_jnt_range[2 * h + 1];
      b.arm = (float)g1m_armature[h];
      b.damp = (float)g1m_damping[h];
      b.axis = g1m_axis_idx[h];
    }
  }
  for (int k = 0; k < kNQ; ++k) M.stand[k] = (float)g1m_qpos_stand[k];
  for (int k = 0; k < 3 * kNC; ++k) M.contact_pos[k] = (float)g1m_contact_pos[k];
  for (int k = 0; k < 3; ++k) M.com0[k] = (float)g1m_com[k];
  M.icom0[0] = (float)g1m_inertia_com[0];
  M.icom0[1] = (float)g1m_inertia_com[4];
  M.icom0[2] = (float)g1m_inertia_com[8];
  M.icom0[3] = (float)g1m_inertia_com[1];
  M.icom0[4] = (float)g1m_inertia_com[2];
  M.icom0[5] = (float)g1m_inertia_com[5];
  return M;
}
#if defined(__CUDACC__)
static __constant__ ModelC c_model = make_model();
#endif
static constexpr ModelC kModel = make_model();
G1_HD const ModelC& model() {
#if defined(__CUDA_ARCH__)
  return c_model;
#else
  return kModel;
#endif
}
G1_HD const BodyC& body(int i) { return model().b[i]; }

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

// ---------------------------------------------- float-float arithmetic
// A value hi + lo held as two floats (unevaluated sum), with the error-free
// transformations TwoSum (Knuth), FastTwoSum (Dekker, |a| >= |b|) and the
// FMA-based TwoProd.  Used for the leg world-pose chain, where the contact
// depth is the difference of two ~0.8 m quantities and kn = 2e4 N/m turns
// FP32 rounding of positions into newton-level force errors.
struct F2 {
  float hi, lo;
};
G1_HD F2 f2(float x) { return F2{x, 0.0f}; }
G1_HD F2 fast_two_sum(float a, float b) {
  const float s = a + b;
  return F2{s, b - (s - a)};
}
G1_HD F2 two_sum(float a, float b) {
  const float s = a + b;
  const float bb = s - a;
  return F2{s, (a - (s - bb)) + (b - bb)};
}
G1_HD F2 two_prod(float a, float b) {
  const float p = a * b;
  return F2{p, fmaf(a, b, -p)};
}
G1_HD F2 ff_add(F2 x, F2 y) {
  const F2 t = two_sum(x.hi, y.hi);
  return fast_two_sum(t.hi, t.lo + (x.lo + y.lo));
}
G1_HD F2 ff_sub(F2 x, F2 y) { return ff_add(x, F2{-y.hi, -y.lo}); }
G1_HD F2 ff_mul(F2 x, F2 y) {
  const F2 p = two_prod(x.hi, y.hi);
  return fast_two_sum(p.hi, fmaf(x.hi, y.lo, fmaf(x.lo, y.hi, p.lo)));
}
G1_HD F2 ff_mul_f(F2 x, float y) {
  const F2 p = two_prod(x.hi, y);
  return fast_two_sum(p.hi, fmaf(x.lo, y, p.lo));
}

// sin / cos of k / 32 rad, hi + lo, |k| <= G1M_SINCOS_K.
struct SinCosTab {
  float v[2 * G1M_SINCOS_K + 1][4];  // sin hi, sin lo, cos hi, cos lo
};
constexpr SinCosTab make_sincos_tab() {
  SinCosTab t{};
  for (int k = 0; k < 2 * G1M_SINCOS_K + 1; ++k) {
    const double sn = g1m_sincos_tab[2 * k], cs = g1m_sincos_tab[2 * k + 1];
    t.v[k][0] = (float)sn;
    t.v[k][1] = (float)(sn - (double)(float)sn);
    t.v[k][2] = (float)cs;
    t.v[k][3] = (float)(cs - (double)(float)cs);
  }
  return t;
}
#if defined(__CUDACC__)
static __device__ SinCosTab d_sincos_tab = make_sincos_tab();
#endif
static constexpr SinCosTab kSinCosTab = make_sincos_tab();

// sin and cos of a float angle to ~1e-14: q = k/32 + r with |r| <= 1/64
// (r is exact: Sterbenz), tabulated sin / cos (k/32), Taylor series of
// sin r and cos r to r^5 / r^6 (truncation < 1e-16), angle addition in
// float-float (the table-driven method of P. T. P. Tang).
G1_HD void sincos_ff(float q, F2& sn, F2& cs) {
  const float kf = rintf(q * 32.0f);
  if (!(fabsf(kf) <= (float)G1M_SINCOS_K)) {  // outside the table (or NaN)
    float s, c;
    sincosf(q, &s, &c);
    sn = f2(s);
    cs = f2(c);
    return;
  }
  const float r = q - kf * (1.0f / 32.0f);
  const int k = (int)kf + G1M_SINCOS_K;
#if defined(__CUDA_ARCH__)
  const float4 e = __ldg(reinterpret_cast<const float4*>(&d_sincos_tab.v[k][0]));
  const F2 S{e.x, e.y}, C{e.z, e.w};
#else
  const F2 S{kSinCosTab.v[k][0], kSinCosTab.v[k][1]}, C{kSinCosTab.v[k][2], kSinCosTab.v[k][3]};
#endif
  const float r2 = r * r;
  const F2 sr = fast_two_sum(r, r * r2 * fmaf(r2, 1.0f / 120.0f, -1.0f / 6.0f));
  const F2 rr = two_prod(r, r);
  const F2 c1 = fast_two_sum(1.0f, -0.5f * rr.hi);
  const F2 cr = fast_two_sum(c1.hi, (c1.lo - 0.5f * rr.lo) + rr.hi * rr.hi * fmaf(rr.hi, -1.0f / 720.0f, 1.0f / 24.0f));
  sn = ff_add(ff_mul(S, cr), ff_mul(C, sr));
  cs = ff_sub(ff_mul(C, cr), ff_mul(S, sr));
}

// Right-multiply a float-float 3x3 by a rotation about basis axis AX with
// (c, s): columns i1 <- c i1 + s i2, i2 <- c i2 - s i1.
template <int AX>
G1_HD void ff_rot_cols(F2* R, F2 c, F2 s) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const F2 x = R[3 * a + i1], y = R[3 * a + i2];
    R[3 * a + i1] = ff_add(ff_mul(c, x), ff_mul(s, y));
    R[3 * a + i2] = ff_sub(ff_mul(c, y), ff_mul(s, x));
  }
}

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
  M3 B = H;
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    B.m[3 * i + col] = c * H.m[3 * i + col] - s * H.m[3 * j + col];
    B.m[3 * j + col] = s * H.m[3 * i + col] + c * H.m[3 * j + col];
  }
  M3 r = B;
#pragma unroll
  for (int row = 0; row < 3; ++row) {
    r.m[3 * row + i] = c * B.m[3 * row + i] - s * B.m[3 * row + j];
    r.m[3 * row + j] = s * B.m[3 * row + i] + c * B.m[3 * row + j];
  }
  return r;
}

// ---------------------------------------- tree rotation T (from the table)
G1_HD V3 rotT(const BodyC& b, const V3& x) {
  if (b.ident) return x;
  V3 r;
#pragma unroll
  for (int a = 0; a < 3; ++a) r.v[a] = b.T[3 * a] * x.v[0] + b.T[3 * a + 1] * x.v[1] + b.T[3 * a + 2] * x.v[2];
  return r;
}
G1_HD V3 rotTT(const BodyC& b, const V3& x) {
  if (b.ident) return x;
  V3 r;
#pragma unroll
  for (int a = 0; a < 3; ++a) r.v[a] = b.T[a] * x.v[0] + b.T[3 + a] * x.v[1] + b.T[6 + a] * x.v[2];
  return r;
}
G1_HD void rotT_sym(const BodyC& b, S3& S) {  // S <- T S T^T
  float B[9];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      B[3 * a + c] = b.T[3 * a] * S.s[sidx(0, c)] + b.T[3 * a + 1] * S.s[sidx(1, c)] + b.T[3 * a + 2] * S.s[sidx(2, c)];
  S3 r;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = a; c < 3; ++c)
      r.s[sidx(a, c)] = B[3 * a] * b.T[3 * c] + B[3 * a + 1] * b.T[3 * c + 1] + B[3 * a + 2] * b.T[3 * c + 2];
  S = r;
}
G1_HD void rotT_gen(const BodyC& b, M3& H) {  // H <- T H T^T
  float B[9];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) B[3 * a + c] = b.T[3 * a] * H.m[c] + b.T[3 * a + 1] * H.m[3 + c] + b.T[3 * a + 2] * H.m[6 + c];
  M3 r;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      r.m[3 * a + c] = B[3 * a] * b.T[3 * c] + B[3 * a + 1] * b.T[3 * c + 1] + B[3 * a + 2] * b.T[3 * c + 2];
  H = r;
}
// p x v
G1_HD V3 pcross(const BodyC& b, const V3& x) {
  return mk3(b.p[1] * x.v[2] - b.p[2] * x.v[1], b.p[2] * x.v[0] - b.p[0] * x.v[2], b.p[0] * x.v[1] - b.p[1] * x.v[0]);
}

// --------------------------------------------------- rigid-body inertias
G1_HD AI body_inertia(const BodyC& b) {
  AI r;
#pragma unroll
  for (int k = 0; k < 6; ++k) r.J.s[k] = b.J[k];
#pragma unroll
  for (int k = 0; k < 9; ++k) r.H.m[k] = b.H[k];
  r.M.s[0] = r.M.s[1] = r.M.s[2] = b.m;
  r.M.s[3] = r.M.s[4] = r.M.s[5] = 0.0f;
  return r;
}

// Pelvis inertia with a per-env mass offset (COM and rotational inertia
// about the COM unchanged): J = Icom + m [c]x [c]x^T, H = m [c]x, M = m 1.
G1_HD AI pelvis_inertia(float dmass) {
  const ModelC& M = model();
  const float cx = M.com0[0], cy = M.com0[1], cz = M.com0[2];
  const float m = M.b[0].m + dmass;
  AI r;
  r.J.s[0] = M.icom0[0] + m * (cy * cy + cz * cz);
  r.J.s[1] = M.icom0[1] + m * (cx * cx + cz * cz);
  r.J.s[2] = M.icom0[2] + m * (cx * cx + cy * cy);
  r.J.s[3] = M.icom0[3] - m * (cx * cy);
  r.J.s[4] = M.icom0[4] - m * (cx * cz);
  r.J.s[5] = M.icom0[5] - m * (cy * cz);
  r.H.m[0] = 0.0f;     r.H.m[1] = -m * cz; r.H.m[2] = m * cy;
  r.H.m[3] = m * cz;   r.H.m[4] = 0.0f;    r.H.m[5] = -m * cx;
  r.H.m[6] = -m * cy;  r.H.m[7] = m * cx;  r.H.m[8] = 0.0f;
  r.M.s[0] = r.M.s[1] = r.M.s[2] = m;
  r.M.s[3] = r.M.s[4] = r.M.s[5] = 0.0f;
  return r;
}

// Rigid-body bias force with gravity (reference src/g1_core.h:113-120):
//   pA = v x* (I v) - [c x (m g_b); m g_b],  [c x (m g); m g] = [H g; m g].
G1_HD SV bias_force(const AI& In, const V3& w, const V3& v, const V3& g) {
  V3 ha, hl;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    ha.v[a] = In.J.s[sidx(a, 0)] * w.v[0] + In.J.s[sidx(a, 1)] * w.v[1] + In.J.s[sidx(a, 2)] * w.v[2] +
              In.H.m[3 * a] * v.v[0] + In.H.m[3 * a + 1] * v.v[1] + In.H.m[3 * a + 2] * v.v[2];
    hl.v[a] = In.H.m[a] * w.v[0] + In.H.m[3 + a] * w.v[1] + In.H.m[6 + a] * w.v[2] + In.M.s[sidx(a, 0)] * v.v[0] +
              In.M.s[sidx(a, 1)] * v.v[1] + In.M.s[sidx(a, 2)] * v.v[2];
  }
  const V3 hg = mk3(In.H.m[0] * g.v[0] + In.H.m[1] * g.v[1] + In.H.m[2] * g.v[2],
                    In.H.m[3] * g.v[0] + In.H.m[4] * g.v[1] + In.H.m[5] * g.v[2],
                    In.H.m[6] * g.v[0] + In.H.m[7] * g.v[1] + In.H.m[8] * g.v[2]);
  SV r;
  r.a = sub(add(crs(w, ha), crs(v, hl)), hg);
  r.l = sub(crs(w, hl), scl(In.M.s[0], g));
  return r;
}

// ---------------------------------------------------------------- scratch
// Per hinge h (body h + 1), 11 slots: k = 0 q (slot h), 1 qd (slot 29 + h),
// and k = 2..10 at slot 58 + 9 h + (k - 2): 2 cos q, 3 sin q, 4-9 U / D
// (backward -> forward), 10 u / D.  The joint state comes first so that the
// rest of the scratch is free between substeps (the policy step reuses it
// for its network tiles).
// Per chain c (0 left leg, 1 right leg, 2 waist, 3 left arm, 4 right arm):
//   kSlotChain + 9 c: twist (6) and gravity (3) of the chain's last body
//   (FK -> backward; the backward pass recovers the other bodies' twist and
//   gravity by moving back up the chain).
// Per foot f: kSlotFoot + 6 f: contact wrench on the foot body (body frame).
// kSlotXchg..: exchanged between the two halves of a split step: the upper
// body's projection into the pelvis (27: J 6, H 9, M 6, bias 6), the base
// acceleration (6), the base state (13) and a reset flag (1).
constexpr int kSlotsPerHinge = 11;
constexpr int kSlotChain = kNJ * kSlotsPerHinge;
constexpr int kSlotFoot = kSlotChain + 5 * 9;
constexpr int kSlotXchg = kSlotFoot + 12;
constexpr int kXUp = kSlotXchg, kXA0 = kSlotXchg + 27, kXBase = kSlotXchg + 33, kXReset = kSlotXchg + 46;
constexpr int kNumSlotsSingle = kSlotXchg;  // one thread per env
constexpr int kNumSlots = kSlotXchg + 47;   // two threads per env
// three threads per env (left leg, right leg, upper body): also the right
// leg's projection into the pelvis (27)
constexpr int kXLeg = kNumSlots;
constexpr int kNumSlots3 = kNumSlots + 27;
// two threads per env: the env's contact anchors (2 per sphere), held on chip
// for every substep of a tile instead of read from and written to global
// memory in each one (the contacts waited on those reads, each right after
// the previous substep's store)
constexpr int kXAnchor = kNumSlots;
constexpr int kNumSlotsSplit = kNumSlots + 2 * kNC;
constexpr int kSlotJointState = 2 * kNJ;  // q and qd of every hinge
G1_CE int hslot(int body, int k) {
  return k < 2 ? k * kNJ + (body - 1) : kSlotJointState + (body - 1) * (kSlotsPerHinge - 2) + (k - 2);
}

// ----------------------------------------------------------- env data
// Base state kept in registers; joint angles and rates live in the scratch.
struct EnvState {
  float pos[3], quat[4], vw[3], wb[3];
};
// One env's arrays that stay in memory during a step (SoA, element i of the
// env at p[i * stride]): PD targets read once per hinge, contact anchors read
// and written by the contacts, last-substep outputs (nullable).
struct EnvIO {
  const float* ctrl;
  float* anchor;  // element i at anchor[i * astride]
  float* foot_pos;
  float* foot_vel;
  float* cf;
  size_t stride;
  size_t astride;
};
struct EnvParams {
  float mu, dmass, kp_scale, kd_scale;
};

// Running FK values of one body: body-frame twist, gravity, and (legs only)
// the world pose in float-float (Rf, Pf) with its float rounding (R, P).
struct FKNode {
  V3 w, v, g;
  M3 R;
  V3 P;
  F2 Rf[9], Pf[3];
};

template <class Scr>
G1_HD void store_sv(Scr& scr, int s0, const SV& x) {
#pragma unroll
  for (int k = 0; k < 3; ++k) scr.put(s0 + k, x.a.v[k]);
#pragma unroll
  for (int k = 0; k < 3; ++k) scr.put(s0 + 3 + k, x.l.v[k]);
}
template <class Scr>
G1_HD SV load_sv(Scr& scr, int s0) {
  SV r;
#pragma unroll
  for (int k = 0; k < 3; ++k) r.a.v[k] = scr.get(s0 + k);
#pragma unroll
  for (int k = 0; k < 3; ++k) r.l.v[k] = scr.get(s0 + 3 + k);
  return r;
}
template <class Scr>
G1_HD void store_end(Scr& scr, int c, const FKNode& n) {
  const int s0 = kSlotChain + 9 * c;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    scr.put(s0 + k, n.w.v[k]);
    scr.put(s0 + 3 + k, n.v.v[k]);
    scr.put(s0 + 6 + k, n.g.v[k]);
  }
}
template <class Scr>
G1_HD void load_end(Scr& scr, int c, V3& w, V3& v, V3& g) {
  const int s0 = kSlotChain + 9 * c;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    w.v[k] = scr.get(s0 + k);
    v.v[k] = scr.get(s0 + 3 + k);
    g.v[k] = scr.get(s0 + 6 + k);
  }
}

// chains: 0 left leg 1-6, 1 right leg 7-12, 2 waist 13-15, 3 left arm
// 16-22, 4 right arm 23-29; legs and waist hang off the pelvis, arms off the
// torso (15)
G1_HD int chain_first(int c) { return c == 0 ? 1 : c == 1 ? 7 : c == 2 ? 13 : c == 3 ? 16 : 23; }
G1_HD int chain_last(int c) { return c == 0 ? 6 : c == 1 ? 12 : c == 2 ? 15 : c == 3 ? 22 : 29; }

G1_HD void sv_zero(SV& x) { x.a = x.l = mk3(0.f, 0.f, 0.f); }
G1_HD void sv_acc(SV& x, const SV& y) {
  x.a = add(x.a, y.a);
  x.l = add(x.l, y.l);
}

// velocity-product term c = v x_m (qd S) = [qd (w x e_ax); qd (v x e_ax)]:
// four non-zeros, angular i1, i2 then linear i1, i2
template <int AX>
G1_HD void vel_product(const V3& w, const V3& v, float qd, float* cv) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  cv[0] = qd * w.v[i2];
  cv[1] = -(qd * w.v[i1]);
  cv[2] = qd * v.v[i2];
  cv[3] = -(qd * v.v[i1]);
}

// ------------------------------------------------------------- FK pass
// reference src/g1_core.h:29-54: parent -> child twist and gravity; with
// kWorld (legs) also the world pose in float-float, and the joint's sin/cos
// from the extended-precision routine.
template <int AX, bool kWorld, class Scr>
G1_HD void fk_body(int i, FKNode& n, Scr& scr) {
  const BodyC& b = body(i);
  const float q = scr.get(hslot(i, 0)), qd = scr.get(hslot(i, 1));
  float s, c;
  F2 sf, cf;
  if constexpr (kWorld) {
    sincos_ff(q, sf, cf);
    s = sf.hi;
    c = cf.hi;
  } else {
    sincosf(q, &s, &c);
  }
  scr.put(hslot(i, 2), c);
  scr.put(hslot(i, 3), s);
  // parent -> child: x_c = A^T T^T x_p ;  v.l uses v_p - p x w_p
  const V3 t = sub(n.v, pcross(b, n.w));
  V3 w = rotAT<AX>(rotTT(b, n.w), c, s);
  const V3 v = rotAT<AX>(rotTT(b, t), c, s);
  const V3 g = rotAT<AX>(rotTT(b, n.g), c, s);
  w.v[AX] += qd;
  if constexpr (kWorld) {
    // world pose in float-float: P_i = P_p + R_p p ; R_i = R_p T A
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      F2 acc = n.Pf[a];
#pragma unroll
      for (int k = 0; k < 3; ++k) acc = ff_add(acc, ff_mul(n.Rf[3 * a + k], F2{b.p[k], b.p_lo[k]}));
      n.Pf[a] = acc;
    }
    if (!b.ident) ff_rot_cols<1>(n.Rf, F2{b.ty_c, b.ty_c_lo}, F2{b.ty_s, b.ty_s_lo});
    ff_rot_cols<AX>(n.Rf, cf, sf);
#pragma unroll
    for (int k = 0; k < 9; ++k) n.R.m[k] = n.Rf[k].hi;
#pragma unroll
    for (int k = 0; k < 3; ++k) n.P.v[k] = n.Pf[k].hi;
  }
  n.w = w;
  n.v = v;
  n.g = g;
}

// FK of the serial chain first..last from the node of its parent.
template <bool kWorld, class Scr>
G1_HD void fk_chain(int first, int last, FKNode& n, Scr& scr) {
#pragma unroll 1
  for (int i = first; i <= last; ++i) {
    switch (body(i).axis) {
      case 0: fk_body<0, kWorld>(i, n, scr); break;
      case 1: fk_body<1, kWorld>(i, n, scr); break;
      default: fk_body<2, kWorld>(i, n, scr); break;
    }
  }
}

// --------------------------------------------------------------- contacts
// Eight spheres, four on each foot (reference src/g1_core.h:123-153).  The
// world wrench about the foot origin is accumulated and rotated to the body
// frame once; returns the wrench's contribution to the foot's bias force.
G1_HD SV foot_contacts(int K0, const FKNode& n, const EnvIO& io, bool last, const StepConfig& cfg, float mu) {
  float* anchor = io.anchor;
  const size_t sd = io.stride, sa = io.astride;
  const V3 ww = mv(n.R, n.w);  // world angular velocity
  const V3 vo = mv(n.R, n.v);  // world velocity of the foot origin
  V3 F = mk3(0.f, 0.f, 0.f), Tq = mk3(0.f, 0.f, 0.f);
  const float radius = (float)g1m_contact_radius;
  const float inv_kt = 1.0f / cfg.contact_kt;
  const ModelC& M = model();
#pragma unroll 1
  for (int k = K0; k < K0 + 4; ++k) {
    const V3 r = mk3(M.contact_pos[3 * k], M.contact_pos[3 * k + 1], M.contact_pos[3 * k + 2]);
    const V3 rw = mv(n.R, r);
    // sphere centre in float-float: P + R r
    F2 pc[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      pc[a] = ff_add(ff_add(n.Pf[a], ff_mul_f(n.Rf[3 * a], r.v[0])),
                     ff_add(ff_mul_f(n.Rf[3 * a + 1], r.v[1]), ff_mul_f(n.Rf[3 * a + 2], r.v[2])));
    const float px = pc[0].hi, py = pc[1].hi;
    const float depth = (radius - pc[2].hi) - pc[2].lo;
    const bool in = depth > 0.0f;
    const V3 vp = add(vo, crs(ww, rw));
    float fn = cfg.contact_kn * depth - cfg.contact_dn * vp.v[2];
    fn = fminf(fmaxf(fn, 0.0f), 500.0f);
    float ax = anchor[(2 * k) * sa], ay = anchor[(2 * k + 1) * sa];
    const bool fresh = ax >= kAnchorFree;
    ax = fresh ? px : ax;
    ay = fresh ? py : ay;
    // spring stretch (p - anchor) with the low part of p kept
    const float dx = (px - ax) + pc[0].lo, dy = (py - ay) + pc[1].lo;
    float ftx = -cfg.contact_kt * dx - cfg.contact_dt * vp.v[0];
    float fty = -cfg.contact_kt * dy - cfg.contact_dt * vp.v[1];
    const float ftn = sqrtf(ftx * ftx + fty * fty), fmax = mu * fn;
    if (ftn > fmax) {
      const float sc = fmax / (ftn + 1e-12f);
      ftx *= sc;
      fty *= sc;
      ax = px + (ftx * inv_kt + pc[0].lo);
      ay = py + (fty * inv_kt + pc[1].lo);
    }
    if (in) {
      anchor[(2 * k) * sa] = ax;
      anchor[(2 * k + 1) * sa] = ay;
      const V3 f = mk3(ftx, fty, fn);
      F = add(F, f);
      Tq = add(Tq, crs(rw, f));
    } else {
      fn = 0.0f;
      anchor[(2 * k) * sa] = kAnchorFree;
      anchor[(2 * k + 1) * sa] = kAnchorFree;
    }
    if (last && io.cf) io.cf[k * sd] = fn;
  }
  SV r;
  r.a = scl(-1.0f, mtv(n.R, Tq));
  r.l = scl(-1.0f, mtv(n.R, F));
  return r;
}

// --------------------------------------------------------- backward pass
// Transform the child articulated inertia Ia (child frame) into the parent
// frame and add it: X* Ia X^-1 with X = (R = T A, p).  Blocks after the
// rotation (J2, H2, M2), then the offset P = [p]x:
//   H' = H2 + P M2 ;  J' = J2 + P H2^T - H' P ;  M' = M2.
template <int AX>
G1_HD void ai_to_parent_add(const BodyC& b, AI& acc, const AI& Ia, float c, float s) {
  S3 J = rotA_sym<AX>(Ia.J, c, s);
  M3 H = rotA_gen<AX>(Ia.H, c, s);
  S3 M = rotA_sym<AX>(Ia.M, c, s);
  if (!b.ident) {
    rotT_sym(b, J);
    rotT_gen(b, H);
    rotT_sym(b, M);
  }
  // H' = H + P M : (P M)[r][col] = (p x M[:,col])_r
  M3 Hn;
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    const V3 pm = pcross(b, mk3(M.s[sidx(0, col)], M.s[sidx(1, col)], M.s[sidx(2, col)]));
#pragma unroll
    for (int r = 0; r < 3; ++r) Hn.m[3 * r + col] = H.m[3 * r + col] + pm.v[r];
  }
  // J' = J + P H^T - H' P ; (P H^T)[r][c] = (p x H[c,:])_r ; (H' P)[r][c] = -(p x H'[r,:])_c
  V3 pHT[3], HnP[3];
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) pHT[cc] = pcross(b, mk3(H.m[3 * cc], H.m[3 * cc + 1], H.m[3 * cc + 2]));
#pragma unroll
  for (int r = 0; r < 3; ++r) HnP[r] = pcross(b, mk3(Hn.m[3 * r], Hn.m[3 * r + 1], Hn.m[3 * r + 2]));
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int cc = r; cc < 3; ++cc) acc.J.s[sidx(r, cc)] += J.s[sidx(r, cc)] + pHT[cc].v[r] + HnP[r].v[cc];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc.H.m[k] += Hn.m[k];
#pragma unroll
  for (int k = 0; k < 6; ++k) acc.M.s[k] += M.s[k];
}

// force child -> parent: [R f.a + p x (R f.l); R f.l]
template <int AX>
G1_HD SV f_to_parent(const BodyC& b, const SV& f, float c, float s) {
  SV r;
  r.l = rotT(b, rotA<AX>(f.l, c, s));
  r.a = add(rotT(b, rotA<AX>(f.a, c, s)), pcross(b, r.l));
  return r;
}

// One hinge of the backward pass with PD servo, soft limits and implicit
// damping (reference src/g1_core.h:156-186).  IA, pA are body i's
// articulated inertia and bias, (w, v) its twist; the projected values are
// added into (accI, accP), expressed in the parent's frame, and (w, v, g)
// are moved to the parent: v_p = X (v_i - qd S), g_p = R g_i.
template <int AX, class Scr>
G1_HD void bwd_body(int i, const AI& IA, const SV& pA, V3& w, V3& v, V3& g, AI& accI, SV& accP,
                    const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const BodyC& b = body(i);
  const int h = i - 1;
  const float c = scr.get(hslot(i, 2)), s = scr.get(hslot(i, 3));
  // U = IA S: column AX of J, row AX of H
  SV U;
#pragma unroll
  for (int a = 0; a < 3; ++a) U.a.v[a] = IA.J.s[sidx(a, AX)];
#pragma unroll
  for (int a = 0; a < 3; ++a) U.l.v[a] = IA.H.m[3 * AX + a];
  const float q = scr.get(hslot(i, 0)), qd = scr.get(hslot(i, 1));
  const float kp = b.kp * ep.kp_scale, kv = b.kv * ep.kd_scale;
  float t = kp * (io.ctrl[h * io.stride] - q) - kv * qd;
  t = fminf(fmaxf(t, -b.lim), b.lim);
  float bd = kv + b.damp;
  if (q < b.lo) {
    t += cfg.limit_kp * (b.lo - q) - cfg.limit_kd * qd;
    bd += cfg.limit_kd;
  }
  if (q > b.hi) {
    t += cfg.limit_kp * (b.hi - q) - cfg.limit_kd * qd;
    bd += cfg.limit_kd;
  }
  const float D = U.a.v[AX] + b.arm + cfg.dt * bd;
  const float u = t - b.damp * qd - pA.a.v[AX];
  const float invD = 1.0f / D;
  float cv[4];
  vel_product<AX>(w, v, qd, cv);
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
    pa.a.v[a] = pA.a.v[a] + Ia.J.s[sidx(a, i1)] * cv[0] + Ia.J.s[sidx(a, i2)] * cv[1] +
                Ia.H.m[3 * a + i1] * cv[2] + Ia.H.m[3 * a + i2] * cv[3] + uD * U.a.v[a];
    pa.l.v[a] = pA.l.v[a] + Ia.H.m[3 * i1 + a] * cv[0] + Ia.H.m[3 * i2 + a] * cv[1] +
                Ia.M.s[sidx(a, i1)] * cv[2] + Ia.M.s[sidx(a, i2)] * cv[3] + uD * U.l.v[a];
  }
  // keep U / D and u / D for the forward pass
  store_sv(scr, hslot(i, 4), W);
  scr.put(hslot(i, 10), uD);
  ai_to_parent_add<AX>(b, accI, Ia, c, s);
  const SV fp = f_to_parent<AX>(b, pa, c, s);
  accP.a = add(accP.a, fp.a);
  accP.l = add(accP.l, fp.l);
  // twist and gravity of the parent
  V3 wm = w;
  wm.v[AX] -= qd;
  const V3 wp = rotT(b, rotA<AX>(wm, c, s));
  v = add(rotT(b, rotA<AX>(v, c, s)), pcross(b, wp));
  w = wp;
  g = rotT(b, rotA<AX>(g, c, s));
}

G1_HD void ai_zero(AI& A) {
#pragma unroll
  for (int k = 0; k < 6; ++k) A.J.s[k] = A.M.s[k] = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; ++k) A.H.m[k] = 0.0f;
}
G1_HD void ai_add(AI& A, const AI& B) {
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    A.J.s[k] += B.J.s[k];
    A.M.s[k] += B.M.s[k];
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) A.H.m[k] += B.H.m[k];
}

// Backward pass over the serial chain first..last.  (IA, pA) are the
// articulated inertia and bias of its last body and (w, v, g) that body's
// twist and gravity; the chain's projection into its parent is returned in
// (outI, outP).  Each body's rigid bias force is computed here from the
// recovered twist (reference src/g1_core.h:113-120).
template <class Scr>
G1_HD void bwd_chain(int first, int last, AI IA, SV pA, V3 w, V3 v, V3 g, AI& outI, SV& outP,
                     const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr) {
#pragma unroll 1
  for (int i = last; i >= first; --i) {
    AI IAp;
    SV pAp;
    if (i > first) {
      IAp = body_inertia(body(i - 1));
    } else {
      ai_zero(IAp);
    }
    sv_zero(pAp);
    switch (body(i).axis) {
      case 0: bwd_body<0>(i, IA, pA, w, v, g, IAp, pAp, io, ep, cfg, scr); break;
      case 1: bwd_body<1>(i, IA, pA, w, v, g, IAp, pAp, io, ep, cfg, scr); break;
      default: bwd_body<2>(i, IA, pA, w, v, g, IAp, pAp, io, ep, cfg, scr); break;
    }
    if (i > first) sv_acc(pAp, bias_force(body_inertia(body(i - 1)), w, v, g));
    IA = IAp;
    pA = pAp;
  }
  outI = IA;
  outP = pA;
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
// The twist is carried down the chain again (v_i = X^-1 v_p + qd S, with the
// rate before this substep's update) for the velocity-product term;
// a_i = X^-1 a_p + c_i ; qdd = u/D - (U/D).a_i ; a_i += qdd S  (reference
// src/g1_core.h:190-201), fused with the hinge's semi-implicit Euler update
// (reference src/g1_core.h:214,221).
template <int AX, class Scr>
G1_HD void fwd_body(int i, SV& a, V3& w, V3& v, float dt, Scr& scr) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const BodyC& b = body(i);
  const float c = scr.get(hslot(i, 2)), s = scr.get(hslot(i, 3));
  const float qd0 = scr.get(hslot(i, 1));
  // twist of body i (as in the FK pass)
  const V3 tv = sub(v, pcross(b, w));
  w = rotAT<AX>(rotTT(b, w), c, s);
  v = rotAT<AX>(rotTT(b, tv), c, s);
  w.v[AX] += qd0;
  float cv[4];
  vel_product<AX>(w, v, qd0, cv);
  const V3 t = sub(a.l, pcross(b, a.a));
  SV an;
  an.a = rotAT<AX>(rotTT(b, a.a), c, s);
  an.l = rotAT<AX>(rotTT(b, t), c, s);
  an.a.v[i1] += cv[0];
  an.a.v[i2] += cv[1];
  an.l.v[i1] += cv[2];
  an.l.v[i2] += cv[3];
  const SV W = load_sv(scr, hslot(i, 4));  // U / D
  const float uD = scr.get(hslot(i, 10));  // u / D
  const float qdd = uD - (W.a.v[0] * an.a.v[0] + W.a.v[1] * an.a.v[1] + W.a.v[2] * an.a.v[2] +
                          W.l.v[0] * an.l.v[0] + W.l.v[1] * an.l.v[1] + W.l.v[2] * an.l.v[2]);
  an.a.v[AX] += qdd;
  a = an;
  const float qd = qd0 + dt * qdd;
  scr.put(hslot(i, 1), qd);
  scr.put(hslot(i, 0), scr.get(hslot(i, 0)) + dt * qd);
}

template <class Scr>
G1_HD void fwd_chain(int first, int last, SV& a, V3& w, V3& v, float dt, Scr& scr) {
#pragma unroll 1
  for (int i = first; i <= last; ++i) {
    switch (body(i).axis) {
      case 0: fwd_body<0>(i, a, w, v, dt, scr); break;
      case 1: fwd_body<1>(i, a, w, v, dt, scr); break;
      default: fwd_body<2>(i, a, w, v, dt, scr); break;
    }
  }
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

// Base world pose in float-float: R(q) of the (not exactly unit) stored
// quaternion, R = I + 2/|q|^2 [..] (the reference normalises, then converts,
// src/g1_core.h:31-32; same matrix), and the position.
G1_HD void base_pose_ff(const EnvState& st, FKNode& n) {
  const float w = st.quat[0], x = st.quat[1], y = st.quat[2], z = st.quat[3];
  const F2 ww = two_prod(w, w), xx = two_prod(x, x), yy = two_prod(y, y), zz = two_prod(z, z);
  const F2 n2 = ff_add(ff_add(ww, xx), ff_add(yy, zz));
  // 2 / |q|^2: float reciprocal refined by one Newton step in float-float
  const float y0 = 1.0f / n2.hi;
  const F2 e = ff_sub(f2(1.0f), ff_mul_f(n2, y0));
  const F2 inv2 = fast_two_sum(2.0f * y0, 2.0f * y0 * e.hi);
  const F2 xy = two_prod(x, y), xz = two_prod(x, z), yz = two_prod(y, z);
  const F2 wx = two_prod(w, x), wy = two_prod(w, y), wz = two_prod(w, z);
  n.Rf[0] = ff_sub(f2(1.0f), ff_mul(inv2, ff_add(yy, zz)));
  n.Rf[1] = ff_mul(inv2, ff_sub(xy, wz));
  n.Rf[2] = ff_mul(inv2, ff_add(xz, wy));
  n.Rf[3] = ff_mul(inv2, ff_add(xy, wz));
  n.Rf[4] = ff_sub(f2(1.0f), ff_mul(inv2, ff_add(xx, zz)));
  n.Rf[5] = ff_mul(inv2, ff_sub(yz, wx));
  n.Rf[6] = ff_mul(inv2, ff_sub(xz, wy));
  n.Rf[7] = ff_mul(inv2, ff_add(yz, wx));
  n.Rf[8] = ff_sub(f2(1.0f), ff_mul(inv2, ff_add(xx, yy)));
#pragma unroll
  for (int k = 0; k < 3; ++k) n.Pf[k] = f2(st.pos[k]);
}

G1_HD void foot_outputs(const FKNode& n, const EnvIO& io, int o) {
  if (io.foot_pos)
#pragma unroll
    for (int k = 0; k < 3; ++k) io.foot_pos[(o + k) * io.stride] = n.P.v[k];
  if (io.foot_vel) {
    const V3 fv = mv(n.R, n.v);
#pragma unroll
    for (int k = 0; k < 3; ++k) io.foot_vel[(o + k) * io.stride] = fv.v[k];
  }
}

// ============================================================ exchange
template <class Scr>
G1_HD void store_ai(Scr& scr, int s0, const AI& A, const SV& p) {
#pragma unroll
  for (int k = 0; k < 6; ++k) scr.put(s0 + k, A.J.s[k]);
#pragma unroll
  for (int k = 0; k < 9; ++k) scr.put(s0 + 6 + k, A.H.m[k]);
#pragma unroll
  for (int k = 0; k < 6; ++k) scr.put(s0 + 15 + k, A.M.s[k]);
  store_sv(scr, s0 + 21, p);
}
template <class Scr>
G1_HD void load_ai(Scr& scr, int s0, AI& A, SV& p) {
#pragma unroll
  for (int k = 0; k < 6; ++k) A.J.s[k] = scr.get(s0 + k);
#pragma unroll
  for (int k = 0; k < 9; ++k) A.H.m[k] = scr.get(s0 + 6 + k);
#pragma unroll
  for (int k = 0; k < 6; ++k) A.M.s[k] = scr.get(s0 + 15 + k);
  p = load_sv(scr, s0 + 21);
}
template <class Scr>
G1_HD void store_base(Scr& scr, const EnvState& st) {
#pragma unroll
  for (int k = 0; k < 3; ++k) scr.put(kXBase + k, st.pos[k]);
#pragma unroll
  for (int k = 0; k < 4; ++k) scr.put(kXBase + 3 + k, st.quat[k]);
#pragma unroll
  for (int k = 0; k < 3; ++k) scr.put(kXBase + 7 + k, st.vw[k]);
#pragma unroll
  for (int k = 0; k < 3; ++k) scr.put(kXBase + 10 + k, st.wb[k]);
}
template <class Scr>
G1_HD void load_base(Scr& scr, EnvState& st) {
#pragma unroll
  for (int k = 0; k < 3; ++k) st.pos[k] = scr.get(kXBase + k);
#pragma unroll
  for (int k = 0; k < 4; ++k) st.quat[k] = scr.get(kXBase + 3 + k);
#pragma unroll
  for (int k = 0; k < 3; ++k) st.vw[k] = scr.get(kXBase + 7 + k);
#pragma unroll
  for (int k = 0; k < 3; ++k) st.wb[k] = scr.get(kXBase + 10 + k);
}

// ================================================================= phases
// The substep split in the phases of the two halves of the tree: the lower
// body (pelvis, legs, contacts, base) and the upper body (waist, arms).  One
// thread runs all of them in order (step); the split kernel runs the lower
// phases on one thread and the upper phases on another, exchanging the upper
// body's projection into the pelvis, the base acceleration and the base
// state through the scratch.

// ------------------------------------------ one leg (three-role split)
// FK of leg c (0 left, 1 right) in extended precision and its contacts;
// stores the chain end, the foot wrench and (last substep) the foot outputs.
template <class Scr>
G1_HD void fk_leg(const EnvState& st, int c, const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr,
                  bool last_sub) {
  FKNode n;
  base_node(st, cfg, n);
  base_pose_ff(st, n);
  fk_chain<true>(chain_first(c), chain_last(c), n, scr);
  const SV wr = foot_contacts(4 * c, n, io, last_sub, cfg, ep.mu);
  store_sv(scr, kSlotFoot + 6 * c, wr);
  store_end(scr, c, n);
  if (last_sub) foot_outputs(n, io, c == 0 ? 0 : 3);
}

// Backward pass of leg c: its projection into the pelvis frame.
template <class Scr>
G1_HD void bwd_leg(int c, const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr, AI& outI, SV& outP) {
  V3 w, v, g;
  load_end(scr, c, w, v, g);
  const int last = chain_last(c);
  const AI IA = body_inertia(body(last));
  SV pA = bias_force(IA, w, v, g);
  sv_acc(pA, load_sv(scr, kSlotFoot + 6 * c));
  bwd_chain(chain_first(c), last, IA, pA, w, v, g, outI, outP, io, ep, cfg, scr);
}

// The pelvis's own articulated inertia and bias force.
G1_HD void pelvis_acc(const EnvState& st, const EnvParams& ep, const StepConfig& cfg, AI& acc0, SV& accP0) {
  FKNode base;
  base_node(st, cfg, base);
  acc0 = pelvis_inertia(ep.dmass);
  accP0 = bias_force(acc0, base.w, base.v, base.g);
}

// Forward pass of leg c from the base acceleration (st: the base state at
// the start of the substep).
template <class Scr>
G1_HD void fwd_leg(const EnvState& st, int c, const SV& a0, const StepConfig& cfg, Scr& scr) {
  FKNode base;
  base_node(st, cfg, base);
  SV a = a0;
  V3 w = base.w, v = base.v;
  fwd_chain(chain_first(c), chain_last(c), a, w, v, cfg.dt, scr);
}

// Base integration (semi-implicit Euler; the free-joint convention of
// fwd_lower_and_base).
G1_HD void integrate_base(EnvState& st, const SV& a0, const StepConfig& cfg) {
  const float dt = cfg.dt;
  FKNode base;
  base_node(st, cfg, base);
  const V3 al = mv(base.R, add(a0.l, crs(base.w, base.v)));
#pragma unroll
  for (int k = 0; k < 3; ++k) st.vw[k] += dt * al.v[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) st.wb[k] += dt * a0.a.v[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) st.pos[k] += dt * st.vw[k];
  const float wx = st.wb[0], wy = st.wb[1], wz = st.wb[2];
  const float wn = sqrtf(wx * wx + wy * wy + wz * wz);
  const float angle = wn * dt;
  if (angle >= 1e-12f) {
    float sh, ch;
    sincosf(0.5f * angle, &sh, &ch);
    const float k = sh / wn;
    const float dq[4] = {ch, k * wx, k * wy, k * wz};
    const float* q = st.quat;
    float r[4];
    r[0] = q[0] * dq[0] - q[1] * dq[1] - q[2] * dq[2] - q[3] * dq[3];
    r[1] = q[0] * dq[1] + q[1] * dq[0] + q[2] * dq[3] - q[3] * dq[2];
    r[2] = q[0] * dq[2] - q[1] * dq[3] + q[2] * dq[0] + q[3] * dq[1];
    r[3] = q[0] * dq[3] + q[1] * dq[2] - q[2] * dq[1] + q[3] * dq[0];
    quat_normalized(r, st.quat);
  }
}

// FK of the legs in extended precision, contacts; stores chain ends, foot
// wrenches and (last substep) the foot outputs.
template <class Scr>
G1_HD void fk_lower(const EnvState& st, const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr,
                    bool last_sub) {
#pragma unroll 1
  for (int c = 0; c < 2; ++c) fk_leg(st, c, io, ep, cfg, scr, last_sub);
}

// FK of the waist and the arms (one call site for the three chains);
// stores chain ends.
template <class Scr>
G1_HD void fk_upper(const EnvState& st, const StepConfig& cfg, Scr& scr) {
  FKNode base, torso;
  base_node(st, cfg, base);
#pragma unroll 1
  for (int c = 2; c < 5; ++c) {
    FKNode n = c == 2 ? base : torso;
    fk_chain<false>(chain_first(c), chain_last(c), n, scr);
    store_end(scr, c, n);
    if (c == 2) torso = n;
  }
}

// Backward pass of the arms into the torso and of the waist: the upper
// body's projection into the pelvis frame.
template <class Scr>
G1_HD void bwd_upper(const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr, AI& outI, SV& outP) {
  V3 w15, v15, g15;
  load_end(scr, 2, w15, v15, g15);
  AI acc15 = body_inertia(body(15));
  SV accP15 = bias_force(acc15, w15, v15, g15);
#pragma unroll 1
  for (int c = 3; c < 5; ++c) {
    V3 w, v, g;
    load_end(scr, c, w, v, g);
    const int last = chain_last(c);
    const AI IA = body_inertia(body(last));
    AI ci;
    SV cp;
    bwd_chain(chain_first(c), last, IA, bias_force(IA, w, v, g), w, v, g, ci, cp, io, ep, cfg, scr);
    ai_add(acc15, ci);
    sv_acc(accP15, cp);
  }
  bwd_chain(13, 15, acc15, accP15, w15, v15, g15, outI, outP, io, ep, cfg, scr);
}

// Backward pass of the legs into the pelvis accumulators (pelvis inertia and
// bias included).
template <class Scr>
G1_HD void bwd_lower(const EnvState& st, const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr,
                     AI& acc0, SV& accP0) {
  pelvis_acc(st, ep, cfg, acc0, accP0);
#pragma unroll 1
  for (int c = 0; c < 2; ++c) {
    AI ci;
    SV cp;
    bwd_leg(c, io, ep, cfg, scr, ci, cp);
    ai_add(acc0, ci);
    sv_acc(accP0, cp);
  }
}

// Forward pass of the legs, then the base integration (semi-implicit Euler;
// base qacc in MuJoCo's free-joint convention, world linear incl. w x v and
// body angular, reference src/g1_core.h:203-206,215-220).
template <class Scr>
G1_HD void fwd_lower_and_base(EnvState& st, const SV& a0, const StepConfig& cfg, Scr& scr) {
#pragma unroll 1
  for (int c = 0; c < 2; ++c) fwd_leg(st, c, a0, cfg, scr);
  integrate_base(st, a0, cfg);
}

// Forward pass of the waist and the arms (the base state is not touched).
template <class Scr>
G1_HD void fwd_upper(const EnvState& st, const SV& a0, const StepConfig& cfg, Scr& scr) {
  const float dt = cfg.dt;
  FKNode base;
  base_node(st, cfg, base);
  SV a = a0;
  V3 w = base.w, v = base.v;
  fwd_chain(13, 15, a, w, v, dt, scr);
  const SV a15 = a;
  const V3 w15 = w, v15 = v;
#pragma unroll 1
  for (int c = 3; c < 5; ++c) {
    a = a15;
    w = w15;
    v = v15;
    fwd_chain(chain_first(c), chain_last(c), a, w, v, dt, scr);
  }
}

// ------------------------------------- role-driven phases (split step)
// The backward and forward passes of either role of the two-thread split
// step through one call site each, so that one compiled copy of the chain
// routines serves both roles' warps (instruction fetch is the step's largest
// stall).  The arithmetic is that of bwd_lower / bwd_upper and
// fwd_lower_and_base / fwd_upper, in the same order.
// role 0: the legs into the pelvis accumulator (pelvis inertia and bias
// included); role 1: the arms into the torso, then the waist into the
// pelvis frame.
template <class Scr>
G1_HD void bwd_role(int role, const EnvState& st, const EnvIO& io, const EnvParams& ep, const StepConfig& cfg,
                    Scr& scr, AI& outI, SV& outP) {
  AI acc;
  SV accP;
  V3 w15, v15, g15;
  if (role == 0) {
    pelvis_acc(st, ep, cfg, acc, accP);
  } else {
    load_end(scr, 2, w15, v15, g15);
    acc = body_inertia(body(15));
    accP = bias_force(acc, w15, v15, g15);
  }
  const int nch = role == 0 ? 2 : 3;
#pragma unroll 1
  for (int k = 0; k < nch; ++k) {
    const int c = role == 0 ? k : (k < 2 ? 3 + k : 2);
    AI IA;
    SV pA;
    V3 w, v, g;
    if (c == 2) {
      IA = acc;
      pA = accP;
      w = w15;
      v = v15;
      g = g15;
    } else {
      load_end(scr, c, w, v, g);
      IA = body_inertia(body(chain_last(c)));
      pA = bias_force(IA, w, v, g);
      if (c < 2) sv_acc(pA, load_sv(scr, kSlotFoot + 6 * c));
    }
    AI ci;
    SV cp;
    bwd_chain(chain_first(c), chain_last(c), IA, pA, w, v, g, ci, cp, io, ep, cfg, scr);
    if (c == 2) {
      outI = ci;
      outP = cp;
    } else {
      ai_add(acc, ci);
      sv_acc(accP, cp);
    }
  }
  if (role == 0) {
    outI = acc;
    outP = accP;
  }
}

// role 0: the legs, then the base integration of st; role 1: the waist,
// then the arms from the torso (st untouched).
template <class Scr>
G1_HD void fwd_role(int role, EnvState& st, const SV& a0, const StepConfig& cfg, Scr& scr) {
  FKNode base;
  base_node(st, cfg, base);
  SV a15;
  V3 w15, v15;
  const int nch = role == 0 ? 2 : 3;
#pragma unroll 1
  for (int k = 0; k < nch; ++k) {
    const int c = role == 0 ? k : 2 + k;
    SV a = a0;
    V3 w = base.w, v = base.v;
    if (c > 2) {
      a = a15;
      w = w15;
      v = v15;
    }
    fwd_chain(chain_first(c), chain_last(c), a, w, v, cfg.dt, scr);
    if (c == 2) {
      a15 = a;
      w15 = w;
      v15 = v;
    }
  }
  if (role == 0) integrate_base(st, a0, cfg);
}

// One substep on one thread: FK -> contacts -> PD + ABA -> integrate
// (reference src/g1_core.h:225-232).  Joint angles / rates are read from and
// written back to the scratch.  With last_sub set, the foot kinematics of
// this substep's FK (before integration) and the contact normal forces are
// written to io's outputs.
template <class Scr>
G1_HD void step(EnvState& st, const EnvIO& io, const EnvParams& ep, const StepConfig& cfg, Scr& scr,
                bool last_sub) {
  fk_lower(st, io, ep, cfg, scr, last_sub);
  fk_upper(st, cfg, scr);
  AI up;
  SV upP;
  bwd_upper(io, ep, cfg, scr, up, upP);
  AI acc0;
  SV accP0;
  bwd_lower(st, io, ep, cfg, scr, acc0, accP0);
  ai_add(acc0, up);
  sv_acc(accP0, upP);
  const SV a0 = base_solve(acc0, accP0);
  fwd_upper(st, a0, cfg, scr);
  fwd_lower_and_base(st, a0, cfg, scr);
}

// Joint angles / rates between the SoA state arrays and the scratch, for the
// hinges of bodies first..last.
template <class Scr>
G1_HD void load_joints(const float* qpos, const float* qvel, size_t stride, Scr& scr, int first = 1,
                       int last = kNJ) {
#pragma unroll 1
  for (int i = first; i <= last; ++i) {
    scr.put(hslot(i, 0), qpos[(6 + i) * stride]);
    scr.put(hslot(i, 1), qvel[(5 + i) * stride]);
  }
}
template <class Scr>
G1_HD void store_joints(float* qpos, float* qvel, size_t stride, Scr& scr, int first = 1, int last = kNJ) {
#pragma unroll 1
  for (int i = first; i <= last; ++i) {
    qpos[(6 + i) * stride] = scr.get(hslot(i, 0));
    qvel[(5 + i) * stride] = scr.get(hslot(i, 1));
  }
}

}  // namespace g1b
