// g1_surfeat.cuh -- the dynamics surrogate's input features and state
// update, with their vector-Jacobian products, for any real type R (host
// and device, so that the products can be checked on the CPU).
//
// Features of one env (159 used of kSurIn):
//   0-28   joint angles q            29-57  joint rates qd
//   58     base height               59-64  first two columns of the base rotation
//   65-67  base linear velocity in the base frame    68-70  base angular velocity
//   71-126 per foot sphere k (7 each): penetration depth (radius - z),
//          in-contact flag, offset of the sphere from its anchor (x, y; 0
//          while the anchor is free), world velocity of the sphere (3)
//   127-155 PD targets                156 friction   157 base-mass offset   158 constant 1
// The sphere terms come from the legs' forward kinematics (the step's own
// FK, reference src/g1_core.h:29-54 and the contact geometry of
// src/g1_core.h:123-153): they are the inputs of the contact model, so the
// network maps them to forces without having to learn the kinematics.
//
// State update (the step's semi-implicit Euler, reference
// src/g1_core.h:212-222, from the predicted qacc): qvel += dt qacc, base
// position += dt v, quaternion q (x) exp(w dt / 2) renormalised, hinge
// angles += dt qd.  Anchors are not updated by the surrogate.
#pragma once
#include "g1_adj.cuh"

namespace g1b::sur {

using adj::add_outer;
using adj::at;
using adj::body;
using adj::BodyA;
using adj::cat;
using adj::cross;
using adj::dot_scross;
using adj::frc_out;
using adj::kNC;
using adj::kNQ;
using adj::kNU;
using adj::kNV;
using adj::M3;
using adj::model;
using adj::ModelA;
using adj::mot_in;
using adj::mul;
using adj::mulT;
using adj::pvec;
using adj::rotAT;
using adj::SV;
using adj::sv;
using adj::sv0;
using adj::V3;
using adj::v3;
using adj::zero3;
constexpr int kSurFeat = 159;
constexpr int kSurIn = 192;  // padded input width (a multiple of the GEMM's 64-column K chunk)
constexpr int kFS = 71;      // first sphere feature
constexpr int kFU = kFS + 7 * kNC;

template <class R>
struct LegNode {
  R c, s;
  adj::V3<R> w, v;  // body twist
  adj::M3<R> Rw;    // world rotation
  adj::V3<R> Pw;    // world position
};

// FK of one hinge of a leg: twist and world pose from the parent's.
template <int AX, class R>
GA_HD void leg_body(int i, R q, R qd, const LegNode<R>& p, LegNode<R>& n) {
  const BodyA<R>& b = body<R>(i);
  n.s = sin(q);
  n.c = cos(q);
  const SV<R> m = mot_in<AX>(b, sv(p.w, p.v), n.c, n.s);
  n.w = m.w;
  at(n.w, AX) += qd;
  n.v = m.l;
  n.Pw = p.Pw + mul(p.Rw, pvec(b));
  M3<R> E;
  for (int a = 0; a < 3; ++a) {
    const V3<R> row = rotAT<AX>(v3(b.ident ? R(a == 0) : b.T[3 * a], b.ident ? R(a == 1) : b.T[3 * a + 1],
                                   b.ident ? R(a == 2) : b.T[3 * a + 2]),
                                n.c, n.s);
    E.m[3 * a] = row.x;
    E.m[3 * a + 1] = row.y;
    E.m[3 * a + 2] = row.z;
  }
  for (int r = 0; r < 3; ++r)
    for (int cc = 0; cc < 3; ++cc)
      n.Rw.m[3 * r + cc] = p.Rw.m[3 * r] * E.m[cc] + p.Rw.m[3 * r + 1] * E.m[3 + cc] + p.Rw.m[3 * r + 2] * E.m[6 + cc];
}

// Base frame of the state: unit quaternion, its norm, rotation, body twist.
template <class R, class X>
GA_HD void base_node(const X& x, R* qn, R& qnorm, LegNode<R>& b0) {
  adj::Base<R> st;
  for (int k = 0; k < 4; ++k) st.quat[k] = x.get(3 + k);
  adj::base_frame(st, qn, qnorm, b0.Rw);
  b0.w = adj::v3(x.get(kNQ + 3), x.get(kNQ + 4), x.get(kNQ + 5));
  b0.v = adj::mulT(b0.Rw, adj::v3(x.get(kNQ), x.get(kNQ + 1), x.get(kNQ + 2)));
  b0.Pw = adj::v3(x.get(0), x.get(1), x.get(2));
  b0.c = R(1);
  b0.s = R(0);
}

// The six bodies of leg f (bodies 6 f + 1 .. 6 f + 6) from the base node.
template <class R, class X>
GA_HD void leg_fk(int f, const X& x, const LegNode<R>& b0, LegNode<R>* nodes) {
  const LegNode<R>* p = &b0;
  for (int j = 0; j < 6; ++j) {
    const int i = 6 * f + 1 + j;
    const R q = x.get(6 + i), qd = x.get(kNQ + 5 + i);
    switch (adj::body<R>(i).axis) {
      case 0: leg_body<0>(i, q, qd, *p, nodes[j]); break;
      case 1: leg_body<1>(i, q, qd, *p, nodes[j]); break;
      default: leg_body<2>(i, q, qd, *p, nodes[j]); break;
    }
    p = &nodes[j];
  }
}

// Features f[0 .. kSurFeat) of one env.  x: the 87 state entries (qpos,
// qvel, anchors), u: the 29 targets.
template <class R, class X, class U>
GA_HD void features(const X& x, const U& u, R mu, R dmass, R* f) {
  for (int j = 0; j < kNU; ++j) f[j] = x.get(7 + j);
  for (int j = 0; j < kNU; ++j) f[29 + j] = x.get(kNQ + 6 + j);
  f[58] = x.get(2);
  R qn[4], qnorm;
  LegNode<R> b0;
  base_node(x, qn, qnorm, b0);
  const M3<R>& R0 = b0.Rw;
  f[59] = R0.m[0];
  f[60] = R0.m[3];
  f[61] = R0.m[6];
  f[62] = R0.m[1];
  f[63] = R0.m[4];
  f[64] = R0.m[7];
  f[65] = b0.v.x;
  f[66] = b0.v.y;
  f[67] = b0.v.z;
  f[68] = b0.w.x;
  f[69] = b0.w.y;
  f[70] = b0.w.z;
  const ModelA<R>& M = model<R>();
  for (int ff = 0; ff < 2; ++ff) {
    LegNode<R> nodes[6];
    leg_fk(ff, x, b0, nodes);
    const LegNode<R>& n = nodes[5];
    for (int jj = 0; jj < 4; ++jj) {
      const int k = 4 * ff + jj;
      const V3<R> r = v3(M.cpos[3 * k], M.cpos[3 * k + 1], M.cpos[3 * k + 2]);
      const V3<R> pc = n.Pw + mul(n.Rw, r);
      const V3<R> vp = mul(n.Rw, n.v + cross(n.w, r));
      const R depth = M.radius - pc.z;
      const R ax = x.get(adj::kAN + 2 * k), ay = x.get(adj::kAN + 2 * k + 1);
      const bool stuck = ax < R(1e29);
      R* g = f + kFS + 7 * k;
      g[0] = depth;
      g[1] = depth > R(0) ? R(1) : R(0);
      g[2] = stuck ? pc.x - ax : R(0);
      g[3] = stuck ? pc.y - ay : R(0);
      g[4] = vp.x;
      g[5] = vp.y;
      g[6] = vp.z;
    }
  }
  for (int j = 0; j < kNU; ++j) f[kFU + j] = u.get(j);
  f[156] = mu;
  f[157] = dmass;
  f[158] = R(1);
}

// Reverse of one leg hinge: twist and world-pose adjoints of body i move
// to the parent; the hinge's angle and rate adjoints are returned.
template <int AX, class R>
GA_HD void leg_body_rev(int i, const LegNode<R>& n, adj::SV<R>& Vb, adj::M3<R>& Rb, adj::V3<R>& Pb, R& qb, R& qdb) {
  constexpr int i1 = (AX + 1) % 3, i2 = (AX + 2) % 3;
  const BodyA<R>& b = body<R>(i);
  qdb += cat(Vb.w, AX);
  qb -= dot_scross<AX>(Vb, sv(n.w, n.v));
  Vb = frc_out<AX>(b, Vb, n.c, n.s);
  for (int a = 0; a < 3; ++a) qb += Rb.m[3 * a + i1] * n.Rw.m[3 * a + i2] - Rb.m[3 * a + i2] * n.Rw.m[3 * a + i1];
  M3<R> E;
  for (int a = 0; a < 3; ++a) {
    const V3<R> row = rotAT<AX>(v3(b.ident ? R(a == 0) : b.T[3 * a], b.ident ? R(a == 1) : b.T[3 * a + 1],
                                   b.ident ? R(a == 2) : b.T[3 * a + 2]),
                                n.c, n.s);
    E.m[3 * a] = row.x;
    E.m[3 * a + 1] = row.y;
    E.m[3 * a + 2] = row.z;
  }
  M3<R> Rp;
  for (int r = 0; r < 3; ++r)
    for (int cc = 0; cc < 3; ++cc)
      Rp.m[3 * r + cc] = Rb.m[3 * r] * E.m[3 * cc] + Rb.m[3 * r + 1] * E.m[3 * cc + 1] + Rb.m[3 * r + 2] * E.m[3 * cc + 2];
  add_outer(Rp, Pb, pvec(b));
  Rb = Rp;
}

// Adjoints of the base rotation R(q / |q|) moved to the stored quaternion.
template <class R>
GA_HD void rot_to_quat(const adj::M3<R>& G, const R* qn, R qnorm, R* qb) {
  const R w = qn[0], xq = qn[1], y = qn[2], zq = qn[3];
  R a[4];
  a[0] = R(2) * (-zq * G.m[1] + y * G.m[2] + zq * G.m[3] - xq * G.m[5] - y * G.m[6] + xq * G.m[7]);
  a[1] = R(2) * (y * G.m[1] + zq * G.m[2] + y * G.m[3] - R(2) * xq * G.m[4] - w * G.m[5] + zq * G.m[6] + w * G.m[7] -
                 R(2) * xq * G.m[8]);
  a[2] = R(2) * (-R(2) * y * G.m[0] + xq * G.m[1] + w * G.m[2] + xq * G.m[3] + zq * G.m[5] - w * G.m[6] + zq * G.m[7] -
                 R(2) * y * G.m[8]);
  a[3] = R(2) * (-R(2) * zq * G.m[0] - w * G.m[1] + xq * G.m[2] + w * G.m[3] - R(2) * zq * G.m[4] + y * G.m[5] +
                 xq * G.m[6] + y * G.m[7]);
  const R od = qn[0] * a[0] + qn[1] * a[1] + qn[2] * a[2] + qn[3] * a[3];
  for (int j = 0; j < 4; ++j) qb[j] += (a[j] - qn[j] * od) / qnorm;
}

// xb (87, accumulated) and ub (29, accumulated) from the feature adjoint fb.
// The flags, friction, mass offset and constant carry no gradient; the
// anchors receive the adjoint of the offsets.
template <class R, class X, class XB, class UB>
GA_HD void features_vjp(const X& x, const R* fb, XB& xb, UB& ub) {
  for (int j = 0; j < kNU; ++j) xb.add(7 + j, fb[j]);
  for (int j = 0; j < kNU; ++j) xb.add(kNQ + 6 + j, fb[29 + j]);
  xb.add(2, fb[58]);
  for (int j = 0; j < kNU; ++j) ub.add(j, fb[kFU + j]);
  R qn[4], qnorm;
  LegNode<R> b0;
  base_node(x, qn, qnorm, b0);
  M3<R> R0b;
  for (int k = 0; k < 9; ++k) R0b.m[k] = R(0);
  R0b.m[0] += fb[59];
  R0b.m[3] += fb[60];
  R0b.m[6] += fb[61];
  R0b.m[1] += fb[62];
  R0b.m[4] += fb[63];
  R0b.m[7] += fb[64];
  V3<R> v0b = v3(fb[65], fb[66], fb[67]);
  V3<R> w0b = v3(fb[68], fb[69], fb[70]);
  V3<R> posb = zero3<R>();
  const ModelA<R>& M = model<R>();
  for (int ff = 0; ff < 2; ++ff) {
    LegNode<R> nodes[6];
    leg_fk(ff, x, b0, nodes);
    const LegNode<R>& n = nodes[5];
    SV<R> Vb = sv0<R>();
    M3<R> Rb;
    for (int k = 0; k < 9; ++k) Rb.m[k] = R(0);
    V3<R> Pb = zero3<R>();
    for (int jj = 0; jj < 4; ++jj) {
      const int k = 4 * ff + jj;
      const V3<R> r = v3(M.cpos[3 * k], M.cpos[3 * k + 1], M.cpos[3 * k + 2]);
      const R* g = fb + kFS + 7 * k;
      const bool stuck = x.get(adj::kAN + 2 * k) < R(1e29);
      V3<R> pcb = v3(stuck ? g[2] : R(0), stuck ? g[3] : R(0), -g[0]);
      if (stuck) {
        xb.add(adj::kAN + 2 * k, -g[2]);
        xb.add(adj::kAN + 2 * k + 1, -g[3]);
      }
      const V3<R> vpb = v3(g[4], g[5], g[6]);
      // pc = P + R r ; vp = R (v + w x r)
      Pb += pcb;
      add_outer(Rb, pcb, r);
      const V3<R> vb = mulT(n.Rw, vpb);
      Vb.l += vb;
      Vb.w += cross(r, vb);
      add_outer(Rb, vpb, n.v + cross(n.w, r));
    }
    for (int j = 5; j >= 0; --j) {
      const int i = 6 * ff + 1 + j;
      R qb = R(0), qdb = R(0);
      switch (body<R>(i).axis) {
        case 0: leg_body_rev<0>(i, nodes[j], Vb, Rb, Pb, qb, qdb); break;
        case 1: leg_body_rev<1>(i, nodes[j], Vb, Rb, Pb, qb, qdb); break;
        default: leg_body_rev<2>(i, nodes[j], Vb, Rb, Pb, qb, qdb); break;
      }
      xb.add(6 + i, qb);
      xb.add(kNQ + 5 + i, qdb);
    }
    // base node: twist (wb, R0^T vw), world pose (R0, pos)
    w0b += Vb.w;
    v0b += Vb.l;
    for (int k = 0; k < 9; ++k) R0b.m[k] += Rb.m[k];
    posb += Pb;
  }
  const V3<R> vw = v3(x.get(kNQ), x.get(kNQ + 1), x.get(kNQ + 2));
  const V3<R> vwb = mul(b0.Rw, v0b);
  add_outer(R0b, vw, v0b);
  xb.add(0, posb.x);
  xb.add(1, posb.y);
  xb.add(2, posb.z);
  xb.add(kNQ, vwb.x);
  xb.add(kNQ + 1, vwb.y);
  xb.add(kNQ + 2, vwb.z);
  xb.add(kNQ + 3, w0b.x);
  xb.add(kNQ + 4, w0b.y);
  xb.add(kNQ + 5, w0b.z);
  R qb[4] = {R(0), R(0), R(0), R(0)};
  rot_to_quat(R0b, qn, qnorm, qb);
  for (int j = 0; j < 4; ++j) xb.add(3 + j, qb[j]);
}

// ----------------------------------------------------------- state update
// In place on the state x (qpos, qvel; anchors untouched) from qacc a[35].
template <class R, class X>
GA_HD void integrate(X& x, const R* a, R dt) {
  for (int i = 0; i < kNV; ++i) x.put(kNQ + i, x.get(kNQ + i) + dt * a[i]);
  for (int i = 0; i < 3; ++i) x.put(i, x.get(i) + dt * x.get(kNQ + i));
  const R wx = x.get(kNQ + 3), wy = x.get(kNQ + 4), wz = x.get(kNQ + 5);
  const R wn = sqrt(wx * wx + wy * wy + wz * wz);
  if (wn * dt >= R(1e-12)) {
    const R sh = sin(R(0.5) * wn * dt), ch = cos(R(0.5) * wn * dt);
    const R k = sh / wn;
    const R d[4] = {ch, k * wx, k * wy, k * wz};
    const R q[4] = {x.get(3), x.get(4), x.get(5), x.get(6)};
    R r[4];
    r[0] = q[0] * d[0] - q[1] * d[1] - q[2] * d[2] - q[3] * d[3];
    r[1] = q[0] * d[1] + q[1] * d[0] + q[2] * d[3] - q[3] * d[2];
    r[2] = q[0] * d[2] - q[1] * d[3] + q[2] * d[0] + q[3] * d[1];
    r[3] = q[0] * d[3] + q[1] * d[2] - q[2] * d[1] + q[3] * d[0];
    const R n = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
    for (int j = 0; j < 4; ++j) x.put(3 + j, r[j] / n);
  }
  for (int h = 0; h < kNU; ++h) x.put(7 + h, x.get(7 + h) + dt * x.get(kNQ + 6 + h));
}

// Reverse of integrate at the state x before the update: lam holds the
// adjoint of the updated state on entry (qpos, qvel entries) and the
// adjoint of x through the update on return; ab (35) gets the adjoint of
// qacc.
template <class R, class X, class L>
GA_HD void integrate_vjp(const X& x, const R* a, R dt, L& lam, R* ab) {
  // rates after the update
  R v1[kNV];
  for (int i = 0; i < kNV; ++i) v1[i] = x.get(kNQ + i) + dt * a[i];
  R v1b[kNV];
  for (int i = 0; i < kNV; ++i) v1b[i] = lam.get(kNQ + i);
  for (int h = 0; h < kNU; ++h) v1b[6 + h] += dt * lam.get(7 + h);  // q' = q + dt qd'
  for (int i = 0; i < 3; ++i) v1b[i] += dt * lam.get(i);            // pos' = pos + dt v'
  const R wx = v1[3], wy = v1[4], wz = v1[5];
  const R wn = sqrt(wx * wx + wy * wy + wz * wz);
  R quatb[4] = {lam.get(3), lam.get(4), lam.get(5), lam.get(6)};
  if (wn * dt >= R(1e-12)) {
    const R h = R(0.5) * dt, xx = wn * h;
    const R sh = sin(xx), ch = cos(xx);
    const R k = sh / wn;
    const R d[4] = {ch, k * wx, k * wy, k * wz};
    const R q[4] = {x.get(3), x.get(4), x.get(5), x.get(6)};
    R r[4];
    r[0] = q[0] * d[0] - q[1] * d[1] - q[2] * d[2] - q[3] * d[3];
    r[1] = q[0] * d[1] + q[1] * d[0] + q[2] * d[3] - q[3] * d[2];
    r[2] = q[0] * d[2] - q[1] * d[3] + q[2] * d[0] + q[3] * d[1];
    r[3] = q[0] * d[3] + q[1] * d[2] - q[2] * d[1] + q[3] * d[0];
    const R rn = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
    R o[4], rb[4];
    for (int j = 0; j < 4; ++j) o[j] = r[j] / rn;
    const R od = o[0] * quatb[0] + o[1] * quatb[1] + o[2] * quatb[2] + o[3] * quatb[3];
    for (int j = 0; j < 4; ++j) rb[j] = (quatb[j] - o[j] * od) / rn;
    quatb[0] = rb[0] * d[0] + rb[1] * d[1] + rb[2] * d[2] + rb[3] * d[3];
    quatb[1] = -rb[0] * d[1] + rb[1] * d[0] - rb[2] * d[3] + rb[3] * d[2];
    quatb[2] = -rb[0] * d[2] + rb[1] * d[3] + rb[2] * d[0] - rb[3] * d[1];
    quatb[3] = -rb[0] * d[3] - rb[1] * d[2] + rb[2] * d[1] + rb[3] * d[0];
    R db[4];
    db[0] = rb[0] * q[0] + rb[1] * q[1] + rb[2] * q[2] + rb[3] * q[3];
    db[1] = -rb[0] * q[1] + rb[1] * q[0] + rb[2] * q[3] - rb[3] * q[2];
    db[2] = -rb[0] * q[2] - rb[1] * q[3] + rb[2] * q[0] + rb[3] * q[1];
    db[3] = -rb[0] * q[3] + rb[1] * q[2] - rb[2] * q[1] + rb[3] * q[0];
    R sinc, fx;
    if (xx < R(0.25)) {
      const R x2 = xx * xx;
      sinc = R(1) - x2 / R(6) + x2 * x2 / R(120) - x2 * x2 * x2 / R(5040);
      fx = -R(1) / R(3) + x2 / R(30) - x2 * x2 / R(840) + x2 * x2 * x2 / R(45360);
    } else {
      sinc = sh / xx;
      fx = (xx * ch - sh) / (xx * xx * xx);
    }
    const R wd = wx * db[1] + wy * db[2] + wz * db[3];
    const R cw = -h * h * sinc * db[0] + h * h * h * fx * wd;
    v1b[3] += cw * wx + h * sinc * db[1];
    v1b[4] += cw * wy + h * sinc * db[2];
    v1b[5] += cw * wz + h * sinc * db[3];
  }
  for (int i = 0; i < kNV; ++i) {
    ab[i] = dt * v1b[i];
    lam.put(kNQ + i, v1b[i]);
  }
  for (int j = 0; j < 4; ++j) lam.put(3 + j, quatb[j]);
  // pos, hinge angles: identity (their adjoints stay as they are)
}

}  // namespace g1b::sur
