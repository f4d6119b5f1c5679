// g1_tangent.cuh -- the G1 step written once for any scalar type, so that
// one source gives the value step (float / double) and its forward-mode
// tangents (Dual<float, K> / Dual<double, K>: a value plus K directional
// derivatives carried through every operation).  The adjoint kernels
// (g1_adjoint.cuh) contract these tangents with the adjoint state to get the
// vector-Jacobian product of one step.
//
// The algorithm is the reference's generic tree walk, operation for
// operation:
//   FK + velocities          reference src/g1_core.h:29-54
//   contacts, PD, ABA        reference src/g1_core.h:109-207
//   semi-implicit Euler      reference src/g1_core.h:212-222
//   spatial algebra          reference src/spatial.h:22-278
// (not the structure-specialised FP32 kernel of g1_phys.cuh: the tangent
// step needs an implementation whose every branch and product is plain to
// differentiate).  Branches (contact touchdown, force clamps, stick / slip,
// soft limits, torque clamp) are taken on the value; the tangent follows the
// branch taken, i.e. the one-sided derivative at a switch.
//
// Model constants are copied at compile time from the generated tables into
// a __constant__ table per precision (float, double).
#pragma once
#include <math.h>

#include "g1_model_data.h"

namespace g1b::tg {

constexpr int kNB = G1M_NB, kNJ = G1M_NB - 1, kNQ = G1M_NQ, kNV = G1M_NV, kNU = G1M_NU, kNC = G1M_NC;
constexpr double kFree = 1e30;

// ------------------------------------------------------------ scalars
template <class R, int K>
struct Dual {
  R v;
  R d[K];
  __host__ __device__ Dual() {}
  __host__ __device__ Dual(R x) : v(x) {
#pragma unroll
    for (int i = 0; i < K; ++i) d[i] = R(0);
  }
};

template <class T>
struct Real {
  using type = T;
};
template <class R, int K>
struct Real<Dual<R, K>> {
  using type = R;
};
template <class T>
using real_t = typename Real<T>::type;

__host__ __device__ __forceinline__ float val(float x) { return x; }
__host__ __device__ __forceinline__ double val(double x) { return x; }
template <class R, int K>
__host__ __device__ __forceinline__ R val(const Dual<R, K>& x) {
  return x.v;
}

#define G1T_BIN(OP, DV)                                                                                  \
  template <class R, int K>                                                                              \
  __host__ __device__ __forceinline__ Dual<R, K> operator OP(const Dual<R, K>& a, const Dual<R, K>& b) { \
    Dual<R, K> r;                                                                                        \
    r.v = a.v OP b.v;                                                                                    \
    _Pragma("unroll") for (int i = 0; i < K; ++i) r.d[i] = DV;                                           \
    return r;                                                                                            \
  }
G1T_BIN(+, a.d[i] + b.d[i])
G1T_BIN(-, a.d[i] - b.d[i])
G1T_BIN(*, a.d[i] * b.v + a.v * b.d[i])
#undef G1T_BIN
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K> operator/(const Dual<R, K>& a, const Dual<R, K>& b) {
  Dual<R, K> r;
  const R inv = R(1) / b.v;
  r.v = a.v * inv;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
  return r;
}
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K> operator-(const Dual<R, K>& a) {
  Dual<R, K> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = -a.d[i];
  return r;
}
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K>& operator+=(Dual<R, K>& a, const Dual<R, K>& b) {
  a = a + b;
  return a;
}
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K>& operator-=(Dual<R, K>& a, const Dual<R, K>& b) {
  a = a - b;
  return a;
}
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K>& operator*=(Dual<R, K>& a, const Dual<R, K>& b) {
  a = a * b;
  return a;
}
// chain rule for f(x) with value fv and derivative dfv
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K> chain(const Dual<R, K>& x, R fv, R dfv) {
  Dual<R, K> r;
  r.v = fv;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = dfv * x.d[i];
  return r;
}
__host__ __device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }
__host__ __device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__host__ __device__ __forceinline__ float tsin(float x) { return sinf(x); }
__host__ __device__ __forceinline__ double tsin(double x) { return sin(x); }
__host__ __device__ __forceinline__ float tcos(float x) { return cosf(x); }
__host__ __device__ __forceinline__ double tcos(double x) { return cos(x); }
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K> tsqrt(const Dual<R, K>& x) {
  const R s = tsqrt(x.v);
  return chain(x, s, R(0.5) / s);
}
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K> tsin(const Dual<R, K>& x) {
  return chain(x, tsin(x.v), tcos(x.v));
}
template <class R, int K>
__host__ __device__ __forceinline__ Dual<R, K> tcos(const Dual<R, K>& x) {
  return chain(x, tcos(x.v), -tsin(x.v));
}

// ------------------------------------------------------------ model
constexpr double ce_sqrt(double x) {
  if (x <= 0) return 0;
  double r = x > 1 ? x : 1.0;
  for (int i = 0; i < 200; ++i) {
    const double n = 0.5 * (r + x / r);
    if (n == r) break;
    r = n;
  }
  return r;
}

template <class R>
struct BodyT {
  R RT[9];              // tree rotation (unit-normalised tree quaternion), row-major
  R tpos[3], ax[3], an[3];
  R mass, com[3], icom[9];
  R arm, damp, kp, kv, lim, lo, hi;  // hinge data (bodies 1..29)
  int parent;
};
template <class R>
struct ModelT {
  BodyT<R> b[kNB];
  int cbody[kNC];
  R cpos[3 * kNC];
  R radius;
};
template <class R>
constexpr ModelT<R> make_model_t() {
  ModelT<R> M{};
  for (int i = 0; i < kNB; ++i) {
    BodyT<R>& b = M.b[i];
    const double* q = g1m_tree_quat + 4 * i;
    const double n = ce_sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const double s = 1.0 / n;
    const double w = q[0] * s, x = q[1] * s, y = q[2] * s, z = q[3] * s;
    const double Rm[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z),     2 * (x * z + w * y),
                          2 * (x * y + w * z),     1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                          2 * (x * z - w * y),     2 * (y * z + w * x),     1 - 2 * (x * x + y * y)};
    for (int k = 0; k < 9; ++k) b.RT[k] = (R)Rm[k];
    for (int k = 0; k < 3; ++k) {
      b.tpos[k] = (R)g1m_tree_pos[3 * i + k];
      b.com[k] = (R)g1m_com[3 * i + k];
    }
    for (int k = 0; k < 9; ++k) b.icom[k] = (R)g1m_inertia_com[9 * i + k];
    b.mass = (R)g1m_mass[i];
    b.parent = g1m_parent[i];
    if (i > 0) {
      const int h = i - 1;
      for (int k = 0; k < 3; ++k) {
        b.ax[k] = (R)g1m_jnt_axis[3 * h + k];
        b.an[k] = (R)g1m_jnt_anchor[3 * h + k];
      }
      b.arm = (R)g1m_armature[h];
      b.damp = (R)g1m_damping[h];
      b.kp = (R)g1m_act_kp[h];
      b.kv = (R)g1m_act_kv[h];
      b.lim = (R)g1m_act_frclim[h];
      b.lo = (R)g1m_jnt_range[2 * h];
      b.hi = (R)g1m_jnt_range[2 * h + 1];
    }
  }
  for (int k = 0; k < kNC; ++k) M.cbody[k] = g1m_contact_body[k];
  for (int k = 0; k < 3 * kNC; ++k) M.cpos[k] = (R)g1m_contact_pos[k];
  M.radius = (R)g1m_contact_radius;
  return M;
}
static __constant__ ModelT<float> c_model_tf = make_model_t<float>();
static __constant__ ModelT<double> c_model_td = make_model_t<double>();
template <class R>
__device__ __forceinline__ const ModelT<R>& model_t();
template <>
__device__ __forceinline__ const ModelT<float>& model_t<float>() {
  return c_model_tf;
}
template <>
__device__ __forceinline__ const ModelT<double>& model_t<double>() {
  return c_model_td;
}

template <class R>
struct CfgT {
  R gravity_z, contact_kn, contact_dn, contact_kt, contact_dt, limit_kp, limit_kd, dt;
};

// ------------------------------------------------------------ algebra
template <class T>
struct V3 {
  T x, y, z;
};
template <class T>
struct M3 {
  T m[9];
};
template <class T>
struct SV {
  V3<T> a, l;
};
template <class T>
struct Se3 {
  M3<T> R;
  V3<T> p;
};
template <class T>
struct M6 {
  T m[21];
};

template <class T>
__device__ __forceinline__ V3<T> mk3(T x, T y, T z) {
  return V3<T>{x, y, z};
}
template <class T>
__device__ __forceinline__ V3<T> add3(const V3<T>& a, const V3<T>& b) {
  return mk3<T>(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <class T>
__device__ __forceinline__ V3<T> sub3(const V3<T>& a, const V3<T>& b) {
  return mk3<T>(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <class T>
__device__ __forceinline__ V3<T> scl3(const T& s, const V3<T>& a) {
  return mk3<T>(s * a.x, s * a.y, s * a.z);
}
template <class T>
__device__ __forceinline__ T dot3(const V3<T>& a, const V3<T>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class T>
__device__ __forceinline__ V3<T> crs3(const V3<T>& a, const V3<T>& b) {
  return mk3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class T, class R>
__device__ __forceinline__ V3<T> cst3(const R* p) {
  return mk3<T>(T(p[0]), T(p[1]), T(p[2]));
}
template <class T>
__device__ __forceinline__ V3<T> mv(const M3<T>& A, const V3<T>& v) {
  return mk3<T>(A.m[0] * v.x + A.m[1] * v.y + A.m[2] * v.z, A.m[3] * v.x + A.m[4] * v.y + A.m[5] * v.z,
                A.m[6] * v.x + A.m[7] * v.y + A.m[8] * v.z);
}
template <class T>
__device__ __forceinline__ V3<T> mtv(const M3<T>& A, const V3<T>& v) {
  return mk3<T>(A.m[0] * v.x + A.m[3] * v.y + A.m[6] * v.z, A.m[1] * v.x + A.m[4] * v.y + A.m[7] * v.z,
                A.m[2] * v.x + A.m[5] * v.y + A.m[8] * v.z);
}
template <class T>
__device__ __forceinline__ M3<T> mm(const M3<T>& A, const M3<T>& B) {
  M3<T> C;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      C.m[3 * i + j] = A.m[3 * i] * B.m[j] + A.m[3 * i + 1] * B.m[3 + j] + A.m[3 * i + 2] * B.m[6 + j];
  return C;
}
template <class T>
__device__ __forceinline__ M3<T> mmT(const M3<T>& A, const M3<T>& B) {
  M3<T> C;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      C.m[3 * i + j] =
          A.m[3 * i] * B.m[3 * j] + A.m[3 * i + 1] * B.m[3 * j + 1] + A.m[3 * i + 2] * B.m[3 * j + 2];
  return C;
}
template <class T>
__device__ __forceinline__ SV<T> mksv(const V3<T>& a, const V3<T>& l) {
  return SV<T>{a, l};
}
template <class T>
__device__ __forceinline__ SV<T> addsv(const SV<T>& u, const SV<T>& w) {
  return mksv(add3(u.a, w.a), add3(u.l, w.l));
}
template <class T>
__device__ __forceinline__ SV<T> subsv(const SV<T>& u, const SV<T>& w) {
  return mksv(sub3(u.a, w.a), sub3(u.l, w.l));
}
template <class T>
__device__ __forceinline__ SV<T> sclsv(const T& s, const SV<T>& u) {
  return mksv(scl3(s, u.a), scl3(s, u.l));
}
template <class T>
__device__ __forceinline__ T dotsv(const SV<T>& u, const SV<T>& w) {
  return dot3(u.a, w.a) + dot3(u.l, w.l);
}
template <class T>
__device__ __forceinline__ SV<T> mact_inv(const Se3<T>& X, const SV<T>& m) {
  return mksv(mtv(X.R, m.a), mtv(X.R, sub3(m.l, crs3(X.p, m.a))));
}
template <class T>
__device__ __forceinline__ SV<T> fact(const Se3<T>& X, const SV<T>& f) {
  const V3<T> l = mv(X.R, f.l);
  return mksv(add3(mv(X.R, f.a), crs3(X.p, l)), l);
}
template <class T>
__device__ __forceinline__ SV<T> crm(const SV<T>& v, const SV<T>& m) {
  return mksv(crs3(v.a, m.a), add3(crs3(v.a, m.l), crs3(v.l, m.a)));
}
template <class T>
__device__ __forceinline__ SV<T> crf(const SV<T>& v, const SV<T>& f) {
  return mksv(add3(crs3(v.a, f.a), crs3(v.l, f.l)), crs3(v.a, f.l));
}
// packed symmetric 6x6 (lower triangle, row-major): reference src/spatial.h:121-172
template <class T>
__device__ __forceinline__ SV<T> m6mul(const M6<T>& A, const SV<T>& u) {
  const T x[6] = {u.a.x, u.a.y, u.a.z, u.l.x, u.l.y, u.l.z};
  T y[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  int idx = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = 0; j < i; ++j) {
      const T Aij = A.m[idx++];
      y[i] += Aij * x[j];
      y[j] += Aij * x[i];
    }
    y[i] += A.m[idx++] * x[i];
  }
  return mksv(mk3<T>(y[0], y[1], y[2]), mk3<T>(y[3], y[4], y[5]));
}
template <class T>
__device__ __forceinline__ void m6subouter(M6<T>& A, const SV<T>& U, const T& invd) {
  const T u[6] = {U.a.x, U.a.y, U.a.z, U.l.x, U.l.y, U.l.z};
  int idx = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) A.m[idx++] -= u[i] * u[j] * invd;
}
// rigid-body spatial inertia about the body origin
template <class T, class R>
__device__ __forceinline__ M6<T> spin(R mass, const R* c, const R* Ic) {
  M6<T> I;
  const R cx[9] = {R(0), -c[2], c[1], c[2], R(0), -c[0], -c[1], c[0], R(0)};
  int idx = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      R v;
      if (i < 3 && j < 3) {
        R s = R(0);
        for (int k = 0; k < 3; ++k) s += cx[3 * i + k] * cx[3 * k + j];
        v = Ic[3 * i + j] - mass * s;
      } else if (i >= 3 && j < 3) {
        v = -mass * cx[3 * (i - 3) + j];
      } else {
        v = (i == j) ? mass : R(0);
      }
      I.m[idx++] = T(v);
    }
  }
  return I;
}
template <class T>
__device__ __forceinline__ M3<T> skew_mul(const V3<T>& p, const M3<T>& A) {  // (p x) A
  M3<T> C;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    C.m[j] = p.y * A.m[6 + j] - p.z * A.m[3 + j];
    C.m[3 + j] = p.z * A.m[j] - p.x * A.m[6 + j];
    C.m[6 + j] = p.x * A.m[3 + j] - p.y * A.m[j];
  }
  return C;
}
template <class T>
__device__ __forceinline__ M3<T> mul_skew(const M3<T>& A, const V3<T>& p) {  // A (p x)
  M3<T> C;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    C.m[3 * i] = A.m[3 * i + 1] * p.z - A.m[3 * i + 2] * p.y;
    C.m[3 * i + 1] = A.m[3 * i + 2] * p.x - A.m[3 * i] * p.z;
    C.m[3 * i + 2] = A.m[3 * i] * p.y - A.m[3 * i + 1] * p.x;
  }
  return C;
}
// P += X I X^T (child articulated inertia into the parent frame), by blocks:
// reference src/spatial.h:174-251
template <class T>
__device__ void psum_transform(M6<T>& P, const M6<T>& I, const Se3<T>& X) {
  const M3<T> J = {{I.m[0], I.m[1], I.m[3], I.m[1], I.m[2], I.m[4], I.m[3], I.m[4], I.m[5]}};
  const M3<T> H = {{I.m[6], I.m[10], I.m[15], I.m[7], I.m[11], I.m[16], I.m[8], I.m[12], I.m[17]}};
  const M3<T> Mb = {{I.m[9], I.m[13], I.m[18], I.m[13], I.m[14], I.m[19], I.m[18], I.m[19], I.m[20]}};
  M3<T> t = mm(X.R, J);
  const M3<T> tJ = mmT(t, X.R);
  t = mm(X.R, H);
  const M3<T> tH = mmT(t, X.R);
  t = mm(X.R, Mb);
  const M3<T> tM = mmT(t, X.R);
  const M3<T> pxM = skew_mul(X.p, tM);
  M3<T> HA, tHT;
#pragma unroll
  for (int i = 0; i < 9; ++i) HA.m[i] = tH.m[i] + pxM.m[i];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) tHT.m[3 * i + j] = tH.m[3 * j + i];
  const M3<T> pxHT = skew_mul(X.p, tHT);
  const M3<T> HApx = mul_skew(HA, X.p);
  M3<T> JA;
#pragma unroll
  for (int i = 0; i < 9; ++i) JA.m[i] = tJ.m[i] + pxHT.m[i] - HApx.m[i];
  P.m[0] += JA.m[0];
  P.m[1] += JA.m[3];
  P.m[2] += JA.m[4];
  P.m[3] += JA.m[6];
  P.m[4] += JA.m[7];
  P.m[5] += JA.m[8];
  P.m[6] += HA.m[0];
  P.m[7] += HA.m[3];
  P.m[8] += HA.m[6];
  P.m[10] += HA.m[1];
  P.m[11] += HA.m[4];
  P.m[12] += HA.m[7];
  P.m[15] += HA.m[2];
  P.m[16] += HA.m[5];
  P.m[17] += HA.m[8];
  P.m[9] += tM.m[0];
  P.m[13] += tM.m[3];
  P.m[14] += tM.m[4];
  P.m[18] += tM.m[6];
  P.m[19] += tM.m[7];
  P.m[20] += tM.m[8];
}
// SPD 6x6 solve by Cholesky: reference src/spatial.h:254-278
template <class T>
__device__ SV<T> m6solve(const M6<T>& A, const SV<T>& b) {
  M6<T> L = A;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const int jj = j * (j + 1) / 2 + j;
#pragma unroll
    for (int k = 0; k < j; ++k) L.m[jj] -= L.m[j * (j + 1) / 2 + k] * L.m[j * (j + 1) / 2 + k];
    L.m[jj] = tsqrt(L.m[jj]);
    const T inv = T(real_t<T>(1)) / L.m[jj];
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
      const int ij = i * (i + 1) / 2 + j;
#pragma unroll
      for (int k = 0; k < j; ++k) L.m[ij] -= L.m[i * (i + 1) / 2 + k] * L.m[j * (j + 1) / 2 + k];
      L.m[ij] *= inv;
    }
  }
  T y[6] = {b.a.x, b.a.y, b.a.z, b.l.x, b.l.y, b.l.z};
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int k = 0; k < i; ++k) y[i] -= L.m[i * (i + 1) / 2 + k] * y[k];
    y[i] = y[i] / L.m[i * (i + 1) / 2 + i];
  }
#pragma unroll
  for (int i = 5; i >= 0; --i) {
#pragma unroll
    for (int k = i + 1; k < 6; ++k) y[i] -= L.m[k * (k + 1) / 2 + i] * y[k];
    y[i] = y[i] / L.m[i * (i + 1) / 2 + i];
  }
  return mksv(mk3<T>(y[0], y[1], y[2]), mk3<T>(y[3], y[4], y[5]));
}

// ------------------------------------------------------------ the step
template <class T>
struct Work {
  Se3<T> liMi[kNB];
  M3<T> oR[kNB];
  V3<T> oP[kNB];
  SV<T> v[kNB];
  M6<T> IA[kNB];
  SV<T> pA[kNB];
  SV<T> U[kNJ];
  T D[kNJ], u[kNJ];
  SV<T> a[kNB];
};

template <class T>
__device__ __forceinline__ SV<T> hinge_S(const BodyT<real_t<T>>& b) {
  const V3<T> ax = cst3<T>(b.ax), an = cst3<T>(b.an);
  return mksv(ax, crs3(an, ax));
}

// One substep in place on (qpos[36], qvel[35], anchor[16]) with PD targets
// ctrl[29]; kp_scale / kd_scale multiply every servo gain; mu and dmass as
// in the value kernels.
template <class T>
__device__ void step(const CfgT<real_t<T>>& cfg, T* qpos, T* qvel, T* anchor, const T* ctrl, const T& kp_scale,
                     const T& kd_scale, real_t<T> mu, real_t<T> dmass, Work<T>& w) {
  using R = real_t<T>;
  const ModelT<R>& M = model_t<R>();
  // ---- FK + velocities: reference src/g1_core.h:29-54
  {
    T qw = qpos[3], qx = qpos[4], qy = qpos[5], qz = qpos[6];
    const T s = T(R(1)) / tsqrt(qw * qw + qx * qx + qy * qy + qz * qz);
    qw = qw * s;
    qx = qx * s;
    qy = qy * s;
    qz = qz * s;
    const T one = T(R(1)), two = T(R(2));
    M3<T>& Rb = w.liMi[0].R;
    Rb.m[0] = one - two * (qy * qy + qz * qz);
    Rb.m[1] = two * (qx * qy - qw * qz);
    Rb.m[2] = two * (qx * qz + qw * qy);
    Rb.m[3] = two * (qx * qy + qw * qz);
    Rb.m[4] = one - two * (qx * qx + qz * qz);
    Rb.m[5] = two * (qy * qz - qw * qx);
    Rb.m[6] = two * (qx * qz - qw * qy);
    Rb.m[7] = two * (qy * qz + qw * qx);
    Rb.m[8] = one - two * (qx * qx + qy * qy);
    w.liMi[0].p = mk3<T>(qpos[0], qpos[1], qpos[2]);
    w.oR[0] = Rb;
    w.oP[0] = w.liMi[0].p;
    w.v[0] = mksv(mk3<T>(qvel[3], qvel[4], qvel[5]), mtv(Rb, mk3<T>(qvel[0], qvel[1], qvel[2])));
  }
#pragma unroll 1
  for (int i = 1; i < kNB; ++i) {
    const BodyT<R>& b = M.b[i];
    const int h = i - 1, par = b.parent;
    const T q = qpos[7 + h], qd = qvel[6 + h];
    // Rodrigues, reference src/spatial.h:63-70
    const T c = tcos(q), s = tsin(q), t = T(R(1)) - c;
    const T ax = T(b.ax[0]), ay = T(b.ax[1]), az = T(b.ax[2]);
    M3<T> RJ;
    RJ.m[0] = c + t * ax * ax;
    RJ.m[1] = t * ax * ay - s * az;
    RJ.m[2] = t * ax * az + s * ay;
    RJ.m[3] = t * ax * ay + s * az;
    RJ.m[4] = c + t * ay * ay;
    RJ.m[5] = t * ay * az - s * ax;
    RJ.m[6] = t * ax * az - s * ay;
    RJ.m[7] = t * ay * az + s * ax;
    RJ.m[8] = c + t * az * az;
    M3<T> RT;
#pragma unroll
    for (int k = 0; k < 9; ++k) RT.m[k] = T(b.RT[k]);
    const V3<T> an = cst3<T>(b.an);
    w.liMi[i].R = mm(RT, RJ);
    w.liMi[i].p = add3(mv(RT, sub3(an, mv(RJ, an))), cst3<T>(b.tpos));
    w.oR[i] = mm(w.oR[par], w.liMi[i].R);
    w.oP[i] = add3(mv(w.oR[par], w.liMi[i].p), w.oP[par]);
    w.v[i] = addsv(mact_inv(w.liMi[i], w.v[par]), sclsv(qd, hinge_S<T>(b)));
  }
  // ---- bias forces: reference src/g1_core.h:113-120
#pragma unroll 1
  for (int i = 0; i < kNB; ++i) {
    const BodyT<R>& b = M.b[i];
    const R m = b.mass + (i == 0 ? dmass : R(0));
    w.IA[i] = spin<T, R>(m, b.com, b.icom);
    const V3<T> gb = mtv(w.oR[i], mk3<T>(T(R(0)), T(R(0)), T(cfg.gravity_z)));
    const V3<T> fg = scl3(T(m), gb);
    const SV<T> f = mksv(crs3(cst3<T>(b.com), fg), fg);
    w.pA[i] = subsv(crf(w.v[i], m6mul(w.IA[i], w.v[i])), f);
  }
  // ---- contacts: reference src/g1_core.h:123-153
#pragma unroll 1
  for (int k = 0; k < kNC; ++k) {
    const int bi = M.cbody[k];
    const V3<T> r = cst3<T>(M.cpos + 3 * k);
    const V3<T> p = add3(mv(w.oR[bi], r), w.oP[bi]);
    const T depth = T(M.radius) - p.z;
    if (val(depth) > R(0)) {
      const V3<T> vp = mv(w.oR[bi], add3(w.v[bi].l, crs3(w.v[bi].a, r)));
      T fn = T(cfg.contact_kn) * depth - T(cfg.contact_dn) * vp.z;
      if (val(fn) < R(0)) fn = T(R(0));
      if (val(fn) > R(500)) fn = T(R(500));
      if (val(anchor[2 * k]) >= R(kFree)) {
        anchor[2 * k] = p.x;
        anchor[2 * k + 1] = p.y;
      }
      T ftx = -T(cfg.contact_kt) * (p.x - anchor[2 * k]) - T(cfg.contact_dt) * vp.x;
      T fty = -T(cfg.contact_kt) * (p.y - anchor[2 * k + 1]) - T(cfg.contact_dt) * vp.y;
      const T ftn = tsqrt(ftx * ftx + fty * fty), fmax = T(mu) * fn;
      if (val(ftn) > val(fmax)) {
        const T sc = fmax / (ftn + T(R(1e-12)));
        ftx = ftx * sc;
        fty = fty * sc;
        anchor[2 * k] = p.x + ftx / T(cfg.contact_kt);
        anchor[2 * k + 1] = p.y + fty / T(cfg.contact_kt);
      }
      const V3<T> fb = mtv(w.oR[bi], mk3<T>(ftx, fty, fn));
      w.pA[bi] = subsv(w.pA[bi], mksv(crs3(r, fb), fb));
    } else {
      anchor[2 * k] = T(R(kFree));
      anchor[2 * k + 1] = T(R(kFree));
    }
  }
  // ---- backward with PD servos, soft limits, implicit damping: reference src/g1_core.h:156-186
#pragma unroll 1
  for (int i = kNB - 1; i >= 1; --i) {
    const BodyT<R>& b = M.b[i];
    const int h = i - 1, par = b.parent;
    const T qd = qvel[6 + h], q = qpos[7 + h];
    const SV<T> Sh = hinge_S<T>(b);
    w.U[h] = m6mul(w.IA[i], Sh);
    const T kp = T(b.kp) * kp_scale, kv = T(b.kv) * kd_scale;
    T t = kp * (ctrl[h] - q) - kv * qd;
    if (val(t) > b.lim) t = T(b.lim);
    if (val(t) < -b.lim) t = T(-b.lim);
    T bd = kv + T(b.damp);
    if (val(q) < b.lo) {
      t = t + T(cfg.limit_kp) * (T(b.lo) - q) - T(cfg.limit_kd) * qd;
      bd = bd + T(cfg.limit_kd);
    }
    if (val(q) > b.hi) {
      t = t + T(cfg.limit_kp) * (T(b.hi) - q) - T(cfg.limit_kd) * qd;
      bd = bd + T(cfg.limit_kd);
    }
    w.D[h] = dotsv(Sh, w.U[h]) + T(b.arm) + T(cfg.dt) * bd;
    w.u[h] = t - T(b.damp) * qd - dotsv(Sh, w.pA[i]);
    const T invd = T(R(1)) / w.D[h];
    const SV<T> c = crm(w.v[i], sclsv(qd, Sh));
    M6<T> Ia = w.IA[i];
    m6subouter(Ia, w.U[h], invd);
    const SV<T> pa = addsv(addsv(w.pA[i], m6mul(Ia, c)), sclsv(w.u[h] * invd, w.U[h]));
    psum_transform(w.IA[par], Ia, w.liMi[i]);
    w.pA[par] = addsv(w.pA[par], fact(w.liMi[i], pa));
  }
  // ---- base solve and forward pass: reference src/g1_core.h:188-206
  T qacc[kNV];
  const SV<T> zero = mksv(mk3<T>(T(R(0)), T(R(0)), T(R(0))), mk3<T>(T(R(0)), T(R(0)), T(R(0))));
  w.a[0] = m6solve(w.IA[0], subsv(zero, w.pA[0]));
#pragma unroll 1
  for (int i = 1; i < kNB; ++i) {
    const BodyT<R>& b = M.b[i];
    const int h = i - 1, par = b.parent;
    const SV<T> Sh = hinge_S<T>(b);
    const SV<T> c = crm(w.v[i], sclsv(qvel[6 + h], Sh));
    const SV<T> ap = addsv(mact_inv(w.liMi[i], w.a[par]), c);
    const T qdd = (w.u[h] - dotsv(w.U[h], ap)) / w.D[h];
    w.a[i] = addsv(ap, sclsv(qdd, Sh));
    qacc[6 + h] = qdd;
  }
  {
    const V3<T> aw = w.a[0].a;
    const V3<T> al = mv(w.oR[0], add3(w.a[0].l, crs3(w.v[0].a, w.v[0].l)));
    qacc[0] = al.x;
    qacc[1] = al.y;
    qacc[2] = al.z;
    qacc[3] = aw.x;
    qacc[4] = aw.y;
    qacc[5] = aw.z;
  }
  // ---- semi-implicit Euler: reference src/g1_core.h:212-222
  const T dt = T(cfg.dt);
#pragma unroll 1
  for (int i = 0; i < kNV; ++i) qvel[i] = qvel[i] + dt * qacc[i];
  qpos[0] = qpos[0] + dt * qvel[0];
  qpos[1] = qpos[1] + dt * qvel[1];
  qpos[2] = qpos[2] + dt * qvel[2];
  {
    // q <- q (x) exp(w dt / 2), body-frame w: reference src/spatial.h:73-79
    const V3<T> wv = mk3<T>(qvel[3], qvel[4], qvel[5]);
    const T wn = tsqrt(dot3(wv, wv));
    const T angle = wn * dt;
    if (val(angle) >= R(1e-12)) {
      const T half = angle * T(R(0.5));
      const T s = tsin(half) / wn;
      const T dw = tcos(half), dx = s * wv.x, dy = s * wv.y, dz = s * wv.z;
      const T aw = qpos[3], ax = qpos[4], ay = qpos[5], az = qpos[6];
      T rw = aw * dw - ax * dx - ay * dy - az * dz;
      T rx = aw * dx + ax * dw + ay * dz - az * dy;
      T ry = aw * dy - ax * dz + ay * dw + az * dx;
      T rz = aw * dz + ax * dy - ay * dx + az * dw;
      const T inv = T(R(1)) / tsqrt(rw * rw + rx * rx + ry * ry + rz * rz);
      qpos[3] = rw * inv;
      qpos[4] = rx * inv;
      qpos[5] = ry * inv;
      qpos[6] = rz * inv;
    }
  }
#pragma unroll 1
  for (int h = 0; h < kNJ; ++h) qpos[7 + h] = qpos[7 + h] + dt * qvel[6 + h];
}

}  // namespace g1b::tg
