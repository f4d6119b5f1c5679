// adj_host.cpp -- the adjoint step of g1sim_b200/csrc/g1_adj.cuh compiled
// for the CPU (TEST INFRASTRUCTURE: tests/test_adjoint_derivation.py checks
// the hand-derived reverse pass against central differences of its own
// primal in double, and the primal against the FP64 oracle).  Nothing in
// the library uses this build.
#include "../../g1sim_b200/csrc/g1_adj.cuh"

using namespace g1b::adj;

namespace {
template <class R>
struct ArrX {
  R* p;
  R get(int k) const { return p[k]; }
  void put(int k, R v) { p[k] = v; }
};
template <class R>
struct ArrU {
  const R* p;
  R get(int k) const { return p[k]; }
};
template <class R>
struct ArrW {
  R* p;
  void put(int k, R v) { p[k] = v; }
};
template <class R>
Cfg<R> cfg_of(const double* c) {
  return Cfg<R>{(R)c[0], (R)c[1], (R)c[2], (R)c[3], (R)c[4], (R)c[5], (R)c[6], (R)c[7]};
}
template <class R>
Par<R> par_of(const double* p) {
  return Par<R>{(R)p[0], (R)p[1], (R)p[2], (R)p[3]};
}
template <class R>
Base<R> base_of(const R* x) {
  Base<R> b;
  for (int k = 0; k < 3; ++k) b.pos[k] = x[k];
  for (int k = 0; k < 4; ++k) b.quat[k] = x[3 + k];
  for (int k = 0; k < 3; ++k) b.vw[k] = x[kQV + k];
  for (int k = 0; k < 3; ++k) b.wb[k] = x[kQV + 3 + k];
  return b;
}
template <class R>
void step(R* x, const R* u, const double* c, const double* p) {
  static thread_local R tape[kTapeSlots];
  Tape<R, 1> tp{tape};
  Base<R> b = base_of(x);
  ArrX<R> xa{x};
  ArrU<R> ua{u};
  primal<true>(b, xa, ua, par_of<R>(p), cfg_of<R>(c), tp);
  for (int k = 0; k < 3; ++k) x[k] = b.pos[k];
  for (int k = 0; k < 4; ++k) x[3 + k] = b.quat[k];
  for (int k = 0; k < 3; ++k) x[kQV + k] = b.vw[k];
  for (int k = 0; k < 3; ++k) x[kQV + 3 + k] = b.wb[k];
}
template <class R>
void vjp(const R* x, const R* u, const double* c, const double* p, R* lam, R* ubar, R* kb) {
  static thread_local R tape[kTapeSlots];
  Tape<R, 1> tp{tape};
  R xc[kState];
  for (int k = 0; k < kState; ++k) xc[k] = x[k];
  Base<R> b = base_of(xc);
  ArrX<R> xa{xc};
  ArrU<R> ua{u};
  ArrX<R> la{lam};
  ArrW<R> ub{ubar};
  const Par<R> par = par_of<R>(p);
  const Cfg<R> cfg = cfg_of<R>(c);
  primal<false>(b, xa, ua, par, cfg, tp);
  R kpb = 0, kdb = 0;
  reverse(b, xa, ua, la, ub, par, cfg, kpb, kdb, tp);
  kb[0] = kpb;
  kb[1] = kdb;
}
// Branch record of the primal: per foot its sphere flags, per hinge its
// servo flags (as the tape holds them).
template <class R>
void flags(const R* x, const R* u, const double* c, const double* p, int* foot2, int* hinge29) {
  static thread_local R tape[kTapeSlots];
  Tape<R, 1> tp{tape};
  R xc[kState];
  for (int k = 0; k < kState; ++k) xc[k] = x[k];
  Base<R> b = base_of(xc);
  ArrX<R> xa{xc};
  ArrU<R> ua{u};
  primal<false>(b, xa, ua, par_of<R>(p), cfg_of<R>(c), tp);
  for (int f = 0; f < 2; ++f) foot2[f] = (int)tp.get(tf(f, kFflag));
  for (int i = 1; i <= kNJ; ++i) hinge29[i - 1] = (int)tp.get(th(i, kHflag));
}
}  // namespace

extern "C" {
void adjh_flags_d(const double* x, const double* u, const double* cfg, const double* par, int* foot2, int* hinge29) {
  flags<double>(x, u, cfg, par, foot2, hinge29);
}
int adjh_state_size() { return kState; }
int adjh_tape_slots() { return kTapeSlots; }
void adjh_step_d(double* x, const double* u, const double* cfg, const double* par) { step<double>(x, u, cfg, par); }
void adjh_step_f(float* x, const float* u, const double* cfg, const double* par) { step<float>(x, u, cfg, par); }
void adjh_vjp_d(const double* x, const double* u, const double* cfg, const double* par, double* lam, double* ubar,
                double* kb) {
  vjp<double>(x, u, cfg, par, lam, ubar, kb);
}
void adjh_vjp_f(const float* x, const float* u, const double* cfg, const double* par, float* lam, float* ubar,
                float* kb) {
  vjp<float>(x, u, cfg, par, lam, ubar, kb);
}
}
