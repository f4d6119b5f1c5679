// sur_host.cpp -- the surrogate's feature and state-update functions of
// g1sim_b200/csrc/g1_surfeat.cuh compiled for the CPU in double (TEST
// INFRASTRUCTURE: tests/test_surrogate_derivation.py checks their
// vector-Jacobian products against central differences; the GPU tests
// compare the device features with these).
#include "../../g1sim_b200/csrc/g1_surfeat.cuh"

using namespace g1b;

namespace {
struct Arr {
  double* p;
  double get(int k) const { return p[k]; }
  void put(int k, double v) { p[k] = v; }
  void add(int k, double v) { p[k] += v; }
};
struct CArr {
  const double* p;
  double get(int k) const { return p[k]; }
};
}  // namespace

extern "C" {
int surh_nfeat() { return sur::kSurFeat; }
void surh_features_d(const double* x, const double* u, double mu, double dmass, double* f) {
  sur::features<double>(CArr{x}, CArr{u}, mu, dmass, f);
}
void surh_features_vjp_d(const double* x, const double* fb, double* xb, double* ub) {
  Arr xa{xb}, ua{ub};
  sur::features_vjp<double>(CArr{x}, fb, xa, ua);
}
void surh_integrate_d(double* x, const double* a, double dt) {
  Arr xa{x};
  sur::integrate<double>(xa, a, dt);
}
void surh_integrate_vjp_d(const double* x, const double* a, double dt, double* lam, double* ab) {
  Arr la{lam};
  sur::integrate_vjp<double>(CArr{x}, a, dt, la, ab);
}
}
