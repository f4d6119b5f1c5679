"""The hand-derived reverse pass of the G1 substep, checked on the CPU.

g1sim_b200/csrc/g1_adj.cuh (the adjoint kernels' step and its
vector-Jacobian product) is compiled for the host in double and float
(tests/native/adj_host.cpp) and checked, with no GPU:

  * its primal against the FP64 oracle's step (same model, different
    operation order): 1e-12 relative;
  * its vector-Jacobian product against central differences of its own
    primal in double (h = 1e-7), for random output adjoints, with respect to
    all 87 state entries, the 29 targets and the two gain scales, on states
    chosen so that every branch of the step is taken somewhere: standing
    contact with stuck anchors, slipping feet, fresh anchors at touchdown,
    the 500 N normal-force clamp, saturated servo torques, both soft joint
    limits, and flight: 1e-6 relative to the largest entry of each product;
  * the float build's product against the double build's: 2e-4 relative in
    2-norm (FP32 rounding of a 30-body recursion; measured up to 2.5e-5).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from g1sim_b200 import workloads
from g1sim_b200.model import g1_model_data as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "adj_host.cpp")
HDR = os.path.join(ROOT, "g1sim_b200", "csrc", "g1_adj.cuh")
LIB = os.path.join(ROOT, "tests", "native", "_build", "libg1adjhost.so")

CFG = np.array([-9.81, 2e4, 280.0, 1e4, 280.0, 200.0, 5.0, 2e-3])
NS = 87
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


@pytest.fixture(scope="module")
def host():
    deps = [SRC, HDR, os.path.join(ROOT, "g1sim_b200", "csrc", "g1_model_derived.h"),
            os.path.join(ROOT, "g1sim_b200", "csrc", "g1_model_data.h")]
    if not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++20", "-fPIC", "-shared", "-o", LIB, SRC], check=True)
    L = C.CDLL(LIB)
    L.adjh_step_d.argtypes = [_dp, _dp, _dp, _dp]
    L.adjh_vjp_d.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp]
    L.adjh_vjp_f.argtypes = [_fp, _fp, _dp, _dp, _fp, _fp, _fp]
    L.adjh_flags_d.argtypes = [_dp, _dp, _dp, _dp, _ip, _ip]
    assert L.adjh_state_size() == NS
    return L


class Step:
    def __init__(self, L, par):
        self.L, self.par = L, np.asarray(par, dtype=np.float64)

    def __call__(self, x, u, par=None):
        x = np.array(x, dtype=np.float64)
        self.L.adjh_step_d(_p(x), _p(np.ascontiguousarray(u, dtype=np.float64)), _p(CFG),
                           _p(self.par if par is None else np.asarray(par, dtype=np.float64)))
        return x

    def vjp(self, x, u, lam):
        lam = np.array(lam, dtype=np.float64)
        ub, kb = np.zeros(29), np.zeros(2)
        self.L.adjh_vjp_d(_p(np.ascontiguousarray(x, dtype=np.float64)), _p(np.ascontiguousarray(u, dtype=np.float64)),
                          _p(CFG), _p(self.par), _p(lam), _p(ub), _p(kb))
        return lam, ub, kb

    def vjp_f(self, x, u, lam):
        lam = np.array(lam, dtype=np.float32)
        ub, kb = np.zeros(29, np.float32), np.zeros(2, np.float32)
        self.L.adjh_vjp_f(_p(np.ascontiguousarray(x, dtype=np.float32), _fp),
                          _p(np.ascontiguousarray(u, dtype=np.float32), _fp), _p(CFG), _p(self.par),
                          _p(lam, _fp), _p(ub, _fp), _p(kb, _fp))
        return lam.astype(np.float64), ub.astype(np.float64), kb.astype(np.float64)

    def flags(self, x, u):
        f, h = np.zeros(2, np.int32), np.zeros(29, np.int32)
        self.L.adjh_flags_d(_p(np.ascontiguousarray(x, dtype=np.float64)), _p(np.ascontiguousarray(u, dtype=np.float64)),
                            _p(CFG), _p(self.par), _p(f, _ip), _p(h, _ip))
        return f, h


def settled_states(oracle, n=6, steps=200, seed=1, par=(0.8, 0.5, 1.1, 0.9)):
    """Drop-test envs after `steps` oracle substeps: standing on stuck anchors."""
    w = workloads.drop_test(nenv=n, seed=seed)
    q, v, a = w["qpos"].copy(), w["qvel"].copy(), w["anchor"].copy()
    kw = {k: np.full(n, val) for k, val in zip(("mu", "dmass", "kp_scale", "kd_scale"), par)}
    oracle.step_soa(steps, oracle.config(dt=2e-3), q, v, a, w["ctrl"], outputs=False, **kw)
    return [(np.concatenate([q[:, e], v[:, e], a[:, e]]), w["ctrl"][:, e].copy()) for e in range(n)]


def cases(oracle):
    base = settled_states(oracle)
    out = [("stand", *base[0]), ("stand2", *base[1])]
    x, u = base[2]
    xs = x.copy()
    xs[36] += 0.6  # base sliding forward: feet slip
    xs[37] -= 0.3
    out.append(("slip", xs, u))
    x, u = base[3]
    xf = x.copy()
    xf[71:] = 1e30  # touchdown: every penetrating sphere takes a fresh anchor
    out.append(("fresh", xf, u))
    x, u = base[4]
    xd = x.copy()
    xd[2] -= 0.035  # deep: normal forces past the 500 N clamp
    out.append(("deep", xd, u))
    x, u = base[5]
    xc = x.copy()
    uc = u.copy()
    uc[[0, 3, 12, 15, 22]] += np.array([1.5, -1.2, 2.0, 1.4, -1.7])  # saturated servo torques
    lo, hi = np.asarray(M.jnt_range)[:, 0], np.asarray(M.jnt_range)[:, 1]
    xc[7 + 4] = lo[4] - 0.04  # below the lower limit
    xc[7 + 19] = hi[19] + 0.03  # above the upper limit
    out.append(("clamp+limits", xc, uc))
    xa = base[0][0].copy()
    xa[2] += 0.3
    xa[71:] = 1e30
    xa[36:71] += np.random.default_rng(3).normal(0, 0.5, 35)
    out.append(("flight", xa, base[0][1]))
    return out


PAR = (0.8, 0.5, 1.1, 0.9)


@pytest.fixture(scope="module")
def all_cases(oracle):
    return cases(oracle)


def test_primal_matches_oracle(host, oracle, all_cases):
    st = Step(host, PAR)
    ocfg = oracle.config(dt=2e-3)
    for name, x, u in all_cases:
        q, v, a = x[:36, None].copy(), x[36:71, None].copy(), x[71:, None].copy()
        oracle.step_soa(1, ocfg, q, v, a, u[:, None], mu=np.array([PAR[0]]), dmass=np.array([PAR[1]]),
                        kp_scale=np.array([PAR[2]]), kd_scale=np.array([PAR[3]]), outputs=False)
        xo = np.concatenate([q[:, 0], v[:, 0], a[:, 0]])
        xs = st(x, u)
        fin = np.abs(xo) < 1e29
        assert np.array_equal(fin, np.abs(xs) < 1e29), name
        err = (np.abs(xs - xo) / np.maximum(np.abs(xo), 1))[fin].max()
        assert err < 1e-12, (name, err)


def test_every_branch_is_covered(host, all_cases):
    st = Step(host, PAR)
    seen = set()
    for name, x, u in all_cases:
        f, h = st.flags(x, u)
        for ff in f:
            for j in range(4):
                b = (ff >> (4 * j)) & 15
                if b & 1:
                    seen.add("contact")
                    seen.add("fresh" if b & 2 else "stuck")
                    seen.add("slip" if b & 4 else "stick")
                    seen.add("fn linear" if b & 8 else "fn clamped")
                else:
                    seen.add("airborne")
        seen.update("torque clamp" for hh in h if hh & 1)
        seen.update("lower limit" for hh in h if hh & 2)
        seen.update("upper limit" for hh in h if hh & 4)
    want = {"contact", "fresh", "stuck", "slip", "stick", "fn linear", "fn clamped", "airborne", "torque clamp",
            "lower limit", "upper limit"}
    assert want <= seen, want - seen


def _fd(st, x, u, lam, h=1e-7):
    fin_in = np.abs(x) < 1e29
    f = lambda xx, uu, pp=None: float(lam @ np.where(np.abs(st(xx, uu, pp)) < 1e29, st(xx, uu, pp), 0.0))  # noqa
    gx = np.zeros(NS)
    for i in np.nonzero(fin_in)[0]:
        d = np.zeros(NS)
        d[i] = h
        gx[i] = (f(x + d, u) - f(x - d, u)) / (2 * h)
    gu = np.zeros(29)
    for j in range(29):
        d = np.zeros(29)
        d[j] = h
        gu[j] = (f(x, u + d) - f(x, u - d)) / (2 * h)
    gk = []
    for k in (2, 3):
        pp, pm = np.array(PAR, dtype=float), np.array(PAR, dtype=float)
        pp[k] += h
        pm[k] -= h
        gk.append((f(x, u, pp) - f(x, u, pm)) / (2 * h))
    return gx, gu, np.array(gk)


def test_vjp_matches_central_differences(host, all_cases):
    st = Step(host, PAR)
    rng = np.random.default_rng(11)
    for name, x, u in all_cases:
        xo = st(x, u)
        for _ in range(2):
            lam = rng.normal(size=NS)
            lam[np.abs(xo) > 1e29] = 0.0  # free anchors carry no adjoint
            gx, gu, gk = st.vjp(x, u, lam)
            fx, fu, fk = _fd(st, x, u, lam)
            fin = np.abs(x) < 1e29
            gx = np.where(fin, gx, 0.0)
            for got, ref, what in ((gx, fx, "state"), (gu, fu, "targets"), (gk, fk, "gains")):
                err = np.abs(got - ref).max() / (np.abs(ref).max() + 1e-12)
                assert err < 1e-6, (name, what, err)


def test_float_build_agrees_with_double(host, all_cases):
    st = Step(host, PAR)
    rng = np.random.default_rng(5)
    for name, x, u in all_cases:
        lam = rng.normal(size=NS)
        lam[np.abs(st(x, u)) > 1e29] = 0.0
        gd, ud, kd = st.vjp(x, u, lam)
        gf, uf, kf = st.vjp_f(x, u, lam)
        fin = np.abs(x) < 1e29
        for a, b, what in ((gf[fin], gd[fin], "state"), (uf, ud, "targets"), (kf, kd, "gains")):
            err = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-12)
            assert err < 2e-4, (name, what, err)
