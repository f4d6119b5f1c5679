"""The surrogate's feature and state-update products, checked on the CPU.

g1sim_b200/csrc/g1_surfeat.cuh (the input features of the dynamics
surrogate -- including the foot spheres' depth, anchor offset and velocity
from the legs' forward kinematics -- and its semi-implicit Euler update) is
compiled for the host in double (tests/native/sur_host.cpp); the
vector-Jacobian products that the surrogate's gradient kernels use are
checked against central differences (h = 1e-6) of the functions themselves,
for random adjoints, on standing states with stuck and free anchors and
random base and joint velocities: 1e-7 relative to the largest entry.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from g1sim_b200 import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "sur_host.cpp")
LIB = os.path.join(ROOT, "tests", "native", "_build", "libg1surhost.so")
_dp = C.POINTER(C.c_double)


def _p(a):
    return np.ascontiguousarray(a).ctypes.data_as(_dp)


@pytest.fixture(scope="module")
def host():
    csrc = os.path.join(ROOT, "g1sim_b200", "csrc")
    deps = [SRC] + [os.path.join(csrc, f) for f in ("g1_surfeat.cuh", "g1_adj.cuh", "g1_model_derived.h",
                                                    "g1_model_data.h")]
    if not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++20", "-fPIC", "-shared", "-o", LIB, SRC], check=True)
    L = C.CDLL(LIB)
    L.surh_features_d.argtypes = [_dp, _dp, C.c_double, C.c_double, _dp]
    L.surh_features_vjp_d.argtypes = [_dp] * 4
    L.surh_integrate_d.argtypes = [_dp, _dp, C.c_double]
    L.surh_integrate_vjp_d.argtypes = [_dp, _dp, C.c_double, _dp, _dp]
    assert L.surh_nfeat() == 159
    return L


def states(oracle, n=6):
    w = workloads.drop_test(nenv=n, seed=1)
    q, v, a = w["qpos"].copy(), w["qvel"].copy(), w["anchor"].copy()
    oracle.step_soa(200, oracle.config(dt=2e-3), q, v, a, w["ctrl"], outputs=False)
    rng = np.random.default_rng(0)
    out = []
    for e in range(n):
        x = np.concatenate([q[:, e], v[:, e], a[:, e]])
        x[36:71] += rng.normal(0, 0.3, 35)
        if e == n - 1:
            x[71:] = 1e30  # free anchors: their offset features vanish
        out.append((x, w["ctrl"][:, e].copy()))
    return out


def test_features_vjp_matches_central_differences(host, oracle):
    rng = np.random.default_rng(1)

    def feat(x, u):
        f = np.zeros(159)
        host.surh_features_d(_p(x), _p(u), 0.8, 0.5, f.ctypes.data_as(_dp))
        return f

    for x, u in states(oracle):
        fb = rng.normal(size=159)
        xb, ub = np.zeros(87), np.zeros(29)
        host.surh_features_vjp_d(_p(x), _p(fb), xb.ctypes.data_as(_dp), ub.ctypes.data_as(_dp))
        h = 1e-6
        fd = np.zeros(87)
        for i in np.nonzero(x < 1e29)[0]:
            d = np.zeros(87)
            d[i] = h
            fd[i] = (fb @ feat(x + d, u) - fb @ feat(x - d, u)) / (2 * h)
        fdu = np.array([(fb @ feat(x, u + h * np.eye(29)[j]) - fb @ feat(x, u - h * np.eye(29)[j])) / (2 * h)
                        for j in range(29)])
        assert np.abs(xb - fd).max() < 1e-7 * np.abs(fd).max()
        assert np.abs(ub - fdu).max() < 1e-7 * np.abs(fdu).max()


def test_integrate_vjp_matches_central_differences(host, oracle):
    rng = np.random.default_rng(2)

    def integ(x, a):
        x = np.array(x)
        host.surh_integrate_d(x.ctypes.data_as(_dp), _p(a), 2e-3)
        return x

    for x, _ in states(oracle):
        a = rng.normal(size=35) * 10
        lam = rng.normal(size=87)
        lam[71:] = 0.0
        la, ab = lam.copy(), np.zeros(35)
        host.surh_integrate_vjp_d(_p(x), _p(a), 2e-3, la.ctypes.data_as(_dp), ab.ctypes.data_as(_dp))
        h = 1e-6
        fdx = np.array([(lam @ integ(x + h * np.eye(87)[i], a) - lam @ integ(x - h * np.eye(87)[i], a)) / (2 * h)
                        if x[i] < 1e29 else 0.0 for i in range(87)])
        fda = np.array([(lam @ integ(x, a + h * np.eye(35)[i]) - lam @ integ(x, a - h * np.eye(35)[i])) / (2 * h)
                        for i in range(35)])
        la[71:] = 0.0
        assert np.abs(la - fdx).max() < 1e-7 * np.abs(fdx).max()
        assert np.abs(ab - fda).max() < 1e-6 * np.abs(fda).max()
