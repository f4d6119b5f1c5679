#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

Needs the reference builds of oracle/Makefile target ``ref`` (compiled from
the reference sources, which exist only in the development container):
  oracle/_ref/libg1host.so      reference src/host_lib.cpp, G1_PRECISION=8
  oracle/_ref/libg1cuda_cpu.so  reference src/g1_kernel.cu kernels through its
                                fake-CUDA shim (FP32, GPU ABI semantics)
Writes:
  ref_host.npz     FK / smooth-FD / step / quaternion / settling vectors (FP64)
  ref_gpu_abi.npz  reset_done outputs (float32, bit-exact target) and FP32
                   g1_cuda_step outputs at the ABI's fixed dt = 1 ms
The random states follow the reference tests' generator
(tests/test_vs_mujoco.py:23-30: rng seed 0, base in U(-1,1), random unit
quaternion, joints in the inner 80% of their range, qvel U(-2,2)).

Run:  make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import NB, NC, NQ, NU, NV, RefHost, RefKernelCPU  # noqa: E402

from g1sim_b200.model import g1_model_data as M  # noqa: E402
from g1sim_b200 import workloads  # noqa: E402

RANGE = np.asarray(M.jnt_range)
STAND = np.asarray(M.qpos_stand)


def random_state(rng):
    qpos = np.zeros(NQ)
    qpos[:3] = rng.uniform(-1, 1, 3)
    q = rng.normal(size=4)
    qpos[3:7] = q / np.linalg.norm(q)
    lo, hi = RANGE[:, 0], RANGE[:, 1]
    qpos[7:] = rng.uniform(lo + 0.1 * (hi - lo), hi - 0.1 * (hi - lo))
    qvel = rng.uniform(-2, 2, NV)
    return qpos, qvel


def host_vectors(ref):
    rng = np.random.default_rng(0)
    out = {}
    # forward kinematics, 20 states
    fk_q, fk_x, fk_r = [], [], []
    for _ in range(20):
        qpos, _ = random_state(rng)
        x, r = ref.fk(qpos)
        fk_q.append(qpos); fk_x.append(x); fk_r.append(r)
    out.update(fk_qpos=np.array(fk_q), fk_xpos=np.array(fk_x), fk_xmat=np.array(fk_r))
    # smooth forward dynamics, 20 states, tau U(-30, 30)
    fd = {k: [] for k in ("qpos", "qvel", "tau", "qacc")}
    for _ in range(20):
        qpos, qvel = random_state(rng)
        tau = rng.uniform(-30, 30, NV)
        fd["qpos"].append(qpos); fd["qvel"].append(qvel); fd["tau"].append(tau)
        fd["qacc"].append(ref.fd(qpos, qvel, tau))
    out.update({"fd_" + k: np.array(v) for k, v in fd.items()})

    # one-step cases from drop-test-like states, at dt 2 ms, with contacts:
    # each case is stepped a number of warm-up substeps first so that anchors,
    # stick and slip states are populated, then one recorded step.
    w = workloads.drop_test(nenv=24, seed=1)
    cases = {k: [] for k in ("qpos0", "qvel0", "anchor0", "ctrl", "nsub", "dt",
                             "qpos1", "qvel1", "anchor1", "fn")}
    for e in range(24):
        qp = w["qpos"][:, e].copy(); qv = w["qvel"][:, e].copy()
        an = w["anchor"][:, e].copy(); ct = w["ctrl"][:, e].copy()
        warm = [0, 10, 20, 25, 30, 40, 60, 100][e % 8]
        if e >= 16:  # push some joints past their limits (soft-limit branch)
            qp[7 + (e % NU)] = RANGE[e % NU, 1] + 0.05
            qp[7 + ((e + 7) % NU)] = RANGE[(e + 7) % NU, 0] - 0.05
        if warm:
            ref.c_step(qp, qv, ct, warm, 2e-3, an)
        nsub = 1 if e % 3 else 5
        cases["qpos0"].append(qp.copy()); cases["qvel0"].append(qv.copy())
        cases["anchor0"].append(an.copy()); cases["ctrl"].append(ct.copy())
        cases["nsub"].append(nsub); cases["dt"].append(2e-3)
        fn = ref.c_step(qp, qv, ct, nsub, 2e-3, an)
        cases["qpos1"].append(qp); cases["qvel1"].append(qv)
        cases["anchor1"].append(an); cases["fn"].append(fn)
    out.update({"step_" + k: np.array(v) for k, v in cases.items()})

    # drop-test trajectory, one env, 250 steps at 2 ms, every 10th state
    qp = w["qpos"][:, 0].copy(); qv = w["qvel"][:, 0].copy()
    an = w["anchor"][:, 0].copy(); ct = w["ctrl"][:, 0].copy()
    out.update(traj_qpos0=qp.copy(), traj_qvel0=qv.copy(), traj_ctrl=ct.copy())
    tq, tv = [], []
    for s in range(250):
        ref.c_step(qp, qv, ct, 1, 2e-3, an)
        if (s + 1) % 10 == 0:
            tq.append(qp.copy()); tv.append(qv.copy())
    out.update(traj_qpos=np.array(tq), traj_qvel=np.array(tv))

    # quaternion integration (reference tests/test_vs_mujoco.py:102-112 state)
    quat = np.array([0.3, -0.5, 0.7, 0.4]); quat /= np.linalg.norm(quat)
    qp = np.zeros(NQ); qv = np.zeros(NV)
    qp[3:7] = quat; qp[2] = 5.0; qv[3:6] = [1.3, -2.1, 0.7]
    an = np.full(2 * NC, 1e30)
    out.update(quat_qpos0=qp.copy(), quat_qvel0=qv.copy())
    ref.c_step(qp, qv, np.zeros(NU), 1, 0.01, an)
    out.update(quat_qpos1=qp.copy(), quat_qvel1=qv.copy())

    # contact settling (reference tests/test_vs_mujoco.py:114-133): 10 s at 2 ms
    qp = STAND.copy(); qp[2] += 0.02
    qv = np.zeros(NV); ct = STAND[7:].copy(); an = np.full(2 * NC, 1e30)
    for _ in range(5000):
        fn = ref.c_step(qp, qv, ct, 1, 2e-3, an)
    out.update(settle_qpos=qp, settle_qvel=qv, settle_anchor=an, settle_fn=fn)
    return out


def gpu_abi_vectors(rk):
    out = {}
    n = 300
    rng = np.random.default_rng(7)
    qp = rng.normal(size=(NQ, n)).astype(np.float32)
    qv = rng.normal(size=(NV, n)).astype(np.float32)
    an = rng.normal(size=(2 * NC, n)).astype(np.float32)
    done = (rng.uniform(size=n) < 0.6).astype(np.uint8)
    out.update(reset_qpos_in=qp.copy(), reset_qvel_in=qv.copy(), reset_anchor_in=an.copy(),
               reset_done=done)
    rk.reset_done(qp, qv, an, done, 42, 0.05, 0.02)
    out.update(reset_qpos=qp.copy(), reset_qvel=qv.copy(), reset_anchor=an.copy())
    qp2 = qp.copy(); qv2 = qv.copy(); an2 = an.copy()
    rk.reset_done(qp2, qv2, an2, np.ones(n, np.uint8), 1234, 0.1, 1.0)
    out.update(reset2_qpos=qp2)

    # FP32 g1_cuda_step at the ABI's dt = 1 ms: drop-test states, 20 substeps
    w = workloads.drop_test(nenv=64, seed=3)
    qp = w["qpos"].astype(np.float32); qv = w["qvel"].astype(np.float32)
    an = w["anchor"].astype(np.float32); ct = w["ctrl"].astype(np.float32)
    out.update(step_qpos0=qp.copy(), step_qvel0=qv.copy(), step_anchor0=an.copy(), step_ctrl=ct)
    fp, fv, cf = rk.step(20, qp, qv, an, ct)
    out.update(step_qpos1=qp, step_qvel1=qv, step_anchor1=an, step_foot_pos=fp,
               step_foot_vel=fv, step_contact_forces=cf)
    return out


def main():
    ref = RefHost(8)
    prec, sizes = ref.sizes()
    assert prec == 8 and sizes == (NB, NQ, NV, NU, NC), (prec, sizes)
    np.savez_compressed(os.path.join(HERE, "ref_host.npz"), **host_vectors(ref))
    np.savez_compressed(os.path.join(HERE, "ref_gpu_abi.npz"), **gpu_abi_vectors(RefKernelCPU()))
    for f in ("ref_host.npz", "ref_gpu_abi.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
