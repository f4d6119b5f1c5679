"""Seeded synthetic inputs for the G1 step workloads (host-side numpy).

Shapes follow the reference's SoA convention, array[i, e] with the env axis
fastest (reference src/g1_kernel.cu:9-10, src/g1sim.py:46-53).  All arrays
are float64 so that the FP64 oracle and the FP32 device path can start from
bit-identical values (cast once to float32, then widen for the oracle).

Workloads:
  drop_test   1,024 envs, dt 2 ms, 250 steps: base at 0.80 m, orientation
              exp(N(0, 0.05 rad)^3), joints stand + N(0, 0.05), qd = 0,
              targets stand + N(0, 0.1) held, friction 1, seed 0.
  randomized  65,536 envs, dt 2 ms, decimation 10, 1,000 substeps: targets
              stand + U(-0.3, 0.3) * (hi - lo) redrawn every policy step (on
              the device), per-env friction U[0.4, 1.0], base-mass offset
              U[-1, +3] kg, initial base height U[0.75, 0.85] m, in-kernel
              reset when the base height drops below 0.3 m.
"""
import numpy as np

from .model import g1_model_data as M

NQ, NV, NU, NC = M.NQ, M.NV, M.NU, M.NC
STAND = np.asarray(M.qpos_stand, dtype=np.float64)
RANGE = np.asarray(M.jnt_range, dtype=np.float64)  # (29, 2)


def rotvec_to_quat(r):
    """(3, n) rotation vectors -> (4, n) unit quaternions (w, x, y, z)."""
    ang = np.sqrt((r * r).sum(axis=0))
    half = 0.5 * ang
    s = np.where(ang > 1e-12, np.sin(half) / np.maximum(ang, 1e-300), 0.5)
    return np.concatenate([np.cos(half)[None], r * s[None]], axis=0)


def free_anchor(nenv):
    return np.full((2 * NC, nenv), 1e30, dtype=np.float64)


def drop_test(nenv=1024, seed=0, z=0.80, orient_sigma=0.05, joint_sigma=0.05, target_sigma=0.1):
    """Initial state and held PD targets of the plain drop test.

    Returns dict(qpos (36,n), qvel (35,n), anchor (16,n), ctrl (29,n), mu (n,)),
    all float64 but exactly representable in float32.
    """
    rng = np.random.default_rng(seed)
    qpos = np.repeat(STAND[:, None], nenv, axis=1)
    qpos[0:2] = 0.0
    qpos[2] = z
    qpos[3:7] = rotvec_to_quat(rng.normal(0.0, orient_sigma, size=(3, nenv)))
    qpos[7:] += rng.normal(0.0, joint_sigma, size=(NU, nenv))
    ctrl = STAND[7:, None] + rng.normal(0.0, target_sigma, size=(NU, nenv))
    out = dict(qpos=qpos, qvel=np.zeros((NV, nenv)), anchor=free_anchor(nenv), ctrl=ctrl,
               mu=np.ones(nenv))
    return {k: v.astype(np.float32).astype(np.float64) for k, v in out.items()}


def randomized(nenv=65536, seed=0):
    """Initial state and per-env parameters of the randomised 65,536-env workload."""
    rng = np.random.default_rng(seed)
    qpos = np.repeat(STAND[:, None], nenv, axis=1)
    qpos[2] = rng.uniform(0.75, 0.85, size=nenv)
    ctrl = np.repeat(STAND[7:, None], nenv, axis=1)
    out = dict(qpos=qpos, qvel=np.zeros((NV, nenv)), anchor=free_anchor(nenv), ctrl=ctrl,
               mu=rng.uniform(0.4, 1.0, size=nenv), dmass=rng.uniform(-1.0, 3.0, size=nenv))
    return {k: v.astype(np.float32).astype(np.float64) for k, v in out.items()}


# Defaults of the randomised rollout (mirrored by the device rollout parameters).
ROLLOUT_DEFAULTS = dict(target_frac=0.3, reset_z=0.3, z0_lo=0.75, z0_hi=0.85, decim=10,
                        dt=2e-3, substeps=1000)
