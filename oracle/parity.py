"""Accuracy of GPU states against the FP64 oracle (TEST INFRASTRUCTURE).

Used by tests/ and by bench.py's accuracy leg (outside its timed region) as
the checker; the product never imports it.

Error metric, per state component: |x_gpu - x_64| / max(|x_64|, 1), both
sides starting from the same float32 state (the GPU's own state widened
exactly to double), so the number measures the kernel's arithmetic and not
the rounding of its inputs.  The model is discontinuous (contact touchdown,
force clamps, stick / slip, soft limits, torque clamp): an env-step whose
FP64 state lies within FP32 rounding of such a threshold (oracle branch
margin < 1) may legitimately take the other branch in FP32; those env-steps
are counted and left out of the maxima.
"""
import numpy as np


def relerr(x, ref):
    return np.abs(x - ref) / np.maximum(np.abs(ref), 1.0)


def _q(a, p):
    return float(np.percentile(a, p)) if a.size else 0.0


def per_substep(oracle, gpu_step, read_state, cfg, ctrl, mu=None, dmass=None, substeps=10):
    """Per-substep error of the GPU step against the oracle.

    gpu_step() advances the GPU envs by one substep; read_state() returns
    (qpos, qvel, anchor) of those envs as float64 arrays [dim][nenv]; ctrl,
    mu, dmass are the envs' float64 targets and parameters.  Each substep
    both sides start from the GPU's state."""
    eq, ev, ea, kept, total = [], [], [], 0, 0
    for _ in range(substeps):
        q64, v64, a64 = read_state()
        mg = oracle.branch_margin(cfg, q64, v64, a64, ctrl, mu=mu, dmass=dmass)
        oracle.step_soa(1, cfg, q64, v64, a64, ctrl, mu=mu, dmass=dmass, outputs=False)
        gpu_step()
        gq, gv, ga = read_state()
        keep = mg >= 1.0
        kept += int(keep.sum())
        total += keep.size
        eq.append(relerr(gq, q64).max(axis=0)[keep])
        ev.append(relerr(gv, v64).max(axis=0)[keep])
        both = (a64 < 1e29) & (ga < 1e29)
        ea.append(np.where(both, np.abs(ga - a64), 0.0).max(axis=0)[keep])
    eq, ev, ea = np.concatenate(eq), np.concatenate(ev), np.concatenate(ea)
    return {"env_substeps": total, "near_branch_fraction": 1.0 - kept / max(total, 1),
            "qpos_max": float(eq.max(initial=0.0)), "qpos_median": _q(eq, 50),
            "qvel_max": float(ev.max(initial=0.0)), "qvel_p99": _q(ev, 99), "qvel_median": _q(ev, 50),
            "anchor_max_m": float(ea.max(initial=0.0))}


def drift(oracle, gpu_run, read_state, cfg, ctrl, mu=None, dmass=None, marks=(10, 100, 400)):
    """Drift of a GPU rollout from the oracle's, both from the same start.

    gpu_run(k) advances the GPU envs by k substeps with ctrl held; at each
    mark the per-env maximum error over qpos and over qvel is summarised
    (median, 90th percentile, max over envs)."""
    q64, v64, a64 = read_state()
    out, done = {}, 0
    for m in marks:
        k = m - done
        oracle.step_soa(k, cfg, q64, v64, a64, ctrl, mu=mu, dmass=dmass, outputs=False)
        gpu_run(k)
        done = m
        gq, gv, _ = read_state()
        eq, ev = relerr(gq, q64).max(axis=0), relerr(gv, v64).max(axis=0)
        out[str(m)] = {"qpos_median": _q(eq, 50), "qpos_p90": _q(eq, 90), "qpos_max": float(eq.max()),
                       "qvel_median": _q(ev, 50), "qvel_p90": _q(ev, 90), "qvel_max": float(ev.max())}
    return out


def composed(oracle, q0, v0, a0, ctrl, gq, gv, cfg, substeps, mu=None, dmass=None):
    """Error of a GPU state after `substeps` substeps (gq, gv) against the
    oracle run from the same float32 start (q0, v0, a0 float64, ctrl held).
    Returns per-env maxima for qpos and qvel plus the oracle's margin at the
    start (the first substep's distance from a branch threshold)."""
    q, v, a = q0.copy(), v0.copy(), a0.copy()
    mg = oracle.branch_margin(cfg, q, v, a, ctrl, mu=mu, dmass=dmass)
    oracle.step_soa(substeps, cfg, q, v, a, ctrl, mu=mu, dmass=dmass, outputs=False)
    return relerr(gq, q).max(axis=0), relerr(gv, v).max(axis=0), mg
