"""Horizon adjoint through the G1 step (needs a B200).

Reference values come from the FP64 oracle on the CPU: the loss of a
64-step rollout, and central finite differences of it (h = 1e-6) with
respect to PD targets, gain scales and the initial state, on all 16 envs of
the workload's FD sample and on problems whose trajectories cross the
model's switches: feet touching down during the horizon, feet slipping
under a base push, joints driven past their soft limits.

  * FP64 device build (g1b_adjoint_f64): loss to 1e-6 relative (the device
    contracts a*b+c into FMAs, the oracle does not; 64 steps of stiff
    contact dynamics grow that 1e-16 difference to ~2e-7), gradients
    to 1e-4 relative of the FD value (FD truncation and rounding at h = 1e-6
    are ~1e-7 here).  Where an FD stencil straddles a switch (its one-sided
    differences disagree) it is repeated with h = 1e-7: the adjoint is the
    derivative along the branch taken (measured: 1 of 56 stencils on the
    touchdown problem, which then agrees to 1e-8);
  * FP32 kernels (g1b_adjoint): loss to 1e-4, gradient fields to 1e-3 in
    relative 2-norm and cosine > 0.9999 against the FP64 build (measured
    ~4e-6 on this settled standing problem);
  * the checkpoint interval changes nothing (bit-identical results);
  * the torch.autograd.Function returns the kernel's gradients.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from g1sim_b200 import adjoint as A
from g1sim_b200.model import g1_model_data as M

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)
H, NENV = 64, 16  # the workload's horizon and its FD sample of 16 envs
STAND = np.asarray(M.qpos_stand)


def problem(golden_host, n=NENV, seed=0, kind="stand"):
    """Settled standing states (the reference's own settling run) with small
    joint / velocity perturbations; targets = stand + N(0, 0.05) per step;
    gain scales U[0.8, 1.2].  kind "touchdown": the stand pose 2-3 cm above
    the ground with free anchors (the feet land during the horizon); "slip":
    the standing state pushed sideways at 0.5-0.7 m/s (the feet slide);
    "limits": targets past the joint ranges on both sides (soft limits)."""
    rng = np.random.default_rng(seed)
    q0 = np.repeat(golden_host["settle_qpos"][:, None], n, axis=1)
    v0 = np.repeat(golden_host["settle_qvel"][:, None], n, axis=1)
    a0 = np.repeat(golden_host["settle_anchor"][:, None], n, axis=1)
    q0[7:] += rng.normal(0, 0.01, size=(29, n))
    v0[6:] += rng.normal(0, 0.05, size=(29, n))
    tg = STAND[7:, None, None].transpose(1, 0, 2) + rng.normal(0, 0.05, size=(H, 29, n))
    if kind == "touchdown":
        q0[:] = STAND[:, None]
        q0[2] = STAND[2] + rng.uniform(0.0, 0.01, n)
        q0[7:] += rng.normal(0, 0.01, size=(29, n))
        v0[:] = 0.0
        a0[:] = 1e30
    elif kind == "slip":
        ang = rng.uniform(0, 2 * np.pi, n)
        sp = rng.uniform(0.5, 0.7, n)
        v0[0] += sp * np.cos(ang)
        v0[1] += sp * np.sin(ang)
    elif kind == "limits":
        rngs = np.asarray(M.jnt_range)
        for j in (3, 9, 16, 23):  # knees and shoulders: past the lower, then the upper limit
            tg[: H // 2, j] = rngs[j, 0] - 0.3
            tg[H // 2:, j] = rngs[j, 1] + 0.3
    kp = rng.uniform(0.8, 1.2, n)
    kd = rng.uniform(0.8, 1.2, n)
    f32 = lambda x: np.asarray(x, np.float32).astype(np.float64)  # noqa: E731  (exact in both precisions)
    return dict(q0=f32(q0), v0=f32(v0), a0=f32(a0), tg=f32(tg), kp=f32(kp), kd=f32(kd))


def oracle_loss(oracle, p, e, tg=None, kp=None, kd=None, q0=None, v0=None, z_ref=0.78, w=0.1):
    from oracle import EnvParams
    cfg = oracle.config(dt=2e-3)
    q = np.ascontiguousarray((p["q0"] if q0 is None else q0)[:, e], dtype=np.float64)
    v = np.ascontiguousarray((p["v0"] if v0 is None else v0)[:, e], dtype=np.float64)
    an = np.ascontiguousarray(p["a0"][:, e], dtype=np.float64)
    tg = p["tg"] if tg is None else tg
    ep = EnvParams(1.0, 0.0, p["kp"][e] if kp is None else kp, p["kd"][e] if kd is None else kd)
    dp = C.POINTER(C.c_double)
    L = 0.0
    for t in range(H):
        u = np.ascontiguousarray(tg[t, :, e], dtype=np.float64)
        oracle.lib.g1o_step(C.byref(cfg), C.byref(ep), q.ctypes.data_as(dp), v.ctypes.data_as(dp),
                            u.ctypes.data_as(dp), an.ctypes.data_as(dp), 1, None, None, None)
        L += (q[2] - z_ref) ** 2 + w * np.sum((q[7:] - u) ** 2)
    return L


def run(p, dtype, checkpoint=8):
    t = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=dtype, device=DEV)  # noqa: E731
    r = A.horizon_adjoint(t(p["tg"]), t(p["kp"]), t(p["kd"]), t(p["q0"]), t(p["v0"]), t(p["a0"]),
                          checkpoint=checkpoint)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy().astype(np.float64) for k, v in r.items()}


@pytest.fixture(scope="module")
def prob(golden_host):
    return problem(golden_host)


@pytest.fixture(scope="module")
def r64(prob):
    return run(prob, torch.float64)


def test_loss_matches_oracle(prob, r64, oracle):
    for e in range(4):
        ref = oracle_loss(oracle, prob, e)
        assert abs(r64["loss"][e] - ref) <= 1e-6 * abs(ref), (e, r64["loss"][e], ref)


def central(f, h=1e-6):
    """Central difference of f(step) at 0 with step h (the workload's FD
    step).  Where the stencil straddles a switch of the model (the central
    differences at h and h / 2 disagree by more than their truncation and
    rounding errors), the difference is taken again with h / 10: the adjoint
    is the derivative along the branch taken, which a stencil across the
    switch does not measure."""
    f0 = f(0.0)
    c1 = (f(h) - f(-h)) / (2 * h)
    c2 = (f(h / 2) - f(-h / 2)) / h
    noise = 8 * np.finfo(np.float64).eps * abs(f0) / h
    if abs(c1 - c2) <= 1e-6 * max(abs(c1), 1e-3) + noise:
        return c1, False
    return (f(h / 10) - f(-h / 10)) / (2 * h / 10), True


def fd_errors(prob, r64, oracle, envs, seed=5, ntargets=3, straddled=None):
    rng = np.random.default_rng(seed)
    errs = []
    note = (lambda s: straddled.append(s)) if straddled is not None else (lambda s: None)  # noqa: E731

    def check(ad, f):
        fd, st = central(f)
        note(st)
        errs.append(abs(ad - fd) / max(abs(fd), 1e-3))

    for e in envs:
        # individual targets
        for _ in range(ntargets):
            t, j = int(rng.integers(H)), int(rng.integers(29))

            def ft(x, t=t, j=j):
                tg = prob["tg"].copy()
                tg[t, j, e] += x
                return oracle_loss(oracle, prob, e, tg=tg)
            check(r64["grad_targets"][t, j, e], ft)
        # gain scales
        for key, gk in (("kp", "grad_kp"), ("kd", "grad_kd")):
            x0 = prob[key][e]
            check(r64[gk][e], lambda x, key=key, x0=x0: oracle_loss(oracle, prob, e, **{key: x0 + x}))
        # a random direction over all targets
        d = rng.normal(size=prob["tg"].shape) * (np.arange(prob["tg"].shape[2]) == e)
        check(float(np.sum(r64["grad_targets"][:, :, e] * d[:, :, e])),
              lambda x, d=d: oracle_loss(oracle, prob, e, tg=prob["tg"] + x * d))
        # initial joint velocity
        k = int(rng.integers(29))

        def fv(x, k=k):
            v = prob["v0"].copy()
            v[6 + k, e] += x
            return oracle_loss(oracle, prob, e, v0=v)
        check(r64["grad_qvel0"][6 + k, e], fv)
    return np.array(errs)


def test_fp64_gradients_match_central_differences(prob, r64, oracle):
    """All 16 envs of the FD sample."""
    errs = fd_errors(prob, r64, oracle, range(NENV))
    print(f"FD check: {len(errs)} entries, max rel err {errs.max():.2e}, median {np.median(errs):.2e}")
    assert np.median(errs) < 1e-6
    assert errs.max() < 1e-4


def switches(prob, oracle, e):
    """Which switches the oracle trajectory of env e crosses."""
    from oracle import EnvParams
    cfg = oracle.config(dt=2e-3)
    q = np.ascontiguousarray(prob["q0"][:, e], dtype=np.float64)
    v = np.ascontiguousarray(prob["v0"][:, e], dtype=np.float64)
    an = np.ascontiguousarray(prob["a0"][:, e], dtype=np.float64)
    ep = EnvParams(1.0, 0.0, prob["kp"][e], prob["kd"][e])
    dp = C.POINTER(C.c_double)
    rng = np.asarray(M.jnt_range)
    seen = set()
    free0 = an >= 1e29
    for t in range(H):
        a_prev = an.copy()
        u = np.ascontiguousarray(prob["tg"][t, :, e], dtype=np.float64)
        oracle.lib.g1o_step(C.byref(cfg), C.byref(ep), q.ctypes.data_as(dp), v.ctypes.data_as(dp),
                            u.ctypes.data_as(dp), an.ctypes.data_as(dp), 1, None, None, None)
        if np.any(free0 & (an < 1e29)):
            seen.add("touchdown")
        stuck = (a_prev < 1e29) & (an < 1e29)
        if np.any(np.abs(an - a_prev)[stuck] > 1e-9):
            seen.add("slip")
        if np.any(q[7:] < rng[:, 0]) or np.any(q[7:] > rng[:, 1]):
            seen.add("limit")
    return seen


@pytest.mark.parametrize("kind,switch", [("touchdown", "touchdown"), ("slip", "slip"), ("limits", "limit")])
def test_fd_across_switches(golden_host, oracle, kind, switch):
    """Trajectories through touchdown, slip and soft-limit switches: the
    adjoint is the derivative of the loss along the branches taken."""
    prob = problem(golden_host, n=NENV, seed=21, kind=kind)
    crossed = [e for e in range(NENV) if switch in switches(prob, oracle, e)]
    assert len(crossed) >= NENV // 2, (kind, crossed)
    r = run(prob, torch.float64)
    for e in range(4):
        ref = oracle_loss(oracle, prob, e)
        assert abs(r["loss"][e] - ref) <= 1e-6 * abs(ref), (kind, e, r["loss"][e], ref)
    straddled = []
    errs = fd_errors(prob, r, oracle, crossed[:8], seed=7, straddled=straddled)
    print(f"{kind}: {len(crossed)} of {NENV} envs cross it; FD check {len(errs)} entries, max rel err "
          f"{errs.max():.2e}, median {np.median(errs):.2e}; {sum(straddled)} stencils straddled a switch")
    assert sum(straddled) <= len(errs) // 10
    assert np.median(errs) < 1e-5
    assert errs.max() < 1e-4


def test_fp32_matches_fp64(prob, r64):
    r32 = run(prob, torch.float32)
    assert np.all(np.abs(r32["loss"] - r64["loss"]) <= 1e-4 * np.abs(r64["loss"]))
    for k in ("grad_targets", "grad_kp", "grad_kd", "grad_qvel0"):
        a, b = r32[k].ravel(), r64[k].ravel()
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
        print(f"{k}: FP32 vs FP64 relative 2-norm error {rel:.2e}, cosine {cos:.6f}")
        assert rel < 1e-3 and cos > 0.9999


def test_checkpoint_interval_changes_nothing(prob):
    a, b, c = run(prob, torch.float32, 8), run(prob, torch.float32, 1), run(prob, torch.float32, 64)
    for k in a:
        assert np.array_equal(a[k], b[k]) and np.array_equal(a[k], c[k]), k


def test_autograd_function(prob):
    t = lambda x, g=False: torch.tensor(np.ascontiguousarray(x), dtype=torch.float32, device=DEV,  # noqa: E731
                                        requires_grad=g)
    tg, kp, kd = t(prob["tg"], True), t(prob["kp"], True), t(prob["kd"], True)
    q0, v0, a0 = t(prob["q0"], True), t(prob["v0"], True), t(prob["a0"])
    w = torch.linspace(0.5, 1.5, NENV, device=DEV)
    loss = A.horizon_loss(tg, kp, kd, q0, v0, a0)
    (loss * w).sum().backward()
    r = run(prob, torch.float32)
    wn = w.cpu().numpy()
    assert np.allclose(tg.grad.cpu().numpy(), r["grad_targets"] * wn, rtol=1e-6, atol=0)
    assert np.allclose(kp.grad.cpu().numpy(), r["grad_kp"] * wn, rtol=1e-6, atol=0)
    assert np.allclose(v0.grad.cpu().numpy(), r["grad_qvel0"] * wn, rtol=1e-6, atol=0)


def test_invalid_arguments_are_rejected(prob):
    t = torch.zeros(H, 29, 4, device=DEV)
    with pytest.raises(AssertionError):
        A.horizon_adjoint(t, None, None, torch.zeros(36, 5, device=DEV), torch.zeros(35, 4, device=DEV),
                          torch.zeros(16, 4, device=DEV))
