"""Gradients through the G1 step: the horizon adjoint behind torch.autograd.

    loss = horizon_loss(targets, kp_scale, kd_scale, qpos0, qvel0, anchor0)
    loss.sum().backward()          # -> targets.grad, kp_scale.grad, ...

The loss of env e over H single-substep steps (dt from the config) is
    L_e = sum_{t=1..H} (z_t - z_ref)^2 + w_track * |q_t - u_{t-1}|^2
with z the base height and q the 29 joint angles; u_t the PD targets of
step t.  Forward and backward run in one call of g1b_adjoint (one CUDA
launch: the forward rollout with checkpoints every `checkpoint` steps, then
the hand-derived reverse-mode sweep of the step, segment by segment); the
autograd Function keeps its gradients for backward.  kp_scale / kd_scale
may be None (scales of 1; no gradient is returned for them).  Arrays are SoA
with the env axis last, as in G1Sim: targets (H, 29, nenv), qpos0 (36,
nenv), ...
"""
import ctypes as C

import torch

from . import _lib


def scratch_size(nenv, horizon, checkpoint):
    pr = _lib.AdjointProblem(horizon, checkpoint, 0.78, 0.1)
    n = C.c_size_t()
    _lib.check(_lib.lib().g1b_adjoint_scratch_size(nenv, C.byref(pr), C.byref(n)), "g1b_adjoint_scratch_size")
    return n.value


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def horizon_adjoint(targets, kp_scale, kd_scale, qpos0, qvel0, anchor0, checkpoint=8, z_ref=0.78, w_track=0.1,
                    config=None, scratch=None, stream=None):
    """Loss and gradients of every env (one call, no autograd).  float32
    tensors use the FP32 kernels, float64 the FP64 validation build."""
    H, nu, n = targets.shape
    assert nu == 29
    dt = targets.dtype
    assert dt in (torch.float32, torch.float64)
    dev = targets.device
    for t, shp in ((qpos0, (36, n)), (qvel0, (35, n)), (anchor0, (16, n)), (kp_scale, (n,)), (kd_scale, (n,))):
        if t is not None:
            assert t.dtype == dt and t.device == dev and tuple(t.shape) == shp and t.is_contiguous()
    assert targets.is_contiguous()
    cfg = config or _lib.default_config(dt=2e-3)
    pr = _lib.AdjointProblem(H, checkpoint, z_ref, w_track)
    need = scratch_size(n, H, checkpoint)
    if scratch is None:
        scratch = torch.empty(need, dtype=dt, device=dev)
    assert scratch.numel() >= need and scratch.dtype == dt
    out = dict(loss=torch.empty(n, dtype=dt, device=dev), grad_targets=torch.empty_like(targets),
               grad_kp=torch.empty(n, dtype=dt, device=dev), grad_kd=torch.empty(n, dtype=dt, device=dev),
               grad_qpos0=torch.empty(36, n, dtype=dt, device=dev), grad_qvel0=torch.empty(35, n, dtype=dt, device=dev))
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    fn = _lib.lib().g1b_adjoint if dt == torch.float32 else _lib.lib().g1b_adjoint_f64
    _lib.check(fn(n, C.byref(cfg), C.byref(pr), _p(qpos0), _p(qvel0), _p(anchor0), _p(targets), _p(kp_scale),
                  _p(kd_scale), _p(out["loss"]), _p(out["grad_targets"]), _p(out["grad_kp"]), _p(out["grad_kd"]),
                  _p(out["grad_qpos0"]), _p(out["grad_qvel0"]), _p(scratch), C.c_void_p(st)), "g1b_adjoint")
    return out


class HorizonLoss(torch.autograd.Function):
    """Per-env horizon loss with gradients for targets, gain scales and the
    initial (qpos, qvel) from the adjoint kernels."""

    @staticmethod
    def forward(ctx, targets, kp_scale, kd_scale, qpos0, qvel0, anchor0, checkpoint, z_ref, w_track, config):
        d = lambda t: None if t is None else t.detach().contiguous()  # noqa: E731
        r = horizon_adjoint(d(targets), d(kp_scale), d(kd_scale), d(qpos0), d(qvel0), d(anchor0), checkpoint, z_ref,
                            w_track, config)
        ctx.has_kp, ctx.has_kd = kp_scale is not None, kd_scale is not None
        ctx.save_for_backward(r["grad_targets"], r["grad_kp"], r["grad_kd"], r["grad_qpos0"], r["grad_qvel0"])
        return r["loss"]

    @staticmethod
    def backward(ctx, g):
        gt, gkp, gkd, gq, gv = ctx.saved_tensors
        return (gt * g, gkp * g if ctx.has_kp else None, gkd * g if ctx.has_kd else None, gq * g, gv * g, None, None,
                None, None, None)


def horizon_loss(targets, kp_scale, kd_scale, qpos0, qvel0, anchor0, checkpoint=8, z_ref=0.78, w_track=0.1,
                 config=None):
    return HorizonLoss.apply(targets, kp_scale, kd_scale, qpos0, qvel0, anchor0, checkpoint, z_ref, w_track, config)
