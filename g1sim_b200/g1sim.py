"""Python surface of the B200 G1 step: the reference's G1Sim, unchanged.

Mirrors the reference's ``src/g1sim.py`` (class G1Sim, :35-170): same
constructor, tensors (SoA, (dim, nenv) float32 on the device), methods
``reset_done`` / ``reset_all`` / ``step`` / ``get_obs`` and observation
layout, bound to libg1cuda.so through ctypes exactly as the reference binds
its build/libg1cuda.so.  The stand keyframe and joint ranges come from the
generated model tables instead of MuJoCo (the reference reads them with
mujoco, :62-72; the values are identical, see g1sim_b200/model).

Extensions (keyword-only, all default to the reference behaviour):
``dt`` / ``config`` select the step configuration (the reference's GPU ABI
fixes dt = 1 ms), ``mu`` / ``dmass`` are per-env friction and base-mass
offset tensors, and ``rollout`` runs the decimated rollout with in-kernel
target redraw and reset.
"""
import ctypes as C

import torch

from . import _lib
from .model import g1_model_data as M

NQ, NV, NU, NC = M.NQ, M.NV, M.NU, M.NC

# reference src/g1sim.py:76-82 (legs, waist, left arm, right arm)
ACTION_SCALE = (
    0.443200, 0.274054, 0.443200, 0.274054, 0.365131, 0.365131,
    0.443200, 0.274054, 0.443200, 0.274054, 0.365131, 0.365131,
    0.443200, 0.365131, 0.365131,
    0.365131, 0.365131, 0.365131, 0.365131, 0.365131, 0.074501, 0.074501,
    0.365131, 0.365131, 0.365131, 0.365131, 0.365131, 0.074501, 0.074501,
)


def _stream(device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _check(t, shape, dtype, device, name):
    if t is None:
        return
    if t.device != device:
        raise ValueError(f"{name} must be on {device}, got {t.device}")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def _require_cuda(device):
    if device.type != "cuda" or not torch.cuda.is_available():
        raise RuntimeError("g1sim_b200 runs on a CUDA device only (no CPU fallback)")


# ------------------------------------------------------------ functional API
def step(qpos, qvel, anchor, ctrl, nsub=1, config=None, mu=None, dmass=None, kp_scale=None,
         kd_scale=None, foot_pos=None, foot_vel=None, contact_forces=None):
    """nsub substeps in place (g1b_step).  All tensors (dim, nenv) float32 on one device."""
    dev = qpos.device
    _require_cuda(dev)
    n = qpos.shape[1]
    f32 = torch.float32
    for t, shp, nm in ((qpos, (NQ, n), "qpos"), (qvel, (NV, n), "qvel"), (anchor, (2 * NC, n), "anchor"),
                       (ctrl, (NU, n), "ctrl"), (mu, (n,), "mu"), (dmass, (n,), "dmass"),
                       (kp_scale, (n,), "kp_scale"), (kd_scale, (n,), "kd_scale"),
                       (foot_pos, (6, n), "foot_pos"), (foot_vel, (6, n), "foot_vel"),
                       (contact_forces, (NC, n), "contact_forces")):
        _check(t, shp, f32, dev, nm)
    cfg = config if config is not None else _lib.default_config()
    rc = _lib.lib().g1b_step(n, int(nsub), C.byref(cfg), _ptr(qpos), _ptr(qvel), _ptr(anchor), _ptr(ctrl),
                             _ptr(mu), _ptr(dmass), _ptr(kp_scale), _ptr(kd_scale), _ptr(foot_pos),
                             _ptr(foot_vel), _ptr(contact_forces), _stream(dev))
    _lib.check(rc, "g1b_step")


def rollout(qpos, qvel, anchor, ctrl, npolicy, decim, config=None, seed=0, step0=0, target_frac=0.3,
            reset_z=0.3, z0=(0.75, 0.85), redraw=True, mu=None, dmass=None, reset_count=None,
            foot_pos=None, foot_vel=None, contact_forces=None):
    """Decimated rollout (g1b_rollout): npolicy x (redraw targets, decim substeps, reset check)."""
    dev = qpos.device
    _require_cuda(dev)
    n = qpos.shape[1]
    f32 = torch.float32
    for t, shp, nm in ((qpos, (NQ, n), "qpos"), (qvel, (NV, n), "qvel"), (anchor, (2 * NC, n), "anchor"),
                       (ctrl, (NU, n), "ctrl"), (mu, (n,), "mu"), (dmass, (n,), "dmass"),
                       (foot_pos, (6, n), "foot_pos"), (foot_vel, (6, n), "foot_vel"),
                       (contact_forces, (NC, n), "contact_forces")):
        _check(t, shp, f32, dev, nm)
    _check(reset_count, (n,), torch.int32, dev, "reset_count")
    cfg = config if config is not None else _lib.default_config(dt=2e-3)
    rp = _lib.RolloutParams(int(seed) & 0xffffffff, int(step0), float(target_frac), float(reset_z),
                            float(z0[0]), float(z0[1]), int(bool(redraw)))
    rc = _lib.lib().g1b_rollout(n, int(npolicy), int(decim), C.byref(cfg), C.byref(rp), _ptr(qpos),
                                _ptr(qvel), _ptr(anchor), _ptr(ctrl), _ptr(mu), _ptr(dmass),
                                _ptr(reset_count), _ptr(foot_pos), _ptr(foot_vel), _ptr(contact_forces),
                                _stream(dev))
    _lib.check(rc, "g1b_rollout")


def reset_done(qpos, qvel, anchor, done, seed=42, noise=0.05, drop=0.02):
    """The reference's g1_cuda_reset_done on tensors."""
    dev = qpos.device
    _require_cuda(dev)
    n = qpos.shape[1]
    _check(done, (n,), torch.uint8, dev, "done")
    _lib.lib().g1_cuda_reset_done(n, _ptr(qpos), _ptr(qvel), _ptr(anchor), _ptr(done),
                                  int(seed) & 0xffffffff, float(noise), float(drop), _stream(dev))
    err = _lib.last_error()
    if err.startswith("g1_cuda_reset_done") or err.startswith("reset_done_kernel"):
        raise RuntimeError(err)


# ------------------------------------------------------------------- G1Sim
class G1Sim:
    """The reference's G1Sim (src/g1sim.py:35-170) on the B200 kernels."""

    def __init__(self, nenv: int, device: torch.device, *, dt=None, config=None, mu=None, dmass=None):
        device = torch.device(device)
        _require_cuda(device)
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.nenv = nenv
        self.device = device
        self.NQ, self.NV, self.NU, self.NC = NQ, NV, NU, NC
        f32 = dict(dtype=torch.float32, device=device)
        # SoA layout: (dim, nenv)  (reference :46-53)
        self.qpos = torch.zeros((NQ, nenv), **f32)
        self.qvel = torch.zeros((NV, nenv), **f32)
        self.anchor = torch.full((2 * NC, nenv), 1e30, **f32)
        self.ctrl = torch.zeros((NU, nenv), **f32)
        self.foot_pos = torch.zeros((6, nenv), **f32)
        self.foot_vel = torch.zeros((6, nenv), **f32)
        self.contact_forces = torch.zeros((NC, nenv), **f32)
        # RL state (reference :55-60)
        self.commands = torch.zeros((3, nenv), **f32)
        self.last_actions = torch.zeros((NU, nenv), **f32)
        self.done = torch.ones(nenv, dtype=torch.uint8, device=device)
        # stand keyframe and joint limits (reference :62-72, from the model tables)
        self.default_qpos = torch.tensor(M.qpos_stand, **f32).unsqueeze(1)
        self.default_joint_pos = self.default_qpos[7:36]
        self.global_gravity = torch.zeros((3, nenv), **f32)
        self.global_gravity[2, :] = -1.0
        rng = torch.tensor(M.jnt_range, **f32)
        self.joint_pos_lower = rng[:, 0].unsqueeze(1)
        self.joint_pos_upper = rng[:, 1].unsqueeze(1)
        # per-actuator action scale: the reference's literal table (:74-82); its
        # comment's 0.25 * effort_limit / stiffness does not reproduce these
        # values with this model's kp, so the values themselves are kept
        self.action_scale = torch.tensor(ACTION_SCALE, **f32).unsqueeze(1)
        # extensions
        if config is None and dt is not None:
            config = _lib.default_config(dt=dt)
        self.config = config
        self.mu = mu
        self.dmass = dmass

    def reset_done(self, done: torch.Tensor, seed: int = 42, noise: float = 0.05, drop: float = 0.02):
        """Resets environments where done is True/1 (reference :84-103)."""
        assert done.shape == (self.nenv,)
        assert done.dtype == torch.uint8
        assert done.device == self.device
        assert done.is_contiguous()
        reset_done(self.qpos, self.qvel, self.anchor, done, seed, noise, drop)

    def reset_all(self, seed: int = 42, noise: float = 0.05, drop: float = 0.02):
        """Resets all environments (reference :105-108)."""
        self.done.fill_(1)
        self.reset_done(self.done, seed, noise, drop)

    def step(self, nsub: int = 1):
        """Steps all environments forward by nsub substeps (reference :110-130)."""
        assert self.ctrl.is_contiguous()
        assert self.qpos.is_contiguous()
        self.last_actions.copy_(self.ctrl)
        if self.config is None and self.mu is None and self.dmass is None:
            # the reference's own entry point and its fixed dt = 1 ms
            _lib.lib().g1_cuda_step(self.nenv, int(nsub), _ptr(self.qpos), _ptr(self.qvel), _ptr(self.anchor),
                                    _ptr(self.ctrl), _ptr(self.foot_pos), _ptr(self.foot_vel),
                                    _ptr(self.contact_forces), _stream(self.device))
            err = _lib.last_error()
            if err.startswith("step_kernel") or err.startswith("cudaFuncSetAttribute"):
                raise RuntimeError(err)
        else:
            step(self.qpos, self.qvel, self.anchor, self.ctrl, nsub, config=self.config, mu=self.mu,
                 dmass=self.dmass, foot_pos=self.foot_pos, foot_vel=self.foot_vel,
                 contact_forces=self.contact_forces)

    def get_obs(self) -> torch.Tensor:
        """Observation (nenv, 99): commands, projected gravity, base lin vel
        (body), base ang vel, joint pos error, joint vel, previous actions
        (reference :132-170)."""
        q = self.qpos[3:7, :]
        qw, qx, qy, qz = q[0], q[1], q[2], q[3]
        q_vec_inv = torch.stack([-qx, -qy, -qz], dim=0)

        def quat_rotate_inverse(v):
            uv = torch.cross(q_vec_inv, v, dim=0)
            uuv = torch.cross(q_vec_inv, uv, dim=0)
            return v + 2.0 * (qw * uv + uuv)

        proj_gravity = quat_rotate_inverse(self.global_gravity)
        base_lin_vel = quat_rotate_inverse(self.qvel[0:3, :])
        obs = torch.cat([
            self.commands,
            proj_gravity,
            base_lin_vel,
            self.qvel[3:6, :],
            self.qpos[7:36, :] - self.default_joint_pos,
            self.qvel[6:35, :],
            self.last_actions,
        ], dim=0).T
        return obs
