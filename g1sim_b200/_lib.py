"""ctypes binding of libg1cuda.so (the C-ABI declared in include/g1sim_b200.h).

The library is the only compute path: if it is missing, or no CUDA device is
present, every entry point raises -- there is no CPU fallback.
"""
import ctypes as C
import os

from .build import LIB

_lib = None


class Config(C.Structure):
    """g1b_config (mirrors the reference G1Config, src/g1_types.h:33-42)."""
    _fields_ = [(n, C.c_float) for n in (
        "gravity_z", "contact_kn", "contact_dn", "contact_kt", "contact_dt",
        "limit_kp", "limit_kd", "dt")]


class RolloutParams(C.Structure):
    """g1b_rollout_params."""
    _fields_ = [("seed", C.c_uint), ("step0", C.c_int), ("target_frac", C.c_float),
                ("reset_z", C.c_float), ("z0_lo", C.c_float), ("z0_hi", C.c_float),
                ("redraw", C.c_int)]


class Policy(C.Structure):
    """g1b_policy: packed actor-critic (device pointers)."""
    _fields_ = [("weights", C.c_void_p), ("bias", C.c_void_p), ("log_std", C.c_void_p),
                ("obs_mean", C.c_void_p), ("obs_var", C.c_void_p)]


class TaskState(C.Structure):
    """g1b_task_state: per-env task state (device pointers, SoA)."""
    _fields_ = [("commands", C.c_void_p), ("prev_action", C.c_void_p), ("cmd_timer", C.c_void_p),
                ("ep_len", C.c_void_p), ("push_timer", C.c_void_p)]


class TaskParams(C.Structure):
    """g1b_task_params."""
    _fields_ = [("seed", C.c_uint), ("step0", C.c_int), ("cmd_lo", C.c_float * 3), ("cmd_hi", C.c_float * 3),
                ("cmd_steps_lo", C.c_int), ("cmd_steps_hi", C.c_int), ("push_steps_lo", C.c_int),
                ("push_steps_hi", C.c_int), ("push_vel", C.c_float * 6), ("max_episode", C.c_int),
                ("tilt_limit", C.c_float), ("reset_seed", C.c_uint), ("reset_noise", C.c_float),
                ("reset_drop", C.c_float), ("flags", C.c_int)]


class RolloutOut(C.Structure):
    """g1b_rollout_out: per-step outputs (device pointers, each nullable)."""
    _fields_ = [(n, C.c_void_p) for n in ("obs", "actions", "mean", "logp", "value", "reward", "done", "reset",
                                         "last_obs", "last_value")]


SAMPLE, PUSH, RESET, COMMANDS = 1, 2, 4, 8


class AdjointProblem(C.Structure):
    """g1b_adjoint_problem."""
    _fields_ = [("horizon", C.c_int), ("checkpoint", C.c_int), ("z_ref", C.c_float), ("w_track", C.c_float)]

_vp = C.c_void_p


class SurLayer(C.Structure):
    """g1b_sur_layer: one surrogate layer's parameters for g1b_sur_adam_cast."""
    _fields_ = [(n, C.c_void_p) for n in ("W", "b", "mW", "vW", "mb", "vb", "gW", "gb", "Wb", "Wt")] + \
        [("rows", C.c_int), ("cols", C.c_int)]


def lib():
    """Load libg1cuda.so once and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        raise RuntimeError(f"{LIB} is missing: build it with `python -m g1sim_b200.build` "
                           "(nvcc, sm_100a); there is no CPU fallback")
    L = C.CDLL(LIB)
    L.g1_cuda_step.argtypes = [C.c_int, C.c_int] + [_vp] * 8
    L.g1_cuda_step.restype = None
    L.g1_cuda_reset_done.argtypes = [C.c_int, _vp, _vp, _vp, _vp, C.c_uint, C.c_float, C.c_float, _vp]
    L.g1_cuda_reset_done.restype = None
    L.g1b_sizes.argtypes = [C.POINTER(C.c_int)] * 5
    L.g1b_default_config.argtypes = [C.POINTER(Config)]
    L.g1b_last_error.restype = C.c_char_p
    L.g1b_step.argtypes = [C.c_int, C.c_int, C.POINTER(Config)] + [_vp] * 12
    L.g1b_rollout.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(Config), C.POINTER(RolloutParams)] + [_vp] * 11
    L.g1b_set_launch.argtypes = [C.c_int, C.c_int, C.c_int]
    L.g1b_get_launch.argtypes = [C.POINTER(C.c_int)] * 3
    L.g1b_autotune.argtypes = [C.c_int, C.c_int, _vp, C.POINTER(C.c_float)]
    L.g1b_ffma_peak.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.g1b_policy_default_params.argtypes = [C.POINTER(TaskParams)]
    L.g1b_policy_sizes.argtypes = [C.POINTER(C.c_int)] * 4
    L.g1b_policy_rollout.argtypes = ([C.c_int, C.c_int, C.c_int, C.POINTER(Config), C.POINTER(TaskParams),
                                      C.POINTER(Policy)] + [_vp] * 6 +
                                     [C.POINTER(TaskState), C.POINTER(RolloutOut)] + [_vp] * 4)
    L.g1b_policy_status.argtypes = [C.POINTER(C.c_int)]
    L.g1b_gemm_bf16.argtypes = [C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int,
                                _vp]
    L.g1b_gemm_status.argtypes = [C.POINTER(C.c_int)]
    L.g1b_gemm_bf16_acc.argtypes = [C.c_int] * 3 + [_vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp]
    L.g1b_gemm_bf16_atb_acc.argtypes = [C.c_int] * 3 + [_vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp]
    L.g1b_sur_linear_silu.argtypes = [C.c_int] * 3 + [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _vp, C.c_int,
                                                       _vp, C.c_int, _vp]
    L.g1b_sur_linear_silu_bwd.argtypes = [C.c_int] * 3 + [_vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int,
                                                           _vp, C.c_int, _vp, _vp]
    L.g1b_sur_loss.argtypes = [C.c_int, C.c_int] + [_vp] * 8
    L.g1b_sur_adam_cast.argtypes = [C.c_int, C.POINTER(SurLayer), _vp, _vp, C.c_float, C.c_float, C.c_float, _vp]
    L.g1b_sur_cast.argtypes = [C.c_int, C.c_int, _vp, _vp, _vp, _vp]
    L.g1b_sur_features.argtypes = [C.c_int] + [_vp] * 12
    L.g1b_sur_features_vjp.argtypes = [C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp]
    L.g1b_sur_integrate.argtypes = [C.c_int, _vp, C.c_int, _vp, _vp, C.c_float, _vp, _vp, _vp]
    L.g1b_sur_integrate_vjp.argtypes = [C.c_int, _vp, _vp, _vp, C.c_int, _vp, _vp, C.c_float, _vp, _vp, _vp,
                                        C.c_int, _vp]
    L.g1b_sur_seed.argtypes = [C.c_int, _vp, _vp, _vp]
    L.g1b_adjoint_scratch_size.argtypes = [C.c_int, C.POINTER(AdjointProblem), C.POINTER(C.c_size_t)]
    for name in ("g1b_adjoint", "g1b_adjoint_f64"):
        getattr(L, name).argtypes = [C.c_int, C.POINTER(Config), C.POINTER(AdjointProblem)] + [_vp] * 14
    _lib = L
    return L


def check(rc, what):
    if rc != 0:
        msg = lib().g1b_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")


def default_config(dt=None):
    c = Config()
    check(lib().g1b_default_config(C.byref(c)), "g1b_default_config")
    if dt is not None:
        c.dt = dt
    return c


def set_launch(mapping, block, blocks_per_sm=0):
    """Launch shape of the step kernels (mapping 0: thread per env, 1: two threads per env)."""
    check(lib().g1b_set_launch(int(mapping), int(block), int(blocks_per_sm)), "g1b_set_launch")


def autotune(nenv, nsub=10, stream=None):
    """Time every launch shape on this device for nenv envs x nsub substeps; keep the fastest.
    Returns (mapping, block, blocks_per_sm, best_ms)."""
    best = C.c_float()
    check(lib().g1b_autotune(int(nenv), int(nsub), stream, C.byref(best)), "g1b_autotune")
    return get_launch() + (best.value,)


def get_launch():
    v = [C.c_int() for _ in range(3)]
    check(lib().g1b_get_launch(*[C.byref(x) for x in v]), "g1b_get_launch")
    return tuple(x.value for x in v)


def last_error():
    return lib().g1b_last_error().decode(errors="replace")


def policy_default_params():
    p = TaskParams()
    check(lib().g1b_policy_default_params(C.byref(p)), "g1b_policy_default_params")
    return p


def policy_sizes():
    v = [C.c_int() for _ in range(4)]
    check(lib().g1b_policy_sizes(*[C.byref(x) for x in v]), "g1b_policy_sizes")
    return tuple(x.value for x in v)


def policy_status():
    """Device status of the policy kernels (synchronises); 0 = ok.  Clears it."""
    code = C.c_int()
    check(lib().g1b_policy_status(C.byref(code)), "g1b_policy_status")
    return code.value
