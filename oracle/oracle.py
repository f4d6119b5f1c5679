"""ctypes front end of the FP64 C oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module.  It loads oracle/_build/libg1oracle.so (our restatement of the
reference's host physics, oracle/g1_oracle.c) and, when present, the
reference's own builds in oracle/_ref/ (oracle/Makefile target ``ref``).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

NB, NQ, NV, NU, NC = 30, 36, 35, 29, 8

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)


class Config(C.Structure):
    """g1o_config (mirrors the reference G1Config, src/g1_types.h:33-42)."""
    _fields_ = [(n, C.c_double) for n in (
        "gravity_z", "contact_kn", "contact_dn", "contact_kt", "contact_dt",
        "limit_kp", "limit_kd", "dt")]


class EnvParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("mu", "dmass", "kp_scale", "kd_scale")]


class RolloutParams(C.Structure):
    _fields_ = [("seed", C.c_uint), ("step0", C.c_int), ("target_frac", C.c_float),
                ("reset_z", C.c_float), ("z0_lo", C.c_float), ("z0_hi", C.c_float),
                ("redraw", C.c_int)]


def _p(a, ct=_dp):
    if a is None:
        return None
    return a.ctypes.data_as(ct)


def build():
    """Compile the oracle (and nothing else) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def _need(a, dtype):
    assert a.dtype == dtype and a.flags.c_contiguous, (a.dtype, a.flags)
    return a


class Oracle:
    """Our FP64 oracle (oracle/g1_oracle.c)."""

    def __init__(self, path=None):
        path = path or os.path.join(BUILD, "libg1oracle.so")
        if not os.path.exists(path):
            build()
        L = self.lib = C.CDLL(path)
        L.g1_sizes.restype = C.c_int
        L.g1_c_fk.argtypes = [_dp, _dp, _dp]
        L.g1_c_fd.argtypes = [_dp, _dp, _dp, _dp]
        L.g1_c_step.argtypes = [_dp, _dp, _dp, C.c_int, C.c_double, _dp, _dp]
        L.g1o_default_config.argtypes = [C.POINTER(Config)]
        L.g1o_step.argtypes = [C.POINTER(Config), C.POINTER(EnvParams), _dp, _dp, _dp, _dp,
                               C.c_int, _dp, _dp, _dp]
        L.g1o_step_soa.argtypes = [C.c_int, C.c_int, C.POINTER(Config), _dp, _dp, _dp, _dp,
                                   _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.g1o_reset_done_soa.argtypes = [C.c_int, _dp, _dp, _dp, C.POINTER(C.c_uint8),
                                         C.c_uint, C.c_float, C.c_float]
        L.g1o_hash.argtypes = [C.c_uint]
        L.g1o_hash.restype = C.c_uint
        L.g1o_uniform.argtypes = [C.c_uint, C.c_uint, C.c_uint]
        L.g1o_uniform.restype = C.c_float
        L.g1o_rollout_soa.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(Config),
                                      C.POINTER(RolloutParams), _dp, _dp, _dp, _dp, _dp, _dp,
                                      C.POINTER(C.c_int)]
        L.g1o_draw_targets.argtypes = [C.c_int, C.c_uint, C.c_int, C.c_float, _fp]
        L.g1o_branch_margin_soa.argtypes = [C.c_int, C.POINTER(Config)] + [_dp] * 7

    # -- reference host ABI names ------------------------------------------
    def sizes(self):
        v = [C.c_int() for _ in range(5)]
        prec = self.lib.g1_sizes(*[C.byref(x) for x in v])
        return prec, tuple(x.value for x in v)

    def fk(self, qpos):
        qpos = np.ascontiguousarray(qpos, dtype=np.float64)
        xpos = np.zeros(NB * 3)
        xmat = np.zeros(NB * 9)
        self.lib.g1_c_fk(_p(qpos), _p(xpos), _p(xmat))
        return xpos.reshape(NB, 3), xmat.reshape(NB, 9)

    def fd(self, qpos, qvel, tau):
        qpos, qvel, tau = (np.ascontiguousarray(a, dtype=np.float64) for a in (qpos, qvel, tau))
        qacc = np.zeros(NV)
        self.lib.g1_c_fd(_p(qpos), _p(qvel), _p(tau), _p(qacc))
        return qacc

    def c_step(self, qpos, qvel, ctrl, nsub, dt, anchor):
        """In place on qpos / qvel / anchor (float64), returns fn[8]."""
        fn = np.zeros(NC)
        self.lib.g1_c_step(_p(_need(qpos, np.float64)), _p(_need(qvel, np.float64)),
                           _p(np.ascontiguousarray(ctrl, dtype=np.float64)), int(nsub),
                           float(dt), _p(fn), _p(_need(anchor, np.float64)))
        return fn

    # -- extended ------------------------------------------------------------
    @staticmethod
    def config(dt=1e-3, **kw):
        c = Config()
        c.gravity_z, c.contact_kn, c.contact_dn, c.contact_kt = -9.81, 2e4, 280.0, 1e4
        c.contact_dt, c.limit_kp, c.limit_kd, c.dt = 280.0, 200.0, 5.0, dt
        for k, v in kw.items():
            setattr(c, k, v)
        return c

    def step_soa(self, nsub, cfg, qpos, qvel, anchor, ctrl, mu=None, dmass=None,
                 kp_scale=None, kd_scale=None, outputs=True):
        """SoA float64 batch step, in place on qpos/qvel/anchor.
        Returns (foot_pos, foot_vel, contact_forces) arrays (6|8, nenv)."""
        nenv = qpos.shape[1]
        for a in (qpos, qvel, anchor):
            _need(a, np.float64)
        ctrl = np.ascontiguousarray(ctrl, dtype=np.float64)
        opt = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
               for a in (mu, dmass, kp_scale, kd_scale)]
        fp = np.zeros((6, nenv)) if outputs else None
        fv = np.zeros((6, nenv)) if outputs else None
        cf = np.zeros((NC, nenv)) if outputs else None
        self.lib.g1o_step_soa(nenv, int(nsub), C.byref(cfg), _p(qpos), _p(qvel), _p(anchor),
                              _p(ctrl), *[_p(a) for a in opt], _p(fp), _p(fv), _p(cf))
        return fp, fv, cf

    def branch_margin(self, cfg, qpos, qvel, anchor, ctrl, mu=None, dmass=None):
        """Per-env normalised distance of the next substep from a branch threshold."""
        nenv = qpos.shape[1]
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (qpos, qvel, anchor, ctrl)]
        opt = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (mu, dmass)]
        out = np.zeros(nenv)
        self.lib.g1o_branch_margin_soa(nenv, C.byref(cfg), *[_p(a) for a in arrs], *[_p(a) for a in opt], _p(out))
        return out

    def reset_done_soa(self, qpos, qvel, anchor, done, seed, noise, drop):
        nenv = qpos.shape[1]
        done = np.ascontiguousarray(done, dtype=np.uint8)
        self.lib.g1o_reset_done_soa(nenv, _p(qpos), _p(qvel), _p(anchor),
                                    done.ctypes.data_as(C.POINTER(C.c_uint8)),
                                    int(seed) & 0xffffffff, float(noise), float(drop))

    def hash(self, x):
        return self.lib.g1o_hash(int(x) & 0xffffffff)

    def uniform(self, seed, stream, counter):
        return self.lib.g1o_uniform(seed & 0xffffffff, stream & 0xffffffff, counter & 0xffffffff)

    def draw_targets(self, nenv, seed, step, frac=0.3):
        out = np.zeros((NU, nenv), dtype=np.float32)
        self.lib.g1o_draw_targets(nenv, int(seed) & 0xffffffff, int(step), float(frac), _p(out, _fp))
        return out

    def rollout_soa(self, npolicy, decim, cfg, rp, qpos, qvel, anchor, ctrl, mu=None,
                    dmass=None, reset_count=None):
        nenv = qpos.shape[1]
        for a in (qpos, qvel, anchor, ctrl):
            _need(a, np.float64)
        opt = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (mu, dmass)]
        rc = _p(reset_count, C.POINTER(C.c_int)) if reset_count is not None else None
        self.lib.g1o_rollout_soa(nenv, int(npolicy), int(decim), C.byref(cfg), C.byref(rp),
                                 _p(qpos), _p(qvel), _p(anchor), _p(ctrl), *[_p(a) for a in opt], rc)


class RefHost:
    """The reference's own FP64 (or FP32) host_lib.cpp build in oracle/_ref/."""

    def __init__(self, precision=8):
        name = "libg1host.so" if precision == 8 else "libg1host32.so"
        path = os.path.join(REF, name)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = self.lib = C.CDLL(path)
        L.g1_c_fk.argtypes = [_dp, _dp, _dp]
        L.g1_c_fd.argtypes = [_dp, _dp, _dp, _dp]
        L.g1_c_step.argtypes = [_dp, _dp, _dp, C.c_int, C.c_double, _dp, _dp]

    def sizes(self):
        v = [C.c_int() for _ in range(5)]
        prec = self.lib.g1_sizes(*[C.byref(x) for x in v])
        return prec, tuple(x.value for x in v)

    fk = Oracle.fk
    fd = Oracle.fd
    c_step = Oracle.c_step


class RefKernelCPU:
    """The reference's GPU-ABI kernels compiled for the CPU (oracle/_ref/libg1cuda_cpu.so)."""

    def __init__(self):
        path = os.path.join(REF, "libg1cuda_cpu.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = self.lib = C.CDLL(path)
        L.ref_cuda_step.argtypes = [C.c_int, C.c_int] + [_fp] * 7
        L.ref_cuda_reset_done.argtypes = [C.c_int, _fp, _fp, _fp, C.POINTER(C.c_uint8),
                                          C.c_uint, C.c_float, C.c_float]

    def step(self, nsub, qpos, qvel, anchor, ctrl):
        nenv = qpos.shape[1]
        fp = np.zeros((6, nenv), np.float32)
        fv = np.zeros((6, nenv), np.float32)
        cf = np.zeros((NC, nenv), np.float32)
        ctrl = np.ascontiguousarray(ctrl, dtype=np.float32)
        self.lib.ref_cuda_step(nenv, nsub, _p(qpos, _fp), _p(qvel, _fp), _p(anchor, _fp),
                               _p(ctrl, _fp), _p(fp, _fp), _p(fv, _fp), _p(cf, _fp))
        return fp, fv, cf

    def reset_done(self, qpos, qvel, anchor, done, seed, noise, drop):
        nenv = qpos.shape[1]
        done = np.ascontiguousarray(done, dtype=np.uint8)
        self.lib.ref_cuda_reset_done(nenv, _p(qpos, _fp), _p(qvel, _fp), _p(anchor, _fp),
                                     done.ctypes.data_as(C.POINTER(C.c_uint8)),
                                     int(seed) & 0xffffffff, float(noise), float(drop))
