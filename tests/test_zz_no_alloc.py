"""g1b_adjoint_noalloc: the horizon adjoint for callers that cannot allocate.

Some callers cannot call cudaMalloc (a real-time loop that reserves all
device memory at start-up, or a host whose device memory belongs to another
allocator and that cannot pass a buffer).  g1b_adjoint_noalloc serves them
with its workspace in a fixed device array inside the library.  These tests
call it through the C-ABI and check, on two calls in a row with different
problem sizes, that it returns what g1b_adjoint returns with caller
scratch, and that a problem larger than the fixed array is refused.

This file is collected last on purpose: it must pass both alone in a fresh
process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from g1sim_b200 import _lib
from g1sim_b200 import adjoint as A
from g1sim_b200.model import g1_model_data as M

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def bind():
    L = _lib.lib()
    vp = C.c_void_p
    L.g1b_adjoint_noalloc.argtypes = [C.c_int, C.POINTER(_lib.Config), C.POINTER(_lib.AdjointProblem)] + [vp] * 13
    L.g1b_adjoint_noalloc.restype = C.c_int
    L.g1b_adjoint_noalloc_capacity.argtypes = []
    L.g1b_adjoint_noalloc_capacity.restype = C.c_size_t
    return L


def inputs(golden_host, n, H, seed):
    rng = np.random.default_rng(seed)
    q0 = np.repeat(golden_host["settle_qpos"][:, None], n, axis=1)
    v0 = np.repeat(golden_host["settle_qvel"][:, None], n, axis=1)
    a0 = np.repeat(golden_host["settle_anchor"][:, None], n, axis=1)
    q0[7:] += rng.normal(0, 0.01, size=(29, n))
    tg = np.asarray(M.qpos_stand)[7:][None, :, None] + rng.normal(0, 0.05, size=(H, 29, n))
    t = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=torch.float32, device=DEV)  # noqa: E731
    return dict(tg=t(tg), kp=t(rng.uniform(0.8, 1.2, n)), kd=t(rng.uniform(0.8, 1.2, n)), q0=t(q0), v0=t(v0),
                a0=t(a0))


def call_noalloc(L, x, H, ckpt):
    n = x["q0"].shape[1]
    out = dict(loss=torch.empty(n, device=DEV), grad_targets=torch.empty_like(x["tg"]),
               grad_kp=torch.empty(n, device=DEV), grad_kd=torch.empty(n, device=DEV),
               grad_qpos0=torch.empty(36, n, device=DEV), grad_qvel0=torch.empty(35, n, device=DEV))
    cfg = _lib.default_config(dt=2e-3)
    pr = _lib.AdjointProblem(H, ckpt, 0.78, 0.1)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    rc = L.g1b_adjoint_noalloc(n, C.byref(cfg), C.byref(pr), p(x["q0"]), p(x["v0"]), p(x["a0"]), p(x["tg"]),
                               p(x["kp"]), p(x["kd"]), p(out["loss"]), p(out["grad_targets"]), p(out["grad_kp"]),
                               p(out["grad_kd"]), p(out["grad_qpos0"]), p(out["grad_qvel0"]),
                               C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream))
    return rc, out


def test_noalloc_matches_scratch_entry_point_twice(golden_host):
    L = bind()
    # two calls in a row, different sizes: the second must not see the first's workspace
    for n, H, ckpt, seed in ((24, 16, 4, 1), (40, 24, 8, 2)):
        x = inputs(golden_host, n, H, seed)
        rc, got = call_noalloc(L, x, H, ckpt)
        assert rc == 0, _lib.last_error()
        ref = A.horizon_adjoint(x["tg"], x["kp"], x["kd"], x["q0"], x["v0"], x["a0"], checkpoint=ckpt)
        torch.cuda.synchronize()
        for k in ref:
            a, b = got[k].cpu().numpy(), ref[k].cpu().numpy()
            assert np.all(np.isfinite(a)), k
            assert np.all(np.abs(a - b) <= 1e-6 * np.maximum(np.abs(b), 1.0)), k


def test_noalloc_rejects_problems_beyond_the_fixed_workspace(golden_host):
    L = bind()
    cap = L.g1b_adjoint_noalloc_capacity()
    assert cap == 1 << 21
    H, ckpt = 64, 8
    per_env = A.scratch_size(1, H, ckpt)  # (H / C + 1 + C) * 87 floats per env
    n = cap // per_env + 1  # one env too many
    x = inputs(golden_host, 2, H, 3)
    cfg = _lib.default_config(dt=2e-3)
    pr = _lib.AdjointProblem(H, ckpt, 0.78, 0.1)
    rc = L.g1b_adjoint_noalloc(n, C.byref(cfg), C.byref(pr), *([None] * 13), None)
    assert rc != 0
    assert "more than the fixed" in _lib.last_error()
    # the largest problem that fits is accepted (one call, outputs sized for it)
    x = inputs(golden_host, n - 1, H, 4)
    rc, out = call_noalloc(L, x, H, ckpt)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert torch.isfinite(out["loss"]).all()
