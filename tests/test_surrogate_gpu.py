"""Dynamics surrogate on the GPU (needs a B200).

  * g1b_gemm_bf16 (tcgen05, BF16 operands, FP32 accumulation) against an FP64
    CPU product of the same BF16 values, single pass and split over K with
    atomics, to 1e-5 relative;
  * the training kernels (forward, loss, backward, input gradient) against a
    CPU FP64 restatement of the same network with the same BF16 rounding
    points, to 3e-3 relative in 2-norm (the two sides may round a hidden
    activation to neighbouring BF16 values when their sums differ in the
    last bits);
  * Adam against its published update rule on the CPU, over three steps of
    the fused optimiser launch (device step count and learning rate);
  * training steps replayed from the captured CUDA graph equal eager ones;
  * training on transitions of the randomised workload lowers the loss;
  * the fallback rollout with bound 0 is the exact step, bit for bit, and
    with the trained network stays finite;
  * across a foot touchdown the exact step's d qacc_z / d z jumps (contact
    stiffness switching on) while the surrogate's, from its backward
    kernels, varies smoothly -- the smooth gradient the surrogate provides;
  * the adjoint kernels' gradient of a one-step loss with respect to the
    targets and the trained surrogate's (its input-gradient kernels) agree in
    direction (cosine > 0.8 over 1,024 envs mid-rollout), and an untrained
    surrogate's does not;
  * the device features equal the host build of g1_surfeat.cuh (the one
    whose products tests/test_surrogate_derivation.py checks);
  * the gradient through a 10-step surrogate rollout (feature, network and
    update products) matches central differences of that rollout;
  * short-horizon target refinement with the surrogate's gradient, judged
    by the exact step, lowers the exact objective of standing envs over a
    100 ms horizon well below the policy's unrefined targets (measured 47 %
    lower; the exact adjoint's gradient on the same budget: 51 %).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from g1sim_b200 import _lib
from g1sim_b200 import g1sim as G
from g1sim_b200 import surrogate as S
from g1sim_b200.model import g1_model_data as M

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def bf(x):
    return x.to(torch.bfloat16)


@pytest.mark.parametrize("M_,N,K,splits", [(256, 512, 512, 1), (128, 64, 512, 1), (384, 128, 128, 1),
                                           (128, 512, 8192, 16), (512, 128, 4096, 8), (128, 16, 128, 1),
                                           (256, 48, 256, 1), (256, 48, 512, 2)])
def test_gemm_matches_fp64(M_, N, K, splits):
    g = torch.Generator(device=DEV).manual_seed(M_ + N + K)
    A = bf(torch.randn(M_, K, device=DEV, generator=g))
    B = bf(torch.randn(N, K, device=DEV, generator=g))
    # the bias holds exactly N floats, followed by NaN: a read past its end shows in C
    fence = torch.full((N + 64,), float("nan"), device=DEV)
    fence[:N] = torch.randn(N, device=DEV, generator=g)
    bias = fence[:N]
    C_ = torch.full((M_, N), 7.0, device=DEV)
    S.gemm(A, B, C_, bias=bias, splits=splits)
    torch.cuda.synchronize()
    assert S.gemm_status() == 0
    ref = A.double().cpu() @ B.double().cpu().T + bias.double().cpu()
    err = ((C_.double().cpu() - ref).norm() / ref.norm()).item()
    assert err < 1e-5, err


@pytest.mark.parametrize("M_,N,K,splits", [(20480, 512, 512, 1), (512, 192, 16384, 16), (256, 192, 64000, 4),
                                           (128, 64, 2368, 2)])
def test_gemm_many_tiles_per_cta(M_, N, K, splits):
    """More tiles than SMs: every CTA reuses both tensor-memory accumulators
    and the operand ring several times; split (stream-K), the CTAs' shares of
    (tile, K chunk) pairs cut tiles at arbitrary chunks (2,000 chunks over
    the SMs) or hold one chunk each (37 chunks), and meet in C atomically."""
    g = torch.Generator(device=DEV).manual_seed(M_ + N)
    A = bf(torch.randn(M_, K, device=DEV, generator=g))
    B = bf(torch.randn(N, K, device=DEV, generator=g))
    C_ = torch.empty(M_, N, device=DEV)
    S.gemm(A, B, C_, splits=splits)
    torch.cuda.synchronize()
    assert S.gemm_status() == 0
    ref = A.double() @ B.double().T
    err = ((C_.double() - ref).norm() / ref.norm()).item()
    assert err < 1e-5, err


@pytest.mark.parametrize("M_,N,K", [(512, 512, 4096), (512, 512, 65536), (64, 512, 8192), (512, 192, 2048),
                                    (208, 64, 256), (1024, 768, 1024), (16, 64, 64)])
def test_gemm_atb_matches_fp64(M_, N, K):
    """C += A^T B from row-major A [K, M] and B [K, N] (MN-major tiles, K
    split over the SMs): the weight-gradient shapes of the surrogate (the
    output layer's M = 64 and the row tiles' zero-filled second half, the
    first layer's N = 192 in three 64-column boxes, K = 65,536), a partial
    row tile (M = 208), N above 256.  The operands sit in wider buffers whose
    extra columns hold NaN, and C in a buffer whose extra rows and columns
    hold 7: a read past M or N, or a write past C, shows."""
    g = torch.Generator(device=DEV).manual_seed(M_ + 3 * N + K)
    Abuf = torch.full((K, M_ + 16), float("nan"), dtype=torch.bfloat16, device=DEV)
    Bbuf = torch.full((K, N + 8), float("nan"), dtype=torch.bfloat16, device=DEV)
    A, B = Abuf[:, :M_], Bbuf[:, :N]
    A.copy_(bf(torch.randn(K, M_, device=DEV, generator=g)))
    B.copy_(bf(torch.randn(K, N, device=DEV, generator=g)))
    Cbuf = torch.full((M_ + 8, N + 4), 7.0, device=DEV)
    C_ = Cbuf[:M_, :N]
    C0 = torch.randn(M_, N, device=DEV, generator=g)
    C_.copy_(C0)
    S.gemm_atb(A, B, C_)
    torch.cuda.synchronize()
    assert S.gemm_status() == 0
    ref = C0.double() + A.double().T @ B.double()
    err = ((C_.double() - ref).norm() / ref.norm()).item()
    assert err < 1e-5, err
    assert bool((Cbuf[M_:] == 7.0).all()) and bool((Cbuf[:, N:] == 7.0).all())


def test_gemm_atb_rejects_bad_shapes():
    A = torch.zeros(128, 64, dtype=torch.bfloat16, device=DEV)
    C_ = torch.zeros(64, 48, device=DEV)
    with pytest.raises(RuntimeError):
        S.gemm_atb(A, torch.zeros(128, 48, dtype=torch.bfloat16, device=DEV), C_)  # N % 64
    C_ = torch.zeros(64, 64, device=DEV)
    with pytest.raises(RuntimeError):
        S.gemm_atb(A[:100], torch.zeros(100, 64, dtype=torch.bfloat16, device=DEV), C_)  # K % 64


def _bf16_close(got, ref):
    """got (BF16) is ref rounded to BF16, up to one unit in the last place
    (the FP32 sums of the kernel and the FP64 reference may straddle a
    rounding boundary), plus the FP32 accumulation error near zero."""
    tol = ref.abs() * 2.0 ** -7 + 1e-5 * ref.abs().mean()
    return bool(((got.double() - ref).abs() <= tol).all())


@pytest.mark.parametrize("M_,N,K", [(256, 512, 512), (20480, 512, 512), (384, 192, 128), (128, 48, 64)])
def test_linear_silu_fused_epilogue(M_, N, K):
    """z = A W^T + b, Z = fp16(z), H = bf16(silu(z)), Ht = H^T in one kernel,
    against FP64."""
    g = torch.Generator(device=DEV).manual_seed(3 * M_ + N)
    A = bf(torch.randn(M_, K, device=DEV, generator=g))
    W = bf(torch.randn(N, K, device=DEV, generator=g) / K ** 0.5)
    fence = torch.full((N + 64,), float("nan"), device=DEV)
    fence[:N] = torch.randn(N, device=DEV, generator=g)
    bias = fence[:N]
    Z = torch.full((M_, N), 7.0, dtype=torch.float16, device=DEV)
    H = torch.zeros(M_, N, dtype=torch.bfloat16, device=DEV)
    Ht = torch.zeros(N, M_, dtype=torch.bfloat16, device=DEV)
    S.linear_silu(A, W, bias, H, Z=Z, Ht=Ht)
    torch.cuda.synchronize()
    assert S.gemm_status() == 0
    zref = A.double() @ W.double().T + bias.double()
    # FP16 rounding (relative 2^-11) of the FP32 sum
    assert ((Z.double() - zref).abs() <= zref.abs() * 2.0 ** -11 + 1e-5 * zref.abs().mean()).all()
    assert _bf16_close(H, zref * torch.sigmoid(zref))
    assert torch.equal(Ht, H.T)
    # without the optional outputs: the same H
    H2 = torch.zeros_like(H)
    S.linear_silu(A, W, bias, H2)
    torch.cuda.synchronize()
    assert torch.equal(H2, H)


@pytest.mark.parametrize("M_,N,K", [(256, 512, 512), (20480, 512, 512), (384, 192, 512), (128, 48, 64),
                                    (256, 768, 256)])
def test_linear_silu_bwd_fused_epilogue(M_, N, K):
    """g = (dZ Wt^T) * silu'(Z), dH = bf16(g), dHt = dH^T, db += column sums of
    g in one kernel, against FP64 (N = 768: three column tiles)."""
    g = torch.Generator(device=DEV).manual_seed(5 * M_ + N)
    dZ = bf(torch.randn(M_, K, device=DEV, generator=g))
    Wt = bf(torch.randn(N, K, device=DEV, generator=g) / K ** 0.5)
    Z = (torch.randn(M_, N, device=DEV, generator=g) * 2).half()
    dH = torch.zeros(M_, N, dtype=torch.bfloat16, device=DEV)
    dHt = torch.zeros(N, M_, dtype=torch.bfloat16, device=DEV)
    db = torch.full((N,), 0.25, device=DEV)
    S.linear_silu_bwd(dZ, Wt, Z, dH, dHt=dHt, db=db)
    torch.cuda.synchronize()
    assert S.gemm_status() == 0
    z = Z.double()
    s = torch.sigmoid(z)
    gref = (dZ.double() @ Wt.double().T) * s * (1 + z * (1 - s))
    assert _bf16_close(dH, gref)
    assert torch.equal(dHt, dH.T)
    dbref = gref.sum(0) + 0.25
    assert ((db.double() - dbref).abs().max() / dbref.abs().max()).item() < 1e-5


def test_linear_silu_rejects_aliasing_and_bad_shapes():
    A = torch.zeros(128, 64, dtype=torch.bfloat16, device=DEV)
    W = torch.zeros(64, 64, dtype=torch.bfloat16, device=DEV)
    Z = torch.zeros(128, 64, dtype=torch.float16, device=DEV)
    with pytest.raises(RuntimeError, match="alias"):
        S.linear_silu_bwd(A, W, Z, A)
    with pytest.raises(RuntimeError, match="M % 128"):
        S.linear_silu(A[:96], W, None, torch.zeros(96, 64, dtype=torch.bfloat16, device=DEV))


@pytest.mark.parametrize("B", [4096, 300])
def test_loss_kernel(B):
    """Weighted MSE, its BF16 gradient and transpose, bias-gradient sums and
    the loss, against torch: 4,096 rows (16-byte transposed stores) and 300
    (a partial block, the element-wise fallback)."""
    g = torch.Generator(device=DEV).manual_seed(B)
    Y = torch.randn(B, 64, device=DEV, generator=g)
    T = torch.randn(B, 64, device=DEV, generator=g)
    w = torch.rand(64, device=DEV, generator=g)
    dY = torch.zeros(B, 64, dtype=torch.bfloat16, device=DEV)
    dYt = torch.zeros(64, B, dtype=torch.bfloat16, device=DEV)
    db = torch.full((64,), 0.5, device=DEV)
    loss = torch.full((1,), 2.0, device=DEV)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    _lib.check(_lib.lib().g1b_sur_loss(B, 64, p(Y), p(T), p(w), p(dY), p(dYt), p(db), p(loss),
                                       C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)), "g1b_sur_loss")
    torch.cuda.synchronize()
    e = Y - T
    grad = 2.0 * w * e / B
    assert torch.equal(dY, grad.to(torch.bfloat16))
    assert torch.equal(dYt, dY.T)
    assert torch.allclose(db, grad.sum(0) + 0.5, rtol=1e-5, atol=1e-6)
    ref = (w.double() * e.double() ** 2).sum() / B + 2.0
    assert abs(loss.item() - ref.item()) <= 1e-5 * abs(ref.item())
    # without the transposed copy (the training step's form): the same dY
    dY2 = torch.zeros_like(dY)
    _lib.check(_lib.lib().g1b_sur_loss(B, 64, p(Y), p(T), p(w), p(dY2), None, p(db), p(loss),
                                       C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)), "g1b_sur_loss")
    torch.cuda.synchronize()
    assert torch.equal(dY2, dY)


def cpu_reference(sur, X, T):
    """FP64 restatement of forward + weighted-MSE loss + backward with the
    kernels' rounding points (BF16 operands of every product, the FP16
    pre-activation of the SiLU derivative)."""
    r = lambda x: x.to(torch.bfloat16).double()  # noqa: E731
    Ws = [r(w.cpu()) for w in sur.W]
    bs = [b.cpu().double() for b in sur.b]
    x = X.cpu().double()
    hs, zs = [x], []
    for i in range(5):
        z = hs[-1] @ Ws[i].T + bs[i]
        zs.append(z)
        if i < 4:
            hs.append(r(z * torch.sigmoid(z)))
    B = X.shape[0]
    w = sur.out_w.cpu().double()
    e = zs[4] - T.cpu().double()
    loss = (w * e * e).sum() / B
    dz = r(2 * w * e / B)
    gW, gb = [None] * 5, [None] * 5
    gb[4] = (2 * w * e / B).sum(0)
    for i in range(4, -1, -1):
        gW[i] = dz.T @ hs[i]
        if i > 0:
            dh = dz @ Ws[i]
            zh = zs[i - 1].float().clamp(-65000, 65000).half().double()  # the FP16 pre-activation kept
            s = torch.sigmoid(zh)
            g = dh * s * (1 + zh * (1 - s))
            gb[i - 1] = g.sum(0)
            dz = r(g)
        else:
            dx = dz @ Ws[0]
    return loss, gW, gb, dx


def test_training_kernels_match_cpu_restatement():
    sur = S.Surrogate(DEV, seed=1)
    with torch.no_grad():
        for b in sur.b:
            b.uniform_(-0.1, 0.1)
    g = torch.Generator(device=DEV).manual_seed(2)
    B = 256
    X = bf(torch.randn(B, S.NIN, device=DEV, generator=g))
    X[:, S.NFEAT:] = 0
    T = torch.randn(B, 64, device=DEV, generator=g)
    sur.forward(X, keep=True)
    loss = sur.backward(X, T, want_dx=True)
    torch.cuda.synchronize()
    assert S.gemm_status() == 0
    l_ref, gW, gb, dx = cpu_reference(sur, X, T)
    assert abs(loss.item() - l_ref.item()) <= 1e-4 * abs(l_ref.item())
    rel = lambda a, b: ((a.double().cpu() - b).norm() / b.norm()).item()  # noqa: E731
    for i in range(5):
        out = sur.W[i].shape[0]
        assert rel(sur.gW[i][:out], gW[i]) < 3e-3, (i, rel(sur.gW[i][:out], gW[i]))
        assert rel(sur.gb[i], gb[i]) < 3e-3, (i, rel(sur.gb[i], gb[i]))
    assert rel(sur.dX(B), dx) < 3e-3


def test_adam_matches_update_rule():
    sur = S.Surrogate(DEV, seed=3)
    w0 = [w.clone() for w in sur.W]
    for gw in sur.gW:
        gw.normal_()
    for gb in sur.gb:
        gb.normal_()
    b0 = [b.clone() for b in sur.b]
    g0 = [gw.clone() for gw in sur.gW] + [gb.clone() for gb in sur.gb]
    sur.adam(lr=1e-2)
    torch.cuda.synchronize()
    for p_new, p_old, g in zip(sur.W + sur.b, w0 + b0, g0):
        m = 0.1 * g
        v = 0.001 * g * g
        ref = p_old - 1e-2 * (m / 0.1) / (torch.sqrt(v / 0.001) + 1e-8)
        assert torch.allclose(p_new, ref, rtol=1e-5, atol=1e-6)
    # BF16 copies and transposes of every layer refreshed
    for i in range(5):
        assert torch.equal(sur.Wb[i], sur.W[i].to(torch.bfloat16))
        assert torch.equal(sur.Wt[i], sur.W[i].T.contiguous().to(torch.bfloat16))


@pytest.mark.parametrize("shapes", [[(40, 70), (37, 5)], [(64, 128), (8, 64), (33, 200), (96, 192)]])
def test_adam_cast_partial_tiles(shapes):
    """The fused optimiser launch on weights that do not fill its 32 x 64
    tiles, with row counts that are not multiples of 8 (element-wise
    transposed stores) beside full tiles (16-byte runs), several layers and
    their biases in one launch, against Adam's first step."""
    g = torch.Generator(device=DEV).manual_seed(len(shapes))
    keep, layers = [], []
    for r, c in shapes:
        t = dict(W=torch.randn(r, c, device=DEV, generator=g), b=torch.randn(r, device=DEV, generator=g),
                 mW=torch.zeros(r, c, device=DEV), vW=torch.zeros(r, c, device=DEV), mb=torch.zeros(r, device=DEV),
                 vb=torch.zeros(r, device=DEV), gW=torch.randn(r, c, device=DEV, generator=g),
                 gb=torch.randn(r, device=DEV, generator=g), Wb=torch.empty(r, c, dtype=torch.bfloat16, device=DEV),
                 Wt=torch.empty(c, r, dtype=torch.bfloat16, device=DEV))
        t["W0"], t["b0"] = t["W"].clone(), t["b"].clone()
        keep.append(t)
        layers.append(_lib.SurLayer(*[t[k].data_ptr() for k in ("W", "b", "mW", "vW", "mb", "vb", "gW", "gb",
                                                                 "Wb", "Wt")], r, c))
    arr = (_lib.SurLayer * len(layers))(*layers)
    step = torch.ones(1, dtype=torch.int32, device=DEV)
    lr = torch.full((1,), 1e-2, device=DEV)
    _lib.check(_lib.lib().g1b_sur_adam_cast(len(layers), arr, C.c_void_p(step.data_ptr()), C.c_void_p(lr.data_ptr()),
                                            0.9, 0.999, 1e-8,
                                            C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)),
               "g1b_sur_adam_cast")
    torch.cuda.synchronize()
    for t in keep:
        for p_new, p_old, gr in ((t["W"], t["W0"], t["gW"]), (t["b"], t["b0"], t["gb"])):
            ref = p_old - 1e-2 * gr / (gr.abs() + 1e-8)  # t = 1: m / c1 = g, sqrt(v / c2) = |g|
            assert torch.allclose(p_new, ref, rtol=1e-5, atol=1e-6)
        assert torch.equal(t["Wb"], t["W"].to(torch.bfloat16))
        assert torch.equal(t["Wt"], t["W"].T.contiguous().to(torch.bfloat16))


def test_adam_bias_correction_over_steps():
    """Three steps of the fused optimiser launch (step count and learning
    rate in device memory) against Adam's update rule with t = 1, 2, 3."""
    sur = S.Surrogate(DEV, seed=4)
    w = sur.W[1].clone().double()
    m = torch.zeros_like(w)
    v = torch.zeros_like(w)
    g = torch.Generator(device=DEV).manual_seed(5)
    for t, lr in ((1, 1e-2), (2, 5e-3), (3, 2e-3)):
        gw = torch.randn(sur.W[1].shape, device=DEV, generator=g)
        sur.gW[1].copy_(gw)
        sur.adam(lr=lr)
        torch.cuda.synchronize()
        m = 0.9 * m + 0.1 * gw.double()
        v = 0.999 * v + 0.001 * gw.double() ** 2
        w = w - lr * (m / (1 - 0.9 ** t)) / (torch.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
        assert torch.allclose(sur.W[1].double(), w, rtol=1e-5, atol=1e-6), t
    assert int(sur.opt_step.item()) == 3 and sur.step_n == 3
    assert torch.equal(sur.Wt[1], sur.W[1].T.contiguous().to(torch.bfloat16))


def test_train_graph_replays_the_eager_step():
    """Training steps replayed from the captured CUDA graph give the weights
    of the same steps launched eagerly, up to the order of the atomic sums:
    Adam's normalised update turns that noise (and the BF16 activations it
    can flip) into weight differences of up to a few 1e-5 where a gradient
    is small, and an entry whose gradient changes sign can move by up to
    2 lr.  So every tensor agrees to 1e-3 relative in norm (measured ~1e-5)
    and no entry differs by more than twice the summed learning rates; a
    replay with a stale learning rate would be off by 2e-4 - 6e-4 per step
    almost everywhere, a few percent of the weights' norm."""
    B = 4096
    g = torch.Generator(device=DEV).manual_seed(6)
    X = bf(torch.randn(B, S.NIN, device=DEV, generator=g))
    X[:, S.NFEAT:] = 0
    T = torch.randn(B, 64, device=DEV, generator=g)
    a, b = S.Surrogate(DEV, seed=7), S.Surrogate(DEV, seed=7)
    lrs = [1e-3, 8e-4, 6e-4, 4e-4]
    for lr in lrs:
        la = float(a.train_step(X, T, lr=lr).item())
    tg = b.capture_train_step(X, T, lrs[0])  # runs the first step eagerly
    for lr in lrs[1:]:
        lb = float(tg.step(lr).item())
    torch.cuda.synchronize()
    assert S.gemm_status() == 0
    assert a.step_n == b.step_n == len(lrs) and int(b.opt_step.item()) == len(lrs)
    assert abs(la - lb) <= 1e-5 * abs(la)
    for wa, wb in zip(a.W + a.b, b.W + b.b):
        d = (wa - wb).abs()
        assert d.norm().item() <= 1e-3 * wa.norm().item()
        assert d.max().item() <= 2 * sum(lrs)


@pytest.fixture(scope="module")
def trained():
    sur = S.Surrogate(DEV, seed=0)
    F, A = S.generate_transitions(sur, 8192, 60, DEV, seed=0)
    S.fit_normalisation(sur, F, A)
    X, T = S.normalise(sur, F[:16384], A[:16384])
    sur.forward(X, keep=True)
    l0 = sur.backward(X, T).item()
    hist = S.train(sur, F, A, steps=400, batch=16384, lr=1e-3)
    sur.forward(X, keep=True)
    l1 = sur.backward(X, T).item()
    torch.cuda.synchronize()
    return sur, l0, l1


def test_training_lowers_the_loss(trained):
    sur, l0, l1 = trained
    print(f"surrogate loss (normalised qacc MSE): before {l0:.4f}, after 400 steps {l1:.4f}")
    assert S.gemm_status() == 0
    assert np.isfinite(l1) and l1 < 0.5 * l0


def make_state(n, seed=0):
    from g1sim_b200 import workloads
    w = workloads.randomized(nenv=n, seed=seed)
    s = {k: torch.tensor(w[k], dtype=torch.float32, device=DEV) for k in ("qpos", "qvel", "anchor", "ctrl")}
    s["contact_forces"] = torch.zeros(8, n, device=DEV)
    return s


def test_fallback_rollout(trained):
    sur, _, _ = trained
    n = 1024
    cfg = _lib.default_config(dt=2e-3)
    a, b = make_state(n), make_state(n)
    frac, _ = S.rollout_with_fallback(sur, a, 20, bound=0.0)
    for _ in range(20):
        G.step(b["qpos"], b["qvel"], b["anchor"], b["ctrl"], 1, config=cfg, contact_forces=b["contact_forces"])
    assert frac == 0.0
    assert torch.equal(a["qpos"], b["qpos"]) and torch.equal(a["qvel"], b["qvel"])
    c = make_state(n, seed=1)
    frac, st = S.rollout_with_fallback(sur, c, 50, bound=1e-3)
    print(f"fallback rollout: {100 * frac:.1f} % of env-steps within 1e-3 of the exact step, one-step error {st}")
    assert torch.isfinite(c["qpos"]).all() and 0.0 <= frac <= 1.0


def test_surrogate_gradient_is_smooth_across_touchdown(trained, oracle):
    """d qacc_z / d z of the exact step (FP64 oracle, central differences)
    jumps where the lowest foot sphere touches down; the surrogate's
    derivative (its backward kernels) does not."""
    sur, _, _ = trained
    stand = np.asarray(M.qpos_stand, dtype=np.float64)
    zs = np.linspace(0.745, 0.765, 64)
    h = 1e-7

    def exact_az(z):
        q = stand.copy()
        q[2] = z
        v = np.zeros(35)
        an = np.full(16, 1e30)
        oracle.c_step(q, v, stand[7:].copy(), 1, 2e-3, an)
        return v[2] / 2e-3

    d_exact = np.array([(exact_az(z + h) - exact_az(z - h)) / (2 * h) for z in zs])
    # surrogate: d (predicted qacc_z) / d z through the input-gradient kernel
    n = 128
    q = torch.tensor(np.repeat(stand[:, None], n, axis=1), dtype=torch.float32, device=DEV)
    q[2, :64] = torch.tensor(zs, dtype=torch.float32, device=DEV)
    v = torch.zeros(35, n, device=DEV)
    ct = q[7:].clone()
    X = torch.empty(n, S.NIN, dtype=torch.bfloat16, device=DEV)
    sur.features(q, v, torch.full((16, n), 1e30, device=DEV), ct, X)
    Y = sur.forward(X, keep=True).clone()
    w = torch.zeros(64, device=DEV)
    w[2] = 1.0
    T = Y.clone()
    T[:, 2] -= n / 2.0  # d loss / d Y = e_2 for every row
    sur.backward(X, T, want_dx=True, weights=w)
    zi = 58  # feature index of the base height
    d_sur = (sur.dX(n)[:64, zi] * sur.in_istd[zi] * sur.out_std[2]).double().cpu().numpy()
    jump_exact = np.abs(np.diff(d_exact)).max()
    jump_sur = np.abs(np.diff(d_sur)).max()
    print(f"max step of d qacc_z/dz between z samples: exact {jump_exact:.1f}, surrogate {jump_sur:.2f} (1/s^2)")
    assert jump_exact > 10.0 * max(jump_sur, 1e-3)


def surrogate_vjp(sur, s, V):
    """V^T d qacc / d targets of the trained surrogate at state s, per env:
    V [n, 35] (upstream gradient of the generalised acceleration); returns
    [29, n], through the network's input-gradient products (input_grad)."""
    n = V.shape[0]
    X = torch.zeros(n, S.NIN, dtype=torch.bfloat16, device=DEV)
    sur.features(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], X)
    sur.forward(X, keep=True)
    Vn = torch.zeros(n, 64, device=DEV)
    Vn[:, :S.NOUT] = V * sur.out_std[:S.NOUT]
    dX = sur.input_grad(X, Vn)
    ctl = slice(127, 156)  # the 29 target features
    return (dX[:, ctl] * sur.in_istd[ctl]).T.contiguous()


def test_adjoint_agrees_with_surrogate_gradient(trained):
    """One-step horizon loss L = (z_1 - 0.78)^2 + 0.1 |q_1 - u_0|^2: its
    gradient with respect to the targets u_0 from the adjoint kernels, minus
    the explicit -0.2 (q_1 - u_0) term, is dt^2 (d qacc / d u_0)^T g with g the
    loss gradient at (z_1, q_1).  The trained surrogate's Jacobian gives the
    same contraction; the two agree in direction over envs mid-rollout, and an
    untrained surrogate does not."""
    from g1sim_b200 import adjoint as A
    sur, _, _ = trained
    n, dt, w = 1024, 2e-3, 0.1
    cfg = _lib.default_config(dt=dt)
    s = make_state(n, seed=4)
    for _ in range(40):  # away from the initial drop, through touchdown
        G.step(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], 1, config=cfg, contact_forces=s["contact_forces"])
    nxt = {k: v.clone() for k, v in s.items()}
    G.step(nxt["qpos"], nxt["qvel"], nxt["anchor"], nxt["ctrl"], 1, config=cfg, contact_forces=nxt["contact_forces"])
    ones = torch.ones(n, device=DEV)
    r = A.horizon_adjoint(s["ctrl"][None].contiguous(), ones, ones, s["qpos"], s["qvel"], s["anchor"], checkpoint=1,
                          z_ref=0.78, w_track=w, config=cfg)
    q1, u0 = nxt["qpos"][7:], s["ctrl"]
    g_exact = r["grad_targets"][0] + 2 * w * (q1 - u0)
    V = torch.zeros(n, S.NOUT, device=DEV)
    V[:, 2] = 2 * (nxt["qpos"][2] - 0.78)
    V[:, 6:] = (2 * w * (q1 - u0)).T
    g_sur = dt * dt * surrogate_vjp(sur, s, V)
    untrained = S.Surrogate(DEV, seed=7)
    untrained.in_mean.copy_(sur.in_mean)
    untrained.in_istd.copy_(sur.in_istd)
    untrained.out_mean.copy_(sur.out_mean)
    untrained.out_std.copy_(sur.out_std)
    g_untr = dt * dt * surrogate_vjp(untrained, s, V)
    torch.cuda.synchronize()
    assert S.gemm_status() == 0

    def cos(a, b):
        a, b = a.double().flatten(), b.double().flatten()
        return (a @ b / (a.norm() * b.norm())).item()

    c_tr, c_un = cos(g_exact, g_sur), cos(g_exact, g_untr)
    ratio = (g_sur.norm() / g_exact.norm()).item()
    print(f"adjoint vs surrogate d L / d u_0 (model part): cosine trained {c_tr:.3f}, untrained {c_un:.3f}, "
          f"norm ratio {ratio:.3f}")
    assert torch.isfinite(g_exact).all() and torch.isfinite(g_sur).all()
    assert c_tr > 0.8 and c_tr > c_un + 0.5


def test_device_features_match_host(oracle):
    import ctypes as Cc
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = os.path.join(root, "tests", "native", "_build", "libg1surhost.so")
    if not os.path.exists(lib):
        os.makedirs(os.path.dirname(lib), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++20", "-fPIC", "-shared", "-o", lib,
                        os.path.join(root, "tests", "native", "sur_host.cpp")], check=True)
    L = Cc.CDLL(lib)
    dp = Cc.POINTER(Cc.c_double)
    L.surh_features_d.argtypes = [dp, dp, Cc.c_double, Cc.c_double, dp]
    n = 256
    s = make_state(n, seed=3)
    cfg = _lib.default_config(dt=2e-3)
    for _ in range(60):  # touchdown and contact: stuck anchors
        G.step(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], 1, config=cfg)
    sur = S.Surrogate(DEV, seed=0)
    mu = torch.linspace(0.4, 1.0, n, device=DEV)
    dm = torch.linspace(-1.0, 3.0, n, device=DEV)
    F = torch.zeros(n, S.NIN, device=DEV)
    X = torch.zeros(n, S.NIN, dtype=torch.bfloat16, device=DEV)
    sur.features(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], X, raw=F, mu=mu, dmass=dm)
    torch.cuda.synchronize()
    x = torch.cat([s["qpos"], s["qvel"], s["anchor"]]).double().cpu().numpy()
    u = s["ctrl"].double().cpu().numpy()
    ref = np.zeros((n, 159))
    for e in range(n):
        f = np.zeros(159)
        L.surh_features_d(np.ascontiguousarray(x[:, e]).ctypes.data_as(dp), np.ascontiguousarray(u[:, e]).ctypes.data_as(dp),
                          float(mu[e]), float(dm[e]), f.ctypes.data_as(dp))
        ref[e] = f
    got = F.double().cpu().numpy()[:, :159]
    assert np.all(F[:, 159:].cpu().numpy() == 0)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1.0)
    flags = np.zeros(159, bool)
    flags[72:127:7] = True  # contact flags: equal except within FP32 rounding of depth 0
    assert err[:, ~flags].max() < 2e-5, err[:, ~flags].max()
    assert (got[:, flags] != ref[:, flags]).mean() < 0.01


@pytest.fixture(scope="module")
def trained_big():
    """The surrogate trained as in the benchmark, at a smaller budget."""
    sur = S.Surrogate(DEV, seed=0)
    F, A = S.generate_transitions(sur, 16384, 120, DEV, seed=0)
    S.fit_normalisation(sur, F, A)
    S.train(sur, F, A, steps=1500, batch=32768, lr=2e-3)
    torch.cuda.synchronize()
    return sur


def mid_rollout_state(n, seed=5, steps=200):
    s = make_state(n, seed=seed)
    cfg = _lib.default_config(dt=2e-3)
    G.rollout(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], steps // 10, 10, config=cfg, seed=seed, step0=0)
    torch.cuda.synchronize()
    return s


@pytest.mark.parametrize("H,min_cos,max_rel", [(1, 0.998, 0.06), (4, 0.98, 0.25)])
def test_rollout_gradient_matches_finite_differences(trained_big, H, min_cos, max_rel):
    """d J_sur / d u by backpropagation through an H-step surrogate rollout
    of standing envs (feature, network and update products) against central
    differences of the same rollout along random target directions.  The
    network's inputs are quantised to BF16 (8 mantissa bits), which puts
    noise of ~0.5 quantum / h into a difference quotient, so h = 0.1 rad;
    measured cosine 0.9997 / 0.991 and relative error 0.03 / 0.13 for 1 / 4
    steps (the mismatch shrinks as h grows: rounding, not the products)."""
    sur = trained_big
    n = 512
    s = standing_state(n, seed=4)
    u = s["ctrl"].clone()
    J, g = S.rollout_grad(sur, s, u, H)
    d = torch.randn(29, n, device=DEV, generator=torch.Generator(device=DEV).manual_seed(3))
    d /= d.norm(dim=0, keepdim=True)
    h = 0.1
    Jp, _ = S.rollout_grad(sur, s, u + h * d, H)
    Jm, _ = S.rollout_grad(sur, s, u - h * d, H)
    fd = ((Jp - Jm) / (2 * h)).double()
    ad = (g * d).sum(0).double()
    torch.cuda.synchronize()
    cos = float((fd @ ad) / (fd.norm() * ad.norm()))
    rel = float((fd - ad).norm() / fd.norm())
    print(f"surrogate {H}-step rollout gradient vs central differences (h = {h}): cosine {cos:.4f}, "
          f"relative error {rel:.3f}")
    assert cos > min_cos and rel < max_rel


def standing_state(n, seed=9, settle=200):
    """Drop-test envs settled on the ground (standing on stuck anchors)."""
    from g1sim_b200 import workloads
    w = workloads.drop_test(nenv=n, seed=seed)
    s = {k: torch.tensor(w[k], dtype=torch.float32, device=DEV) for k in ("qpos", "qvel", "anchor", "ctrl")}
    G.step(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], settle, config=_lib.default_config(dt=2e-3))
    torch.cuda.synchronize()
    return s


def test_refinement_gain(trained_big):
    """The targets a policy chose for standing envs (the drop test's noisy
    stand targets) refined over a 100 ms horizon toward the reference base
    height 0.78 m, 10 judged iterations per env."""
    import time
    sur = trained_big
    n, H = 1024, 50
    s = standing_state(n)
    u0 = s["ctrl"].clone()
    J0 = S.exact_objective(s, u0, H, u0=u0, reg=0.1)
    t0 = time.perf_counter()
    _, Js, frac = S.refine_targets(sur, s, u0, H=H, iters=10, mode="surrogate")
    torch.cuda.synchronize()
    ts = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, Je, _ = S.refine_targets(sur, s, u0, H=H, iters=10, mode="exact")
    torch.cuda.synchronize()
    te = time.perf_counter() - t0
    m0, ms, me = float(J0.mean()), float(Js.mean()), float(Je.mean())
    print(f"refinement over {H} substeps, {n} envs: exact objective {m0:.5f} unrefined -> {ms:.5f} with the "
          f"surrogate's gradient ({ts:.2f} s) | {me:.5f} with the exact adjoint's ({te:.2f} s); "
          f"envs improved {float((Js < J0).float().mean()):.3f} / {float((Je < J0).float().mean()):.3f}")
    assert bool((Js <= J0).all())  # the judge never accepts a worse update
    # measured: 0.0632 -> 0.0332 (surrogate) and 0.0310 (exact adjoint)
    assert ms < 0.7 * m0
