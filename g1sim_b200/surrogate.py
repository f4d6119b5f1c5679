"""Learned one-step dynamics surrogate of the G1 step.

An MLP 192 -> 4 x 512 (SiLU) -> 64 over a normalised feature vector of the
state and the PD targets (joint angles and rates, base height, the first two
columns of the base rotation, body-frame base velocities, per foot sphere
its penetration depth, contact flag, offset from its anchor and world
velocity, targets, friction, base-mass offset; 159 used, padded to 192;
csrc/g1_surfeat.cuh) predicting the normalised generalised acceleration of
the step (35 used, padded to 64).  The state delta is dt * qacc for qvel;
qpos follows by the step's semi-implicit Euler (sur_integrate_kernel).

Training runs on the library's own kernels: BF16 tcgen05 GEMMs with FP32
accumulation (g1b_gemm_bf16) for the forward pass, the input-gradient and
the weight-gradient products; element-wise SiLU, SiLU', the loss and its
gradient, Adam and the BF16 weight copies in g1_surrogate.cuh.  Torch only
allocates the buffers and zeroes the gradient accumulators.

The exact step stays the judge: `rollout_with_fallback` advances each env
with the surrogate only where its one-step error against the exact step is
within a bound (1e-3, relative per state component) and with the exact step
elsewhere.

What the surrogate is for is its gradient: `rollout_grad` differentiates a
short-horizon objective through a surrogate rollout (features, network and
state update each have a vector-Jacobian product kernel), which is smooth
across the contact switches where the exact step's derivative jumps.
`refine_targets` uses it for short-horizon refinement of the PD targets a
policy chose, with the exact step as the judge of every update (an update
that does not lower the exact objective is rejected and its step size
halved) and as the fallback (envs whose surrogate one-step error exceeds the
bound take the exact adjoint's gradient).
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from . import g1sim as G
from .model import g1_model_data as M

DIMS = [192, 512, 512, 512, 512, 64]
NFEAT, NOUT, NIN = 159, 35, 192


def train_flops(batch):
    """Floating-point operations of one training step on `batch` rows: the
    forward products, the weight gradients, and the input gradients of every
    layer but the first (a training step needs no d loss / d X)."""
    macs = sum(DIMS[i] * DIMS[i + 1] for i in range(5))
    return 2 * batch * (3 * macs - DIMS[0] * DIMS[1])


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _st(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def gemm(A, B, C_, bias=None, splits=1, acc=False):
    """C = A @ B^T (+ bias): A [M, K], B [N, K] BF16 row-major, C [M, N] FP32
    (tcgen05 kernel).  acc: C += A @ B^T instead, K split over the SMs (no bias)."""
    M_, K = A.shape
    N = B.shape[0]
    assert B.shape[1] == K and C_.shape == (M_, N) and A.dtype == B.dtype == torch.bfloat16
    if acc:
        assert bias is None
        _lib.check(_lib.lib().g1b_gemm_bf16_acc(M_, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(C_),
                                                C_.stride(0), _st(A.device)), "g1b_gemm_bf16_acc")
        return
    _lib.check(_lib.lib().g1b_gemm_bf16(M_, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(C_), C_.stride(0),
                                        _p(bias), splits, _st(A.device)), "g1b_gemm_bf16")


def gemm_atb(A, B, C_):
    """C += A^T @ B: A [K, M], B [K, N] BF16 row-major, C [M, N] FP32, K split
    over the SMs (tcgen05 kernel reading MN-major tiles): the weight gradient
    dW += dZ^T H from the activations as the layers store them."""
    K, M_ = A.shape
    N = B.shape[1]
    assert B.shape[0] == K and C_.shape == (M_, N) and A.dtype == B.dtype == torch.bfloat16
    _lib.check(_lib.lib().g1b_gemm_bf16_atb_acc(M_, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(C_),
                                                C_.stride(0), _st(A.device)), "g1b_gemm_bf16_atb_acc")


def linear_silu(A, W, bias, H, Z=None, Ht=None):
    """One hidden layer, fused: z = A @ W^T + bias; H = bf16(silu(z)) [M, N];
    Z = z (FP16 [M, N], optional: the backward pass's SiLU derivative);
    Ht = H^T ([N, M] BF16, optional)."""
    M_, K = A.shape
    N = W.shape[0]
    assert W.shape[1] == K and H.shape == (M_, N) and A.dtype == W.dtype == torch.bfloat16
    assert Z is None or (Z.shape == (M_, N) and Z.dtype == torch.float16)
    assert Ht is None or (Ht.shape[0] == N and Ht.shape[1] >= M_)
    _lib.check(_lib.lib().g1b_sur_linear_silu(M_, N, K, _p(A), A.stride(0), _p(W), W.stride(0), _p(bias), _p(Z),
                                              Z.stride(0) if Z is not None else 0, _p(H), H.stride(0), _p(Ht),
                                              Ht.stride(0) if Ht is not None else 0, _st(A.device)),
               "g1b_sur_linear_silu")


def linear_silu_bwd(dZ, Wt, Z, dH, dHt=None, db=None):
    """Backward through a layer and the previous activation, fused:
    g = (dZ @ Wt^T) * silu'(Z) (Z FP16); dH = bf16(g) [M, N]; dHt = dH^T (optional);
    db += column sums of g (optional).  dH must not share memory with dZ."""
    M_, K = dZ.shape
    N = Wt.shape[0]
    assert Wt.shape[1] == K and dH.shape == (M_, N) and Z.shape[0] == M_ and Z.shape[1] >= N
    assert Z.dtype == torch.float16
    assert dHt is None or (dHt.shape[0] == N and dHt.shape[1] >= M_)
    _lib.check(_lib.lib().g1b_sur_linear_silu_bwd(M_, N, K, _p(dZ), dZ.stride(0), _p(Wt), Wt.stride(0), _p(Z),
                                                  Z.stride(0), _p(dH), dH.stride(0), _p(dHt),
                                                  dHt.stride(0) if dHt is not None else 0, _p(db), _st(dZ.device)),
               "g1b_sur_linear_silu_bwd")


def gemm_status():
    c = C.c_int()
    _lib.check(_lib.lib().g1b_gemm_status(C.byref(c)), "g1b_gemm_status")
    return c.value


class Surrogate:
    """Parameters (FP32 masters, Adam moments, BF16 copies) and training."""

    def __init__(self, device, seed=0):
        self.device = device
        g = torch.Generator().manual_seed(seed)
        self.W, self.b = [], []
        for i in range(5):
            fan_in, fan_out = DIMS[i], DIMS[i + 1]
            w = torch.zeros(fan_out, fan_in)
            used_in = NFEAT if i == 0 else fan_in
            used_out = NOUT if i == 4 else fan_out
            bound = (6.0 / (used_in + used_out)) ** 0.5
            w[:used_out, :used_in] = (torch.rand(used_out, used_in, generator=g) * 2 - 1) * bound
            self.W.append(w.to(device))
            self.b.append(torch.zeros(fan_out, device=device))
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.Wb = [torch.empty(w.shape, dtype=torch.bfloat16, device=device) for w in self.W]
        self.Wt = [torch.empty(w.shape[1], w.shape[0], dtype=torch.bfloat16, device=device) for w in self.W]
        # every gradient and the loss in one buffer, zeroed by one launch per backward pass
        # (the weight gradients are summed into it by split-K GEMMs)
        shapes = [tuple(w.shape) for w in self.W] + [tuple(b.shape) for b in self.b] + [(1,)]
        sizes = [int(np.prod(sh)) for sh in shapes]
        self._grad = torch.zeros(sum(sizes), device=device)
        views, off = [], 0
        for sh, n in zip(shapes, sizes):
            views.append(self._grad[off:off + n].view(sh))
            off += n
        self.gW, self.gb, self.loss_buf = views[:5], views[5:10], views[10]
        self.step_n = 0
        # Adam's step count and learning rate live on the device, so that a
        # CUDA graph of the training step replays with the current ones
        self.opt_step = torch.zeros(1, dtype=torch.int32, device=device)
        self.lr_dev = torch.full((1,), 1e-3, device=device)
        self._layers = (_lib.SurLayer * 5)(*[
            _lib.SurLayer(*[t.data_ptr() for t in (self.W[i], self.b[i], self.mW[i], self.vW[i], self.mb[i],
                                                    self.vb[i], self.gW[i], self.gb[i], self.Wb[i], self.Wt[i])],
                          self.W[i].shape[0], self.W[i].shape[1]) for i in range(5)])
        self.in_mean = torch.zeros(NIN, device=device)
        self.in_istd = torch.ones(NIN, device=device)
        self.out_mean = torch.zeros(64, device=device)
        self.out_std = torch.ones(64, device=device)
        self.out_w = torch.zeros(64, device=device)
        self.out_w[:NOUT] = 1.0 / NOUT
        self._ws = {}
        self.cast()

    def cast(self):
        L = _lib.lib()
        for w, wb, wt in zip(self.W, self.Wb, self.Wt):
            _lib.check(L.g1b_sur_cast(w.shape[0], w.shape[1], _p(w), _p(wb), _p(wt), _st(self.device)), "sur_cast")

    def _work(self, B):
        if B not in self._ws:
            d, bf = self.device, torch.bfloat16
            self._ws[B] = dict(
                # pre-activations: FP16 for the hidden layers (their SiLU derivative), FP32 output
                Z=[None] + [torch.empty(B, DIMS[i], dtype=torch.float16, device=d) for i in range(1, 5)] +
                  [torch.empty(B, DIMS[5], device=d)],
                H=[None] + [torch.empty(B, DIMS[i], dtype=bf, device=d) for i in range(1, 5)],
                dX=torch.empty(B, NIN, device=d),
                dY=torch.zeros(B, 64, device=d),
                dZ=torch.empty(B, 512, dtype=bf, device=d),
                dZ2=torch.empty(B, 512, dtype=bf, device=d))
        return self._ws[B]

    def features(self, qpos, qvel, anchor, ctrl, X, Xt=None, raw=None, mu=None, dmass=None):
        """Normalised BF16 features X [n, 192] of the SoA state (Xt [192, n]
        and the raw FP32 features raw [n, 192] optional)."""
        n = qpos.shape[1]
        _lib.check(_lib.lib().g1b_sur_features(n, _p(qpos), _p(qvel), _p(anchor), _p(ctrl), _p(mu), _p(dmass),
                                                _p(self.in_mean), _p(self.in_istd), _p(X), _p(Xt), _p(raw),
                                                _st(self.device)), "sur_features")

    def forward(self, X, keep=False):
        """Normalised prediction Y [B, 64] (FP32) for BF16 inputs X [B, 128]."""
        B = X.shape[0]
        w = self._work(B)
        L = _lib.lib()
        h = X
        for i in range(4):  # hidden layers: GEMM, bias and SiLU in one kernel
            linear_silu(h, self.Wb[i], self.b[i], w["H"][i + 1], Z=w["Z"][i + 1] if keep else None)
            h = w["H"][i + 1]
        gemm(h, self.Wb[4], w["Z"][5], bias=self.b[4])
        return w["Z"][5]

    def backward(self, X, T, want_dx=False, weights=None):
        """Loss of the last forward(X, keep=True) against normalised targets T
        [B, 64] (weighted MSE, per-output weights), and the gradients of every
        parameter (self.gW, self.gb); with want_dx also d loss / d X (FP32
        [B, 192], in self.dX(B))."""
        B = X.shape[0]
        w = self._work(B)
        L = _lib.lib()
        st = _st(self.device)
        self._grad.zero_()  # every parameter gradient and the loss
        dZ = w["dZ"]
        wv = self.out_w if weights is None else weights
        # dY = d loss / d Y as BF16 [B][64] (the start of dZ)
        _lib.check(L.g1b_sur_loss(B, 64, _p(w["Z"][5]), _p(T), _p(wv), _p(dZ), None, _p(self.gb[4]),
                                  _p(self.loss_buf), st), "sur_loss")
        bufs = [w["dZ"], w["dZ2"]]  # the layer's dZ and the previous layer's, alternating
        for i in range(4, -1, -1):
            Din, Dout = DIMS[i], DIMS[i + 1]
            dz = bufs[i & 1].view(-1)[:B * Dout].view(B, Dout)
            # dW_i = dZ_i^T . H_{i-1} (the batch split over the SMs, summed into the zeroed gradient)
            gemm_atb(dz, w["H"][i] if i > 0 else X, self.gW[i])
            if i > 0:
                # dZ_{i-1} = (dZ_i . W_i) * SiLU'(Z_{i-1}), its transpose and bias gradient, one kernel
                nxt = bufs[(i - 1) & 1].view(-1)[:B * Din].view(B, Din)
                linear_silu_bwd(dz, self.Wt[i], w["Z"][i], nxt, db=self.gb[i - 1])
            elif want_dx:
                gemm(dz, self.Wt[0], w["dX"])
        return self.loss_buf

    def dX(self, B):
        return self._work(B)["dX"]

    def input_grad(self, X, dY):
        """d / d X of <dY, Y> for the last forward(X, keep=True): dY [B, 64]
        FP32 adjoint of the normalised output; returns dX [B, 192] (FP32).
        The network's backward products without the weight gradients."""
        B = X.shape[0]
        w = self._work(B)
        _lib.check(_lib.lib().g1b_sur_seed(B * 64, _p(dY), _p(w["dZ"]), _st(self.device)), "sur_seed")
        bufs = [w["dZ"], w["dZ2"]]
        for i in range(4, -1, -1):
            Din, Dout = DIMS[i], DIMS[i + 1]
            dz = bufs[i & 1].view(-1)[:B * Dout].view(B, Dout)
            if i > 0:
                linear_silu_bwd(dz, self.Wt[i], w["Z"][i], bufs[(i - 1) & 1].view(-1)[:B * Din].view(B, Din))
            else:
                gemm(dz, self.Wt[0], w["dX"])
        return w["dX"]

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        """One Adam step of every layer and the BF16 weight copies, one launch.
        lr: the learning rate, written to the device first (None: keep the
        device's; the form a captured graph uses)."""
        if lr is not None:
            self.lr_dev.fill_(lr)
        self.opt_step.add_(1)
        self.step_n += 1
        _lib.check(_lib.lib().g1b_sur_adam_cast(5, self._layers, _p(self.opt_step), _p(self.lr_dev), b1, b2, eps,
                                                _st(self.device)), "sur_adam_cast")

    def train_step(self, X, T, lr=1e-3):
        self.forward(X, keep=True)
        loss = self.backward(X, T)
        self.adam(lr)
        return loss

    def capture_train_step(self, X, T, lr):
        """A CUDA graph of train_step on the fixed buffers X, T (write the
        next minibatch into them, then call the returned step(lr)).  Runs one
        eager training step first (with `lr`), which prepares every kernel."""
        return TrainGraph(self, X, T, lr)

    def integrate(self, Y, qpos, qvel, dt):
        n = qpos.shape[1]
        _lib.check(_lib.lib().g1b_sur_integrate(n, _p(Y), Y.stride(0), _p(self.out_mean), _p(self.out_std), dt,
                                                 _p(qpos), _p(qvel), _st(self.device)), "sur_integrate")


class TrainGraph:
    """One surrogate training step (forward, loss, backward, Adam) captured as
    a CUDA graph on fixed input buffers: the ~25 launches of a step replay
    without the host in between.  The learning rate and Adam's step count are
    read from device memory, so each replay uses the current ones."""

    def __init__(self, sur, X, T, lr):
        self.sur = sur
        dev = sur.device
        s = torch.cuda.Stream(dev)
        s.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(s):
            sur.train_step(X, T, lr=lr)  # a real step, which also prepares the kernels
        torch.cuda.current_stream(dev).wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=s):
            self.loss = sur.train_step(X, T, lr=None)
        sur.step_n -= 1  # the capture ran no step

    def step(self, lr=None):
        """One training step; returns the (device) loss buffer."""
        if lr is not None:
            self.sur.lr_dev.fill_(lr)
        self.graph.replay()
        self.sur.step_n += 1
        return self.loss


# ------------------------------------------------------------- data
def generate_transitions(sur, n_envs, n_steps, device, dt=2e-3, decim=10, seed=0):
    """Transitions of the randomised workload's simulator (targets stand +
    U(-0.3, 0.3) x range redrawn every `decim` steps, friction / base mass
    randomised, reset below 0.3 m): raw features F [N, 192] and qacc
    targets [N, 35] for N = n_envs * n_steps."""
    from . import workloads
    w = workloads.randomized(nenv=n_envs, seed=seed)
    f32 = dict(dtype=torch.float32, device=device)
    s = {k: torch.tensor(w[k], **f32) for k in ("qpos", "qvel", "anchor", "ctrl")}
    mu, dm = torch.tensor(w["mu"], **f32), torch.tensor(w["dmass"], **f32)
    fp, fv, cf = (torch.zeros(d, n_envs, **f32) for d in (6, 6, 8))
    rng = torch.Generator(device=device).manual_seed(seed)
    stand = torch.tensor(np.asarray(M.qpos_stand)[7:], **f32)[:, None]
    rg = torch.tensor(np.asarray(M.jnt_range), **f32)
    span = (rg[:, 1] - rg[:, 0])[:, None]
    cfg = _lib.default_config(dt=dt)
    N = n_envs * n_steps
    F = torch.empty(N, NIN, **f32)
    A = torch.empty(N, 35, **f32)
    Xtmp = torch.empty(n_envs, NIN, dtype=torch.bfloat16, device=device)
    done = torch.zeros(n_envs, dtype=torch.uint8, device=device)
    for t in range(n_steps):
        if t % decim == 0:
            u = torch.rand(29, n_envs, generator=rng, device=device)
            s["ctrl"].copy_(stand + (2 * u - 1) * 0.3 * span)
        rows = slice(t * n_envs, (t + 1) * n_envs)
        sur.features(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], Xtmp, None, F[rows], mu=mu, dmass=dm)
        v0 = s["qvel"].clone()
        G.step(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], 1, config=cfg, mu=mu, dmass=dm, foot_pos=fp,
               foot_vel=fv, contact_forces=cf)
        A[rows] = ((s["qvel"] - v0) / dt).T
        if t % decim == decim - 1:
            done.copy_((s["qpos"][2] < 0.3).to(torch.uint8))
            if bool(done.any()):
                G.reset_done(s["qpos"], s["qvel"], s["anchor"], done, seed=seed + t)
    return F, A


def fit_normalisation(sur, F, A):
    m = F.mean(0)
    sd = F.std(0)
    sd = torch.where(sd > 1e-6, sd, torch.ones_like(sd))
    m[NFEAT:] = 0
    sd[NFEAT:] = 1
    m[NFEAT - 1] = 0  # the constant feature stays 1
    sd[NFEAT - 1] = 1
    sur.in_mean.copy_(m)
    sur.in_istd.copy_(1.0 / sd)
    am, asd = A.mean(0), A.std(0).clamp_min(1e-6)
    sur.out_mean.zero_()
    sur.out_std.fill_(1.0)
    sur.out_mean[:NOUT] = am
    sur.out_std[:NOUT] = asd


def normalise(sur, F, A=None):
    """BF16 inputs X [N, 192] (and FP32 targets T [N, 64]) from raw features."""
    X = ((F - sur.in_mean) * sur.in_istd).to(torch.bfloat16)
    if A is None:
        return X
    T = torch.zeros(A.shape[0], 64, device=A.device)
    T[:, :NOUT] = (A - sur.out_mean[:NOUT]) / sur.out_std[:NOUT]
    return X, T


def train(sur, F, A, steps, batch=65536, lr=1e-3, seed=0, log_every=0):
    """Minibatch training on the library's kernels; returns the loss history.
    Each minibatch is gathered into fixed buffers and the step replayed as a
    CUDA graph (the first step runs eagerly and captures it)."""
    X, T = normalise(sur, F, A)
    N = X.shape[0]
    dev = X.device
    g = torch.Generator(device=dev).manual_seed(seed)
    xb = torch.empty(batch, NIN, dtype=torch.bfloat16, device=dev)
    tb = torch.empty(batch, T.shape[1], device=dev)
    hist, tg = [], None
    for k in range(steps):
        idx = torch.randint(0, N, (batch,), generator=g, device=dev)
        torch.index_select(X, 0, idx, out=xb)
        torch.index_select(T, 0, idx, out=tb)
        cur_lr = lr * (0.1 ** (k / max(steps, 1)))
        if tg is None:
            tg = sur.capture_train_step(xb, tb, cur_lr)
            loss = tg.loss
        else:
            loss = tg.step(cur_lr)
        if log_every and k % log_every == 0:
            hist.append((k, float(loss.item())))
    return hist


def _pad_rows(n):
    return n + (-n) % 128


def predict_next(sur, s, dt, mu=None, dmass=None):
    """Surrogate one-step prediction from the state dict s (copies)."""
    n = s["qpos"].shape[1]
    X = torch.zeros(_pad_rows(n), NIN, dtype=torch.bfloat16, device=sur.device)
    sur.features(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], X, mu=mu, dmass=dmass)
    Y = sur.forward(X)[:n]
    q, v = s["qpos"].clone(), s["qvel"].clone()
    sur.integrate(Y.contiguous(), q, v, dt)
    return q, v


def one_step_error(sur, s, dt=2e-3, mu=None, dmass=None):
    """Per-env one-step error of the surrogate against the exact step from
    state s: max over qpos and qvel components of |x_sur - x| / max(|x|, 1)."""
    qs, vs = predict_next(sur, s, dt, mu, dmass)
    ex = {k: s[k].clone() for k in ("qpos", "qvel", "anchor")}
    G.step(ex["qpos"], ex["qvel"], ex["anchor"], s["ctrl"], 1, config=_lib.default_config(dt=dt), mu=mu, dmass=dmass)
    eq = ((qs - ex["qpos"]).abs() / ex["qpos"].abs().clamp_min(1.0)).amax(0)
    ev = ((vs - ex["qvel"]).abs() / ex["qvel"].abs().clamp_min(1.0)).amax(0)
    return torch.maximum(eq, ev), qs, vs, ex


def rollout_with_fallback(sur, s, steps, dt=2e-3, bound=1e-3, mu=None, dmass=None):
    """Advance every env `steps` steps: with the surrogate where its one-step
    error against the exact step is <= bound (relative per component of
    qpos and qvel), else with the exact step.  Returns (fraction of env-steps
    taken by the surrogate, statistics of the one-step error: median, 90th
    percentile and the fractions of env-steps within 1e-3, 1e-2 and 1e-1)."""
    used, errs = 0, []
    n = s["qpos"].shape[1]
    for _ in range(steps):
        err, qs, vs, ex = one_step_error(sur, s, dt, mu, dmass)
        ok = err <= bound
        used += int(ok.sum().item())
        errs.append(err)
        s["qpos"].copy_(torch.where(ok[None], qs, ex["qpos"]))
        s["qvel"].copy_(torch.where(ok[None], vs, ex["qvel"]))
        s["anchor"].copy_(ex["anchor"])
    e = torch.cat(errs)
    stats = {"median": float(e.median().item()), "p90": float(torch.quantile(e[:1 << 24].float(), 0.9).item()),
             "within_1e-3": float((e <= 1e-3).float().mean().item()),
             "within_1e-2": float((e <= 1e-2).float().mean().item()),
             "within_1e-1": float((e <= 1e-1).float().mean().item())}
    return used / float(n * steps), stats


# ---------------------------------------------- gradients and refinement
# Short-horizon objective of a target vector u held for H substeps from the
# state s (the adjoint workload's height term plus a proximity term to the
# policy's targets u0):  J(u) = sum_{t=1..H} (z_t - z_ref)^2 + reg |u - u0|^2.

def exact_objective(s, u, H, z_ref=0.78, dt=2e-3, mu=None, dmass=None, u0=None, reg=0.0):
    """J per env with the exact step (the judge).  s is not modified."""
    x = {k: s[k].clone() for k in ("qpos", "qvel", "anchor")}
    cfg = _lib.default_config(dt=dt)
    J = torch.zeros(u.shape[1], device=u.device)
    for _ in range(H):
        G.step(x["qpos"], x["qvel"], x["anchor"], u, 1, config=cfg, mu=mu, dmass=dmass)
        J += (x["qpos"][2] - z_ref) ** 2
    if u0 is not None and reg > 0:
        J += reg * ((u - u0) ** 2).sum(0)
    return J


def exact_grad(s, u, H, z_ref=0.78, dt=2e-3, u0=None, reg=0.0):
    """dJ/du by the exact step's adjoint (g1b_adjoint, targets held: the
    per-step target gradients summed); friction 1, no mass offset."""
    from . import adjoint as A
    n = u.shape[1]
    tg = u[None].expand(H, 29, n).contiguous()
    r = A.horizon_adjoint(tg, None, None, s["qpos"].contiguous(), s["qvel"].contiguous(), s["anchor"].contiguous(),
                          checkpoint=min(8, H), z_ref=z_ref, w_track=0.0, config=_lib.default_config(dt=dt))
    g = r["grad_targets"].sum(0)
    if u0 is not None and reg > 0:
        g = g + 2 * reg * (u - u0)
    return g


def rollout_grad(sur, s, u, H, z_ref=0.78, dt=2e-3, mu=None, dmass=None, u0=None, reg=0.0):
    """(J_sur, dJ_sur/du) per env through an H-step surrogate rollout from
    the exact state s (anchors held at their values in s), by
    backpropagation through the feature, network and update kernels."""
    L = _lib.lib()
    st = _st(sur.device)
    n = u.shape[1]
    B = _pad_rows(n)
    X = torch.zeros(B, NIN, dtype=torch.bfloat16, device=sur.device)
    qs, vs, Ys = [s["qpos"].clone()], [s["qvel"].clone()], []
    an = s["anchor"]
    J = torch.zeros(n, device=u.device)
    for _ in range(H):  # forward: keep the states and the network outputs
        q, v = qs[-1].clone(), vs[-1].clone()
        sur.features(q, v, an, u, X, mu=mu, dmass=dmass)
        Y = sur.forward(X)[:n].clone()
        sur.integrate(Y, q, v, dt)
        Ys.append(Y)
        qs.append(q)
        vs.append(v)
        J += (q[2] - z_ref) ** 2
    lq = torch.zeros_like(qs[0])
    lv = torch.zeros_like(vs[0])
    lq[2] = 2 * (qs[H][2] - z_ref)
    ub = torch.zeros_like(u)
    dY = torch.zeros(B, 64, device=sur.device)
    for t in range(H - 1, -1, -1):
        _lib.check(L.g1b_sur_integrate_vjp(n, _p(qs[t]), _p(vs[t]), _p(Ys[t]), Ys[t].stride(0), _p(sur.out_mean),
                                           _p(sur.out_std), dt, _p(lq), _p(lv), _p(dY), 64, st), "sur_integrate_vjp")
        sur.features(qs[t], vs[t], an, u, X, mu=mu, dmass=dmass)
        sur.forward(X, keep=True)
        dX = sur.input_grad(X, dY)
        _lib.check(L.g1b_sur_features_vjp(n, _p(qs[t]), _p(vs[t]), _p(an), _p(sur.in_istd), _p(dX), NIN, _p(lq),
                                          _p(lv), None, _p(ub), st), "sur_features_vjp")
        if t >= 1:
            lq[2] += 2 * (qs[t][2] - z_ref)
    if u0 is not None and reg > 0:
        J = J + reg * ((u - u0) ** 2).sum(0)
        ub = ub + 2 * reg * (u - u0)
    return J, ub


def refine_targets(sur, s, u0, H=10, iters=10, step=0.05, mode="surrogate", bound=None, z_ref=0.78, dt=2e-3,
                   mu=None, dmass=None, reg=0.1):
    """Short-horizon refinement of the targets u0 [29, n] a policy chose at
    state s: `iters` normalised gradient steps on J (of `step` rad in the
    29-dim target space, per env), each judged by the exact step: an update
    that does not lower the exact J is rejected and that env's step halved.
    mode "surrogate": gradients through the surrogate rollout; with `bound`,
    envs whose surrogate one-step error at s exceeds it fall back to the
    exact adjoint's gradient.  mode "exact": the exact adjoint only.
    Returns (u, J_exact per env, fraction of envs on the surrogate's
    gradient)."""
    u = u0.clone()
    n = u.shape[1]
    J = exact_objective(s, u, H, z_ref, dt, mu, dmass, u0, reg)
    alpha = torch.full((n,), step, device=u.device)
    use_sur = torch.ones(n, dtype=torch.bool, device=u.device) if mode == "surrogate" else \
        torch.zeros(n, dtype=torch.bool, device=u.device)
    if mode == "surrogate" and bound is not None:
        err, _, _, _ = one_step_error(sur, {**s, "ctrl": u}, dt, mu, dmass)
        use_sur &= err <= bound
    for _ in range(iters):
        g = torch.zeros_like(u)
        if bool(use_sur.any()):
            g = rollout_grad(sur, s, u, H, z_ref, dt, mu, dmass, u0, reg)[1]
        if not bool(use_sur.all()):
            g = torch.where(use_sur[None], g, exact_grad(s, u, H, z_ref, dt, u0, reg))
        d = g / g.norm(dim=0).clamp_min(1e-12)
        cand = u - alpha[None] * d
        Jc = exact_objective(s, cand, H, z_ref, dt, mu, dmass, u0, reg)
        ok = Jc < J
        u = torch.where(ok[None], cand, u)
        J = torch.where(ok, Jc, J)
        alpha = torch.where(ok, alpha, 0.5 * alpha)
    return u, J, float(use_sur.float().mean().item())
