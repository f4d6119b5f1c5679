"""Learned one-step dynamics surrogate of the G1 step.

An MLP 128 -> 4 x 512 (SiLU) -> 64 over a normalised feature vector of the
state and the PD targets (joint angles and rates, base height, the first two
columns of the base rotation, body-frame base velocities, foot-sphere
contact flags, targets; 109 used, padded to 128) predicting the normalised
generalised acceleration of the step (35 used, padded to 64).  The state
delta is dt * qacc for qvel; qpos follows by the step's semi-implicit Euler
(sur_integrate_kernel).

Training runs on the library's own kernels: BF16 tcgen05 GEMMs with FP32
accumulation (g1b_gemm_bf16) for the forward pass, the input-gradient and
the weight-gradient products; element-wise SiLU, SiLU', the loss and its
gradient, Adam and the BF16 weight copies in g1_surrogate.cuh.  Torch only
allocates the buffers and zeroes the gradient accumulators.

The exact step stays the judge: `rollout_with_fallback` advances each env
with the surrogate only where its one-step error against the exact step is
within a bound (1e-3, relative per state component) and with the exact step
elsewhere.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from . import g1sim as G
from .model import g1_model_data as M

DIMS = [128, 512, 512, 512, 512, 64]
NFEAT, NOUT = 109, 35


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _st(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def gemm(A, B, C_, bias=None, splits=1):
    """C = A @ B^T (+ bias): A [M, K], B [N, K] BF16 row-major, C [M, N] FP32 (tcgen05 kernel)."""
    M_, K = A.shape
    N = B.shape[0]
    assert B.shape[1] == K and C_.shape == (M_, N) and A.dtype == B.dtype == torch.bfloat16
    _lib.check(_lib.lib().g1b_gemm_bf16(M_, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(C_), C_.stride(0),
                                        _p(bias), splits, _st(A.device)), "g1b_gemm_bf16")


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
        self.gW = [torch.zeros(max(w.shape[0], 128), w.shape[1], device=device) for w in self.W]
        self.gb = [torch.zeros_like(b) for b in self.b]
        self.step_n = 0
        self.in_mean = torch.zeros(128, device=device)
        self.in_istd = torch.ones(128, device=device)
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
                Z=[None] + [torch.empty(B, DIMS[i], device=d) for i in range(1, 6)],
                H=[None] + [torch.empty(B, DIMS[i], dtype=bf, device=d) for i in range(1, 5)],
                Ht=[None] + [torch.empty(DIMS[i], B, dtype=bf, device=d) for i in range(1, 5)],
                dH=torch.empty(B, 512, device=d),
                dX=torch.empty(B, 128, device=d),
                dZ=torch.empty(B, 512, dtype=bf, device=d),
                dZt=torch.zeros(512, B, dtype=bf, device=d),
                loss=torch.zeros(1, device=d))
        return self._ws[B]

    def features(self, qpos, qvel, ctrl, cf, X, Xt=None, raw=None):
        n = qpos.shape[1]
        _lib.check(_lib.lib().g1b_sur_features(n, _p(qpos), _p(qvel), _p(ctrl), _p(cf), _p(self.in_mean),
                                                _p(self.in_istd), _p(X), _p(Xt), _p(raw), _st(self.device)),
                   "sur_features")

    def forward(self, X, keep=False):
        """Normalised prediction Y [B, 64] (FP32) for BF16 inputs X [B, 128]."""
        B = X.shape[0]
        w = self._work(B)
        L = _lib.lib()
        h = X
        for i in range(5):
            gemm(h, self.Wb[i], w["Z"][i + 1], bias=self.b[i])
            if i < 4:
                _lib.check(L.g1b_sur_act(B, DIMS[i + 1], _p(w["Z"][i + 1]), _p(w["H"][i + 1]),
                                         _p(w["Ht"][i + 1]) if keep else None, _st(self.device)), "sur_act")
                h = w["H"][i + 1]
        return w["Z"][5]

    def backward(self, X, Xt, T, want_dx=False, weights=None):
        """Loss of the last forward(X, keep=True) against normalised targets T
        [B, 64] (weighted MSE, per-output weights), and the gradients of every
        parameter (self.gW, self.gb); with want_dx also d loss / d X (FP32
        [B, 128], in self.dX(B)).  Xt: X transposed [128, B]."""
        B = X.shape[0]
        w = self._work(B)
        L = _lib.lib()
        st = _st(self.device)
        for g_ in self.gb:
            g_.zero_()
        w["loss"].zero_()
        dZ, dZt = w["dZ"], w["dZt"]
        dZt[64:128].zero_()
        wv = self.out_w if weights is None else weights
        # dY = d loss / d Y as BF16 [B][64] (start of dZ) and [64][B] (rows of dZt)
        _lib.check(L.g1b_sur_loss(B, 64, _p(w["Z"][5]), _p(T), _p(wv), _p(dZ), _p(dZt), _p(self.gb[4]),
                                  _p(w["loss"]), st), "sur_loss")
        for i in range(4, -1, -1):
            Din, Dout = DIMS[i], DIMS[i + 1]
            dz = dZ.view(-1)[:B * Dout].view(B, Dout)
            rows = max(Dout, 128)
            hin_t = w["Ht"][i] if i > 0 else Xt
            # dW_i = dZ_i^T . H_{i-1} (split over the batch, atomically summed)
            gemm(dZt[:rows], hin_t, self.gW[i][:rows], splits=max(1, min(64, B // 2048)))
            if i > 0:
                dh = w["dH"].view(-1)[:B * Din].view(B, Din)
                gemm(dz, self.Wt[i], dh)  # dH_{i-1} = dZ_i . W_i
                _lib.check(L.g1b_sur_act_bwd(B, Din, _p(dh), _p(w["Z"][i]), _p(dZ), _p(dZt), _p(self.gb[i - 1]),
                                             st), "sur_act_bwd")
            elif want_dx:
                gemm(dz, self.Wt[0], w["dX"])
        return w["loss"]

    def dX(self, B):
        return self._work(B)["dX"]

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_n += 1
        L = _lib.lib()
        st = _st(self.device)
        for i in range(5):
            gw = self.gW[i][:self.W[i].shape[0]]  # leading rows: contiguous
            _lib.check(L.g1b_sur_adam(self.W[i].numel(), _p(self.W[i]), _p(gw),
                                      _p(self.mW[i]), _p(self.vW[i]), lr, b1, b2, eps, self.step_n, st), "sur_adam")
            _lib.check(L.g1b_sur_adam(self.b[i].numel(), _p(self.b[i]), _p(self.gb[i]), _p(self.mb[i]),
                                      _p(self.vb[i]), lr, b1, b2, eps, self.step_n, st), "sur_adam")
        self.cast()

    def train_step(self, X, Xt, T, lr=1e-3):
        self.forward(X, keep=True)
        loss = self.backward(X, Xt, T)
        self.adam(lr)
        return loss

    def integrate(self, Y, qpos, qvel, dt):
        n = qpos.shape[1]
        _lib.check(_lib.lib().g1b_sur_integrate(n, _p(Y), Y.stride(0), _p(self.out_mean), _p(self.out_std), dt,
                                                 _p(qpos), _p(qvel), _st(self.device)), "sur_integrate")


# ------------------------------------------------------------- data
def generate_transitions(sur, n_envs, n_steps, device, dt=2e-3, decim=10, seed=0):
    """Transitions of the randomised workload's simulator (targets stand +
    U(-0.3, 0.3) x range redrawn every `decim` steps, friction / base mass
    randomised, reset below 0.3 m): raw features F [N, 128] and qacc
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
    F = torch.empty(N, 128, **f32)
    A = torch.empty(N, 35, **f32)
    Xtmp = torch.empty(n_envs, 128, dtype=torch.bfloat16, device=device)
    done = torch.zeros(n_envs, dtype=torch.uint8, device=device)
    for t in range(n_steps):
        if t % decim == 0:
            u = torch.rand(29, n_envs, generator=rng, device=device)
            s["ctrl"].copy_(stand + (2 * u - 1) * 0.3 * span)
        rows = slice(t * n_envs, (t + 1) * n_envs)
        sur.features(s["qpos"], s["qvel"], s["ctrl"], cf, Xtmp, None, F[rows])
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
    """BF16 inputs X [N, 128] (and FP32 targets T [N, 64]) from raw features."""
    X = ((F - sur.in_mean) * sur.in_istd).to(torch.bfloat16)
    if A is None:
        return X
    T = torch.zeros(A.shape[0], 64, device=A.device)
    T[:, :NOUT] = (A - sur.out_mean[:NOUT]) / sur.out_std[:NOUT]
    return X, T


def train(sur, F, A, steps, batch=65536, lr=1e-3, seed=0, log_every=0):
    """Minibatch training on the library's kernels; returns the loss history."""
    X, T = normalise(sur, F, A)
    N = X.shape[0]
    g = torch.Generator(device=X.device).manual_seed(seed)
    hist = []
    for k in range(steps):
        idx = torch.randint(0, N, (batch,), generator=g, device=X.device)
        xb = X[idx].contiguous()
        xt = xb.T.contiguous()
        tb = T[idx].contiguous()
        cur_lr = lr * (0.1 ** (k / max(steps, 1)))
        loss = sur.train_step(xb, xt, tb, lr=cur_lr)
        if log_every and k % log_every == 0:
            hist.append((k, float(loss.item())))
    return hist


def predict_next(sur, s, dt):
    """Surrogate one-step prediction from the state dict s (copies)."""
    n = s["qpos"].shape[1]
    X = torch.empty(n, 128, dtype=torch.bfloat16, device=sur.device)
    sur.features(s["qpos"], s["qvel"], s["ctrl"], s["contact_forces"], X)
    pad = (-n) % 128
    if pad:
        X = torch.cat([X, torch.zeros(pad, 128, dtype=torch.bfloat16, device=sur.device)])
    Y = sur.forward(X)[:n]
    q, v = s["qpos"].clone(), s["qvel"].clone()
    sur.integrate(Y.contiguous(), q, v, dt)
    return q, v


def rollout_with_fallback(sur, s, steps, dt=2e-3, bound=1e-3, mu=None, dmass=None):
    """Advance every env `steps` steps: with the surrogate where its one-step
    error against the exact step is <= bound (relative per component of
    qpos and qvel), else with the exact step.  Returns (fraction of env-steps
    taken by the surrogate, statistics of the one-step error: median, 90th
    percentile and the fractions of env-steps within 1e-2 and 1e-1)."""
    cfg = _lib.default_config(dt=dt)
    used, errs = 0, []
    n = s["qpos"].shape[1]
    for _ in range(steps):
        qs, vs = predict_next(sur, s, dt)
        ex = {k: s[k].clone() for k in ("qpos", "qvel", "anchor")}
        G.step(ex["qpos"], ex["qvel"], ex["anchor"], s["ctrl"], 1, config=cfg, mu=mu, dmass=dmass,
               contact_forces=s["contact_forces"])
        eq = ((qs - ex["qpos"]).abs() / ex["qpos"].abs().clamp_min(1.0)).amax(0)
        ev = ((vs - ex["qvel"]).abs() / ex["qvel"].abs().clamp_min(1.0)).amax(0)
        err = torch.maximum(eq, ev)
        ok = err <= bound
        used += int(ok.sum().item())
        errs.append(err)
        s["qpos"].copy_(torch.where(ok[None], qs, ex["qpos"]))
        s["qvel"].copy_(torch.where(ok[None], vs, ex["qvel"]))
        s["anchor"].copy_(ex["anchor"])
    e = torch.cat(errs)
    stats = {"median": float(e.median().item()), "p90": float(torch.quantile(e[:1 << 24].float(), 0.9).item()),
             "within_1e-2": float((e <= 1e-2).float().mean().item()),
             "within_1e-1": float((e <= 1e-1).float().mean().item())}
    return used / float(n * steps), stats
