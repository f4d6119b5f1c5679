"""Policy-fused rollout kernel on the GPU (needs a B200).

Checks, each against an independent restatement:
  * observation: numpy restatement of the reference G1Sim.get_obs
    (src/g1sim.py:132-170), FP32, to 1e-6;
  * critic value and actor mean: torch emulation of the kernel's numerics
    (BF16 operands and activations, FP32 accumulation; policy.
    kernel_mlp_reference) to 2e-3 absolute + relative -- the two sides may
    round a hidden activation to different BF16 neighbours when their FP32
    sums differ in the last bits;
  * PD targets: stand + action * scale in FP32, bit for bit;
  * physics of the policy step: the FP64 oracle from the same state with the
    kernel's targets (and pushes) over the 10 substeps, qpos within 1e-5;
  * action noise: Box-Muller on the oracle's counter-based uniforms (FP64),
    to 1e-5; log-probabilities from torch.distributions.Normal;
  * reward and termination: policy.reward_and_done, the torch restatement
    of the reference compute_reward_and_done (examples/train.py:143-218);
  * resets: the oracle's restatement of the reference reset kernel, bit for
    bit; timers and command redraws within their ranges;
  * one launch of 8 policy steps equals 8 launches of one, bit for bit.
"""
import numpy as np
import pytest
import torch

from g1sim_b200 import _lib, workloads
from g1sim_b200 import policy as P
from g1sim_b200.model import g1_model_data as M

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)
STAND = np.asarray(M.qpos_stand, dtype=np.float64)
SCALE = P.ACTION_SCALE.numpy()


def dev(a, dtype=torch.float32):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def host(t):
    return t.detach().cpu().numpy().astype(np.float64)


def relerr(x, ref):
    return np.abs(x - ref) / np.maximum(np.abs(ref), 1.0)


def make_sim(n, seed=0, z=0.80):
    w = workloads.drop_test(nenv=n, seed=seed, z=z)
    s = {k: dev(w[k]) for k in ("qpos", "qvel", "anchor", "ctrl")}
    for k, d in (("foot_pos", 6), ("foot_vel", 6), ("contact_forces", 8)):
        s[k] = torch.zeros(d, n, device=DEV)
    return s


def make_policy(seed=0):
    g = torch.Generator().manual_seed(seed)
    ac = P.ActorCritic().xavier_(g)
    with torch.no_grad():
        for m in ac.modules():
            if isinstance(m, torch.nn.Linear):
                m.bias.uniform_(-0.05, 0.05, generator=g)
        ac.std.uniform_(-1.5, -0.5, generator=g)
        ac.obs_mean.normal_(0.0, 0.1, generator=g)
        ac.obs_var.uniform_(0.3, 3.0, generator=g)
    return ac


def quat_rot_inv(q, v):
    """reference src/g1sim.py:146-154, float32."""
    qw = q[0]
    u = -q[1:4]
    uv = np.cross(u, v, axis=0)
    uuv = np.cross(u, uv, axis=0)
    return v + np.float32(2.0) * (qw * uv + uuv)


def obs_reference(qpos, qvel, cmd, last_ctrl):
    """Restatement of the reference G1Sim.get_obs in float32 -> (n, 99)."""
    qpos, qvel = qpos.astype(np.float32), qvel.astype(np.float32)
    n = qpos.shape[1]
    grav = np.zeros((3, n), np.float32)
    grav[2] = -1.0
    q = qpos[3:7]
    obs = np.concatenate([cmd.astype(np.float32), quat_rot_inv(q, grav), quat_rot_inv(q, qvel[0:3]), qvel[3:6],
                          qpos[7:36] - STAND[7:, None].astype(np.float32), qvel[6:35],
                          last_ctrl.astype(np.float32)], axis=0)
    return obs.T


def params(flags, **kw):
    p = _lib.policy_default_params()
    p.flags = flags
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def task_u(oracle, seed, purpose, e, stp, j):
    s = (seed + purpose * 0x9E3779B9) & 0xffffffff
    return oracle.uniform(s, e, stp * 64 + j)


def run(sim, packed, task, buf, npolicy, p, step0=0, seed=0, bootstrap=True, t0=0):
    P.policy_rollout(sim, packed, task, buf, npolicy, decim=10, params=p, step0=step0, seed=seed,
                     bootstrap=bootstrap, t0=t0)
    torch.cuda.synchronize()
    assert _lib.policy_status() == 0


@pytest.fixture(scope="module")
def net():
    ac = make_policy(0)
    return ac, P.pack_policy(ac, DEV)


@pytest.mark.parametrize("n", [1, 130, 300])
def test_observation_and_networks_match(net, n):
    ac, packed = net
    sim = make_sim(n, seed=4)
    task = P.TaskState(n, DEV, seed=5)
    buf = P.RolloutBuffers(1, n, DEV, mean=True)
    q0, v0, c0 = host(sim["qpos"]), host(sim["qvel"]), host(sim["ctrl"])
    cmd0 = host(task.commands)
    run(sim, packed, task, buf, 1, params(0))
    obs_ref = obs_reference(q0, v0, cmd0, c0)
    obs = buf.obs[0].cpu().numpy()
    assert np.abs(obs - obs_ref).max() < 1e-6
    mean_ref, val_ref = P.kernel_mlp_reference(ac.to(DEV), buf.obs[0])
    err_m = (buf.mean[0] - mean_ref).abs() / (1 + mean_ref.abs())
    err_v = (buf.values[0] - val_ref).abs() / (1 + val_ref.abs())
    print(f"n={n} mean err max {err_m.max().item():.2e} value err max {err_v.max().item():.2e}")
    assert err_m.max().item() < 2e-3 and err_v.max().item() < 2e-3
    # deterministic action = mean, targets stand + a * scale in FP32
    assert torch.equal(buf.actions[0], buf.mean[0])
    a = buf.actions[0].cpu().numpy().T.astype(np.float32)
    tgt = (STAND[7:, None].astype(np.float32) + a * SCALE[:, None]).astype(np.float32)
    assert np.array_equal(sim["ctrl"].cpu().numpy(), tgt)
    # bootstrap value of the final state
    obs1 = obs_reference(host(sim["qpos"]), host(sim["qvel"]), host(task.commands), host(sim["ctrl"]))
    assert np.abs(buf.last_obs.cpu().numpy() - obs1).max() < 1e-6
    _, v1 = P.kernel_mlp_reference(ac, buf.last_obs)
    assert ((buf.last_value - v1).abs() / (1 + v1.abs())).max().item() < 2e-3


def test_policy_step_physics_matches_oracle(net, oracle):
    ac, packed = net
    n = 256
    sim = make_sim(n, seed=6)
    task = P.TaskState(n, DEV, seed=7)
    task.push_timer.fill_(1)  # every env is pushed before the substeps
    q64, v64, a64 = host(sim["qpos"]), host(sim["qvel"]), host(sim["anchor"])
    seed, stp = 11, 3
    run(sim, packed, task, None, 1, params(_lib.PUSH), step0=stp, seed=seed, bootstrap=False)
    pv = [0.5, 0.5, 0.4, 0.52, 0.52, 0.78]
    for e in range(n):
        for i in range(6):
            u = np.float32(task_u(oracle, seed, 3, e, stp, i))
            dv = np.float32(np.float32(u * np.float32(2.0 * np.float32(pv[i]))) - np.float32(pv[i]))
            v64[i, e] = np.float32(np.float32(v64[i, e]) + dv)
    oracle.step_soa(10, oracle.config(dt=2e-3), q64, v64, a64, host(sim["ctrl"]), outputs=False)
    eq, ev = relerr(host(sim["qpos"]), q64), relerr(host(sim["qvel"]), v64)
    print(f"policy-step physics qpos max {eq.max():.2e} qvel max {ev.max():.2e}")
    assert eq.max() < 1e-6  # measured 1.7e-7
    assert ev.max() < 5e-5  # 10 compounded substeps after a push (measured 5.9e-6)
    t = task.push_timer.cpu().numpy()
    assert ((t >= 50) & (t < 150)).all()


def test_sampling_logprob_and_reward(net, oracle):
    ac, packed = net
    n = 200
    sim = make_sim(n, seed=8)
    task = P.TaskState(n, DEV, seed=9)
    task.prev_action.normal_(0.0, 0.3)
    prev = task.prev_action.clone()
    buf = P.RolloutBuffers(1, n, DEV, mean=True)
    seed, stp = 21, 5
    run(sim, packed, task, buf, 1, params(_lib.SAMPLE), step0=stp, seed=seed)
    mean, act = buf.mean[0].cpu().numpy().astype(np.float64), buf.actions[0].cpu().numpy().astype(np.float64)
    sig = np.exp(ac.std.detach().cpu().numpy().astype(np.float64))
    eps = np.zeros((n, 29))
    for e in range(n):
        for j in range(29):
            u1 = 1.0 - task_u(oracle, seed, 1, e, stp, j)
            u2 = task_u(oracle, seed, 2, e, stp, j)
            eps[e, j] = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    assert np.abs(act - (mean + sig * eps)).max() < 1e-5 * (1 + np.abs(act).max())
    dist = torch.distributions.Normal(buf.mean[0].cpu().double(), torch.tensor(sig))
    lp_ref = dist.log_prob(buf.actions[0].cpu().double()).sum(-1).numpy()
    assert np.abs(buf.log_probs[0].cpu().numpy() - lp_ref).max() < 1e-4
    assert torch.equal(task.prev_action, buf.actions[0].T.contiguous())
    # reward / termination from the post-step state (commands unchanged: no redraw flag)
    r_ref, d_ref = P.reward_and_done(buf.last_obs, buf.actions[0], prev.T, sim["qpos"], sim["foot_pos"],
                                     sim["foot_vel"], sim["contact_forces"])
    err = ((buf.rewards[0] - r_ref).abs() / (1 + r_ref.abs())).max().item()
    print(f"reward err max {err:.2e}, reward mean {buf.rewards[0].mean().item():.3f}")
    assert err < 1e-4
    assert torch.equal(buf.dones[0], d_ref)


def test_termination_reset_and_command_timers(net, oracle):
    ac, packed = net
    n = 160
    sim = make_sim(n, seed=10)
    # envs 0..39 start lying on their side (tilt 90 deg > 70 deg): terminated after the step
    q = sim["qpos"]
    q[3, :40] = np.cos(np.pi / 4)
    q[4, :40] = np.sin(np.pi / 4)
    q[5, :40] = 0.0
    q[6, :40] = 0.0
    q[2, :40] = 0.3
    task = P.TaskState(n, DEV, seed=11)
    task.cmd_timer[:] = 5
    task.cmd_timer[80:120] = 1       # redraw after this step
    task.ep_len[:] = 0
    task.ep_len[120:140] = 999       # timeout after this step
    task.push_timer.fill_(100)
    task.prev_action.fill_(0.7)
    cmd0 = task.commands.clone()
    buf = P.RolloutBuffers(1, n, DEV)
    seed, stp = 31, 2
    run(sim, packed, task, buf, 1, params(_lib.SAMPLE | _lib.RESET | _lib.COMMANDS), step0=stp, seed=seed)
    done = buf.dones[0].cpu().numpy().astype(bool)
    rs = buf.resets[0].cpu().numpy().astype(bool)
    assert done[:40].all()
    assert rs[:40].all() and rs[120:140].all()
    assert not done[120:140].any()
    # reset state: the reference reset kernel's formula, bit for bit
    qp, qv, an = host(sim["qpos"]), host(sim["qvel"]), host(sim["anchor"])
    r64 = [np.zeros((d, n)) for d in (36, 35, 16)]
    oracle.reset_done_soa(*r64, rs.astype(np.uint8), 42, 0.1, 0.02)
    assert np.array_equal(qp[:, rs], r64[0][:, rs]) and (qv[:, rs] == 0).all() and (an[:, rs] == np.float32(1e30)).all()
    el = task.ep_len.cpu().numpy()
    assert (el[rs] == 0).all() and (el[~rs] == 1).all()
    pa = task.prev_action.cpu().numpy()
    assert (pa[:, rs] == 0).all() and (pa[:, ~rs] == buf.actions[0].cpu().numpy().T[:, ~rs]).all()
    ct = task.cmd_timer.cpu().numpy()
    redrawn = rs | (np.arange(n) >= 80) & (np.arange(n) < 120)
    assert ((ct[redrawn] >= 150) & (ct[redrawn] < 250)).all()
    assert (ct[~redrawn] == 4).all()
    cmd = task.commands.cpu().numpy()
    assert np.array_equal(cmd[:, ~redrawn], cmd0.cpu().numpy()[:, ~redrawn])
    assert not np.array_equal(cmd[:, redrawn], cmd0.cpu().numpy()[:, redrawn])
    lo, hi = np.array([-1.0, -0.5, -1.0])[:, None], np.array([1.0, 0.5, 1.0])[:, None]
    assert ((cmd >= lo) & (cmd <= hi)).all()
    # the bootstrap observation is taken after the resets and redraws
    obs1 = obs_reference(qp, qv, cmd, host(sim["ctrl"]))
    assert np.abs(buf.last_obs.cpu().numpy() - obs1).max() < 1e-6


def test_one_launch_equals_step_by_step(net):
    ac, packed = net
    n, T = 300, 8
    allf = _lib.SAMPLE | _lib.PUSH | _lib.RESET | _lib.COMMANDS
    sa, sb = make_sim(n, seed=12), None
    sb = {k: v.clone() for k, v in sa.items()}
    ta, tb = P.TaskState(n, DEV, seed=13), P.TaskState(n, DEV, seed=13)
    ba, bb = P.RolloutBuffers(T, n, DEV), P.RolloutBuffers(T, n, DEV)
    run(sa, packed, ta, ba, T, params(allf), step0=0, seed=3)
    for k in range(T):
        run(sb, packed, tb, bb, 1, params(allf), step0=k, seed=3, bootstrap=(k == T - 1), t0=k)
    for x, y in ((ba.obs, bb.obs), (ba.actions, bb.actions), (ba.log_probs, bb.log_probs),
                 (ba.values, bb.values), (ba.rewards, bb.rewards), (ba.dones, bb.dones),
                 (ba.last_value, bb.last_value)):
        assert torch.equal(x, y)
    for k in sa:
        assert torch.equal(sa[k], sb[k]), k
    assert torch.isfinite(ba.rewards).all() and torch.isfinite(ba.values).all()


def test_invalid_arguments_are_rejected(net):
    ac, packed = net
    n = 64
    sim = make_sim(n)
    task = P.TaskState(n, DEV)
    sim_no_feet = dict(sim, foot_pos=None)
    with pytest.raises(RuntimeError, match="foot_pos"):
        P.policy_rollout(sim_no_feet, packed, task, None, 1)
    with pytest.raises(RuntimeError, match="decim"):
        P.policy_rollout(sim, packed, task, None, 1, decim=0)


def test_fused_network_vs_fp32_forward(net):
    """The accuracy cost of the kernel's BF16 network: its actor mean and
    critic value on the observations it built, against the reference's FP32
    ActorCritic.forward (examples/train.py:71-75) on the same observations
    and normaliser."""
    ac, packed = net
    n = 2048
    sim = make_sim(n, seed=12)
    task = P.TaskState(n, DEV, seed=13)
    buf = P.RolloutBuffers(4, n, DEV, mean=True)
    run(sim, packed, task, buf, 4, params(_lib.SAMPLE | _lib.RESET), seed=2)
    acd = ac.to(DEV)
    with torch.no_grad():
        obs = buf.obs.reshape(-1, 99)
        mean32, _ = acd(obs)
        val32 = acd.critic(acd.normalize_obs(obs)).squeeze(-1)
    dm = (buf.mean.reshape(-1, 29) - mean32).abs()
    dv = (buf.values.reshape(-1) - val32).abs()
    print(f"fused BF16 network vs FP32 forward, {obs.shape[0]} observations: actor mean |dev| median "
          f"{float(dm.median()):.2e} max {float(dm.max()):.2e} (|mean| avg {float(mean32.abs().mean()):.3f}); "
          f"critic |dev| median {float(dv.median()):.2e} max {float(dv.max()):.2e} "
          f"(|value| avg {float(val32.abs().mean()):.3f})")
    # measured: mean |dev| median 1.7e-3, max 2.2e-2; value median 1.9e-3, max 2.0e-2
    assert float(dm.median()) < 5e-3 and float(dm.max()) < 5e-2
    assert float(dv.median()) < 5e-3 and float(dv.max()) < 5e-2
