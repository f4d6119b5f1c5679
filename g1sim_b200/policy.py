"""Policy-fused rollout: the PPO actor-critic evaluated inside the step kernel.

Mirrors the reference's RL layer (examples/train.py):
  ActorCritic          same modules and state-dict names as the reference
                       (train.py:16-47), so a reference policy.pt loads as is
  pack_policy          ActorCritic -> the fused kernel's BF16 weight layout
  TaskState            per-env command / timers / previous action
                       (train.py:257-261, 264)
  PolicyRollout        npolicy policy steps of decim substeps in ONE kernel
                       launch: observation, normalisation, critic, actor,
                       sampling, PD targets, pushes, physics, reward,
                       termination, resets, command redraws
  reward_and_done      torch restatement of compute_reward_and_done
                       (train.py:143-218), used to check the kernel
  kernel_mlp_reference torch emulation of the kernel's network numerics
                       (BF16 operands and activations, FP32 accumulation)
  ppo_update / gae     the reference's PPO update and GAE
                       (train.py:104-121, 326-390)

Differences from the reference loop, by design of a fused rollout:
  * the observation normaliser is frozen during a rollout call and updated
    afterwards from the rollout's observations, batch by batch, with the
    reference's update rule (train.py:50-66); the reference updates it
    before every policy step;
  * the RNG streams of action noise, pushes and command draws are the
    kernel's counter-based hash, not torch's generator;
  * resets use the reference reset kernel's formula (seed 42, noise 0.1,
    drop 0.02: src/g1_kernel.cu:85-103, train.py:293) in the same kernel.
"""
import ctypes as C

import numpy as np
import torch
import torch.nn as nn

from . import _lib
from .model import g1_model_data as M

NOBS, NACT = 99, 29
OBS_PAD = 112
# (in, out, K pad, N pad, K chunk) of the critic's then the actor's layers
_LAYERS = {
    "critic": [(NOBS, 512, OBS_PAD, 512, 16), (512, 256, 512, 256, 32), (256, 128, 256, 128, 64),
               (128, 1, 128, 16, 128)],
    "actor": [(NOBS, 512, OBS_PAD, 512, 16), (512, 256, 512, 256, 32), (256, 128, 256, 128, 64),
              (128, NACT, 128, 32, 128)],
}
# reference src/g1sim.py:77-83
ACTION_SCALE = torch.tensor([
    0.443200, 0.274054, 0.443200, 0.274054, 0.365131, 0.365131,
    0.443200, 0.274054, 0.443200, 0.274054, 0.365131, 0.365131,
    0.443200, 0.365131, 0.365131,
    0.365131, 0.365131, 0.365131, 0.365131, 0.365131, 0.074501, 0.074501,
    0.365131, 0.365131, 0.365131, 0.365131, 0.365131, 0.074501, 0.074501], dtype=torch.float32)
# reference examples/train.py:244-256
STD_WALKING = torch.tensor([0.3, 0.15, 0.15, 0.35, 0.25, 0.1, 0.3, 0.15, 0.15, 0.35, 0.25, 0.1, 0.2, 0.08, 0.1,
                            0.15, 0.15, 0.1, 0.15, 0.3, 0.3, 0.3, 0.15, 0.15, 0.1, 0.15, 0.3, 0.3, 0.3])
STD_RUNNING = torch.tensor([0.5, 0.2, 0.2, 0.6, 0.35, 0.15, 0.5, 0.2, 0.2, 0.6, 0.35, 0.15, 0.3, 0.08, 0.2,
                            0.5, 0.2, 0.15, 0.35, 0.3, 0.3, 0.3, 0.5, 0.2, 0.15, 0.35, 0.3, 0.3, 0.3])


class ActorCritic(nn.Module):
    """The reference network (examples/train.py:16-47), same parameter names."""

    def __init__(self, num_obs=NOBS, num_actions=NACT):
        super().__init__()
        self.actor = nn.Sequential(nn.Linear(num_obs, 512), nn.ELU(), nn.Linear(512, 256), nn.ELU(),
                                   nn.Linear(256, 128), nn.ELU(), nn.Linear(128, num_actions))
        self.critic = nn.Sequential(nn.Linear(num_obs, 512), nn.ELU(), nn.Linear(512, 256), nn.ELU(),
                                    nn.Linear(256, 128), nn.ELU(), nn.Linear(128, 1))
        self.std = nn.Parameter(torch.zeros(num_actions))
        self.register_buffer("obs_mean", torch.zeros(num_obs))
        self.register_buffer("obs_var", torch.ones(num_obs))
        self.register_buffer("obs_count", torch.tensor(1e-4))
        self.clip_obs = 5.0

    def xavier_(self, generator=None):
        """Xavier-uniform weights, zero biases (the policy-fused workload's init)."""
        for seq in (self.actor, self.critic):
            for m in seq:
                if isinstance(m, nn.Linear):
                    nn.init.xavier_uniform_(m.weight, generator=generator)
                    nn.init.zeros_(m.bias)
        return self

    def update_obs_norm(self, obs):
        """Running mean / variance merge (reference train.py:50-66)."""
        batch_mean = obs.mean(dim=0)
        batch_var = obs.var(dim=0, unbiased=False)
        batch_count = obs.shape[0]
        delta = batch_mean - self.obs_mean
        tot_count = self.obs_count + batch_count
        new_mean = self.obs_mean + delta * batch_count / tot_count
        m_a = self.obs_var * self.obs_count
        m_b = batch_var * batch_count
        m2 = m_a + m_b + torch.square(delta) * self.obs_count * batch_count / tot_count
        self.obs_mean.copy_(new_mean)
        self.obs_var.copy_(m2 / tot_count)
        self.obs_count.copy_(tot_count)

    def normalize_obs(self, obs):
        return torch.clamp((obs - self.obs_mean) / torch.sqrt(self.obs_var + 1e-8), -self.clip_obs, self.clip_obs)

    def forward(self, obs):
        return self.actor(self.normalize_obs(obs)), self.std.exp()

    def evaluate(self, obs, action):
        """Log-prob, value and entropy (reference train.py:74-82)."""
        obs_norm = self.normalize_obs(obs)
        mean = self.actor(obs_norm)
        dist = torch.distributions.Normal(mean, self.std.exp())
        return dist.log_prob(action).sum(dim=-1), self.critic(obs_norm).squeeze(-1), dist.entropy().sum(dim=-1)


def _linears(seq):
    return [m for m in seq if isinstance(m, nn.Linear)]


def pack_weights(ac):
    """BF16 weight blob of the fused kernel: critic layers then actor layers;
    each W (out x in) zero-padded to N x K and stored per K-chunk of KC
    columns as [KC/8][N/8][8][8] (8x8 core matrices, K fastest)."""
    parts, biases = [], []
    for net in ("critic", "actor"):
        for lin, (fin, fout, kp, np_, kc) in zip(_linears(getattr(ac, net)), _LAYERS[net]):
            w = torch.zeros(np_, kp, dtype=torch.float32, device=lin.weight.device)
            w[:fout, :fin] = lin.weight.detach().float()
            w = w.to(torch.bfloat16)
            for c in range(kp // kc):
                sub = w[:, c * kc:(c + 1) * kc]  # (N, KC)
                parts.append(sub.reshape(np_ // 8, 8, kc // 8, 8).permute(2, 0, 1, 3).contiguous().reshape(-1))
            b = torch.zeros(np_, dtype=torch.float32, device=lin.weight.device)
            b[:fout] = lin.bias.detach().float()
            biases.append(b)
    return torch.cat(parts), torch.cat(biases)


class PackedPolicy:
    """Device copy of an ActorCritic in the kernel's layout."""

    def __init__(self, ac, device):
        wb, bb = pack_weights(ac)
        nbytes, nbias, _, _ = _lib.policy_sizes()
        assert wb.numel() * 2 == nbytes and bb.numel() == nbias, (wb.numel() * 2, nbytes, bb.numel(), nbias)
        self.weights = wb.to(device).contiguous()
        self.bias = bb.to(device).contiguous()
        self.log_std = ac.std.detach().float().to(device).contiguous()
        self.obs_mean = ac.obs_mean.detach().float().to(device).contiguous()
        self.obs_var = ac.obs_var.detach().float().to(device).contiguous()

    def struct(self):
        return _lib.Policy(self.weights.data_ptr(), self.bias.data_ptr(), self.log_std.data_ptr(),
                           self.obs_mean.data_ptr(), self.obs_var.data_ptr())


def pack_policy(ac, device="cuda"):
    return PackedPolicy(ac, device)


def load_policy_pt(path, device="cuda"):
    """An ActorCritic from a reference policy.pt (train.py:422-433)."""
    ac = ActorCritic()
    ac.load_state_dict(torch.load(path, map_location="cpu"))
    return ac.to(device)


def kernel_mlp_reference(ac, obs):
    """Torch emulation of the fused kernel's network numerics: normalised
    observation and hidden activations rounded to BF16, BF16 weights, FP32
    accumulation and bias.  Returns (actor mean, critic value)."""
    def run(seq, x):
        lins = _linears(seq)
        h = x.to(torch.bfloat16).float()
        for i, lin in enumerate(lins):
            h = h @ lin.weight.detach().to(torch.bfloat16).float().T + lin.bias.detach().float()
            if i + 1 < len(lins):
                h = torch.nn.functional.elu(h).to(torch.bfloat16).float()
        return h
    x = ac.normalize_obs(obs.float())
    return run(ac.actor, x), run(ac.critic, x).squeeze(-1)


class TaskState:
    """Per-env task state, SoA (reference train.py:257-261, 264)."""

    def __init__(self, nenv, device, seed=0, params=None):
        g = torch.Generator(device="cpu").manual_seed(seed)
        p = params or _lib.policy_default_params()
        lo = torch.tensor(list(p.cmd_lo)).unsqueeze(1)
        hi = torch.tensor(list(p.cmd_hi)).unsqueeze(1)
        self.commands = (lo + torch.rand(3, nenv, generator=g) * (hi - lo)).to(device).contiguous()
        self.prev_action = torch.zeros(NACT, nenv, device=device)
        self.cmd_timer = torch.zeros(nenv, dtype=torch.int32, device=device)  # train.py:257
        self.ep_len = torch.zeros(nenv, dtype=torch.int32, device=device)
        self.push_timer = torch.randint(p.push_steps_lo, p.push_steps_hi, (nenv,), generator=g,
                                        dtype=torch.int32).to(device)

    def struct(self):
        return _lib.TaskState(self.commands.data_ptr(), self.prev_action.data_ptr(), self.cmd_timer.data_ptr(),
                              self.ep_len.data_ptr(), self.push_timer.data_ptr())


def _ptr(t):
    return None if t is None else t.data_ptr()


class RolloutBuffers:
    """Kernel outputs of one rollout, [T][nenv][...] (reference train.py:94-101)."""

    def __init__(self, nsteps, nenv, device, mean=False):
        f = dict(device=device, dtype=torch.float32)
        self.obs = torch.zeros(nsteps, nenv, NOBS, **f)
        self.actions = torch.zeros(nsteps, nenv, NACT, **f)
        self.mean = torch.zeros(nsteps, nenv, NACT, **f) if mean else None
        self.log_probs = torch.zeros(nsteps, nenv, **f)
        self.values = torch.zeros(nsteps, nenv, **f)
        self.rewards = torch.zeros(nsteps, nenv, **f)
        self.dones = torch.zeros(nsteps, nenv, dtype=torch.uint8, device=device)
        self.resets = torch.zeros(nsteps, nenv, dtype=torch.uint8, device=device)
        self.last_obs = torch.zeros(nenv, NOBS, **f)
        self.last_value = torch.zeros(nenv, **f)

    def struct(self, t0=0):
        n = self.obs.shape[1]
        off = lambda x, w: None if x is None else x.data_ptr() + t0 * n * w * x.element_size()  # noqa: E731
        return _lib.RolloutOut(off(self.obs, NOBS), off(self.actions, NACT), off(self.mean, NACT),
                               off(self.log_probs, 1), off(self.values, 1), off(self.rewards, 1),
                               off(self.dones, 1), off(self.resets, 1), self.last_obs.data_ptr(),
                               self.last_value.data_ptr())


def policy_rollout(sim_state, packed, task, buffers, npolicy, decim=10, config=None, params=None, step0=0,
                   seed=0, mu=None, dmass=None, t0=0, stream=None, bootstrap=True):
    """npolicy policy steps in one launch of the fused kernel.

    sim_state: dict of the SoA tensors qpos, qvel, anchor, ctrl, foot_pos,
    foot_vel, contact_forces (device float32, [dim][nenv]).  Outputs go to
    buffers[t0 : t0 + npolicy]; with bootstrap, buffers.last_obs/last_value
    get the observation and value of the final state."""
    p = params or _lib.policy_default_params()
    p.seed = seed
    p.step0 = step0
    cfg = config or _lib.default_config(dt=2e-3)
    out = buffers.struct(t0) if buffers is not None else _lib.RolloutOut()
    if not bootstrap:
        out.last_obs = None
        out.last_value = None
    s = sim_state
    nenv = s["qpos"].shape[1]
    st = stream if stream is not None else torch.cuda.current_stream(s["qpos"].device).cuda_stream
    L = _lib.lib()
    _lib.check(L.g1b_policy_rollout(nenv, npolicy, decim, C.byref(cfg), C.byref(p), C.byref(packed.struct()),
                                    _ptr(s["qpos"]), _ptr(s["qvel"]), _ptr(s["anchor"]), _ptr(s["ctrl"]),
                                    _ptr(mu), _ptr(dmass), C.byref(task.struct()), C.byref(out),
                                    _ptr(s["foot_pos"]), _ptr(s["foot_vel"]), _ptr(s["contact_forces"]), st),
               "g1b_policy_rollout")


def reward_and_done(obs, actions, prev_actions, qpos, foot_pos, foot_vel, contact_forces,
                    std_walking=STD_WALKING, std_running=STD_RUNNING):
    """Torch restatement of the reference compute_reward_and_done
    (examples/train.py:143-218): obs (nenv, 99), actions / prev_actions
    (nenv, 29), qpos (36, nenv), foot arrays SoA.  Returns (reward, done)."""
    dev = obs.device
    sw, sr = std_walking.to(dev).unsqueeze(0), std_running.to(dev).unsqueeze(0)
    rng = torch.tensor(np.asarray(M.jnt_range), dtype=torch.float32, device=dev)
    lower, upper = rng[:, 0:1], rng[:, 1:2]
    commands, proj_gravity, lin_vel, ang_vel = obs[:, 0:3], obs[:, 3:6], obs[:, 6:9], obs[:, 9:12]
    xy_error = torch.sum(torch.square(commands[:, :2] - lin_vel[:, :2]), dim=1)
    rew_lin_vel = torch.exp(-(xy_error + torch.square(lin_vel[:, 2])) / 0.25)
    yaw_error = torch.square(commands[:, 2] - ang_vel[:, 2])
    roll_pitch = torch.sum(torch.square(ang_vel[:, :2]), dim=1)
    rew_ang_vel = torch.exp(-(yaw_error + roll_pitch) / 0.5)
    rew_orient = torch.exp(-torch.sum(torch.square(proj_gravity[:, :2]), dim=1) / 0.2)
    total_speed = torch.norm(commands[:, :2], dim=1) + torch.abs(commands[:, 2])
    standing = (total_speed < 0.05).float().unsqueeze(1)
    running = (total_speed >= 1.5).float().unsqueeze(1)
    walking = 1.0 - standing - running
    std = 0.05 * standing + sw * walking + sr * running
    rew_pose = torch.exp(-torch.mean(torch.square(obs[:, 12:41]) / (std ** 2), dim=1))
    rew_action_rate = torch.sum(torch.square(actions - prev_actions), dim=1)
    q = qpos[7:36, :]
    jr = upper - lower
    oob = torch.clamp(q - (upper - 0.05 * jr), min=0.0) + torch.clamp((lower + 0.05 * jr) - q, min=0.0)
    rew_dof_limits = torch.sum(oob, dim=0)
    lsq = torch.square(foot_vel[0]) + torch.square(foot_vel[1])
    rsq = torch.square(foot_vel[3]) + torch.square(foot_vel[4])
    active = (total_speed > 0.05).float()
    clearance = (torch.abs(foot_pos[2] - 0.1) * torch.sqrt(lsq + 1e-6) +
                 torch.abs(foot_pos[5] - 0.1) * torch.sqrt(rsq + 1e-6)) * active
    lc = (torch.sum(contact_forces[0:4], dim=0) > 1.0).float()
    rc = (torch.sum(contact_forces[4:8], dim=0) > 1.0).float()
    slip = (lsq * lc + rsq * rc) * active
    reward = (2.0 * rew_lin_vel + 2.0 * rew_ang_vel + rew_orient + rew_pose - rew_dof_limits - 2.0 * clearance -
              0.5 * slip - 0.05 * rew_action_rate - 0.05 * roll_pitch)
    tilt = torch.acos(torch.clamp(-proj_gravity[:, 2], -1.0, 1.0)).abs()
    done = (tilt > 70.0 * 3.14159 / 180.0).to(torch.uint8)
    return reward, done


def gae(rewards, values, dones, next_value, next_done, gamma=0.99, lam=0.95):
    """Returns and advantages (reference train.py:104-121, same indexing)."""
    T = rewards.shape[0]
    advs = torch.zeros_like(rewards)
    last = torch.zeros_like(next_value)
    for t in reversed(range(T)):
        if t == T - 1:
            nnt = 1.0 - next_done.float()
            nv = next_value
        else:
            nnt = 1.0 - dones[t + 1].float()
            nv = values[t + 1]
        delta = rewards[t] + gamma * nv * nnt - values[t]
        advs[t] = last = delta + gamma * lam * nnt * last
    return advs + values, advs


def ppo_update(ac, optimizer, buf, returns, advs, epochs=5, minibatches=4, clip=0.2, max_grad_norm=1.0,
               generator=None, perms=None):
    """PPO epochs x minibatches (reference train.py:330-390).  Returns mean KL.
    perms: optional minibatch order, one permutation of the samples per epoch
    (default: torch.randperm with `generator`)."""
    advs = (advs - advs.mean()) / (advs.std() + 1e-8)
    b_obs = buf.obs.reshape(-1, NOBS)
    b_actions = buf.actions.reshape(-1, NACT)
    b_logp = buf.log_probs.reshape(-1)
    b_returns = returns.reshape(-1)
    b_advs = advs.reshape(-1)
    b_values = buf.values.reshape(-1)
    n = b_obs.shape[0]
    mb = n // minibatches
    # the KL of each minibatch is summed on the device and read once at the end
    # (the reference reads it per minibatch, train.py:402-403; one sync instead of 20)
    kl_sum, count = torch.zeros((), dtype=torch.float64, device=b_obs.device), 0
    for ep in range(epochs):
        idx = perms[ep] if perms is not None else torch.randperm(n, device=b_obs.device, generator=generator)
        for s in range(0, n, mb):
            j = idx[s:s + mb]
            new_logp, values, entropy = ac.evaluate(b_obs[j], b_actions[j])
            ratio = torch.exp(new_logp - b_logp[j])
            surr = torch.min(ratio * b_advs[j], torch.clamp(ratio, 1 - clip, 1 + clip) * b_advs[j])
            vclip = b_values[j] + (values - b_values[j]).clamp(-clip, clip)
            critic_loss = torch.max((values - b_returns[j]).pow(2), (vclip - b_returns[j]).pow(2)).mean()
            loss = -surr.mean() + critic_loss - 0.01 * entropy.mean()
            optimizer.zero_grad()
            loss.backward()
            nn.utils.clip_grad_norm_(ac.parameters(), max_grad_norm)
            optimizer.step()
            with torch.no_grad():
                kl_sum += (b_logp[j] - new_logp).mean()
                count += 1
    return float(kl_sum.item()) / max(count, 1)
