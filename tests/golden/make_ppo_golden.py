#!/usr/bin/env python3
"""Generate tests/golden/ref_ppo.npz with the REFERENCE's own PPO pieces.

The reference's training script (examples/train.py) is imported from where
it lies, with its simulator module (src/g1sim.py, which needs MuJoCo)
replaced by a stub, so that its own ActorCritic (train.py:16-93) and
RolloutBuffer.compute_returns (train.py:102-141) run on CPU.  A synthetic
rollout (24 policy steps x 16 envs: observations, the reference network's
own sampled actions, log-probabilities and values, random rewards and
dones) is turned into returns and advantages by the reference buffer, and
one PPO update (5 epochs x 4 minibatches, train.py:330-373: normalised
advantages, clipped surrogate and value losses, entropy bonus, gradient-norm
clip 1.0, Adam lr 1e-3) is applied with fixed minibatch permutations (saved,
in place of the script's torch.randperm) to the reference network.  The
fixture holds a fingerprint of the network before (the test rebuilds it
from the same seed), 512 sampled entries of every tensor after, the buffer,
the permutations, the returns, advantages and the mean KL.

Run:  python tests/golden/make_ppo_golden.py [<reference root>]
      (default: $REF_SRC, else /root/reference)
"""
import importlib.util
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
T, N = 24, 16


def load_reference(root):
    src = types.ModuleType("src")
    stub = types.ModuleType("src.g1sim")
    stub.G1Sim = object  # the simulator is not used here
    sys.modules["src"], sys.modules["src.g1sim"] = src, stub
    spec = importlib.util.spec_from_file_location("ref_train", os.path.join(root, "examples", "train.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_SRC", "/root/reference")
    ref = load_reference(root)
    torch.manual_seed(0)
    ac = ref.ActorCritic(num_obs=99, num_actions=29)
    with torch.no_grad():
        ac.std.uniform_(-0.7, -0.3)
    ac.update_obs_norm(torch.randn(2048, 99) * 1.5 + 0.2)
    buf = ref.RolloutBuffer(N, T, 99, 29, "cpu")
    g = torch.Generator().manual_seed(1)
    for t in range(T):
        obs = torch.randn(N, 99, generator=g) * 1.5 + 0.2
        with torch.no_grad():
            act, logp, val = ac.act(obs, update_norm=False)
        rew = torch.randn(N, generator=g) * 0.5 + 1.0
        done = (torch.rand(N, generator=g) < 0.05).to(torch.uint8)
        buf.add(obs, act, logp, rew, done, val)
    next_obs = torch.randn(N, 99, generator=g) * 1.5 + 0.2
    with torch.no_grad():
        _, _, next_value = ac.act(next_obs, update_norm=False)
    next_done = (torch.rand(N, generator=g) < 0.05).to(torch.uint8)
    returns, advs = buf.compute_returns(next_value, next_done)
    sd0 = {k: v.detach().clone().numpy() for k, v in ac.state_dict().items()}

    # one PPO update as the reference script runs it, minibatch order fixed
    epochs, batch = 5, T * N
    mb = batch // 4
    clip, max_grad_norm = 0.2, 1.0
    opt = torch.optim.Adam(ac.parameters(), lr=1e-3)
    advs_n = (advs - advs.mean()) / (advs.std() + 1e-8)
    b_obs, b_act = buf.obs.reshape(-1, 99), buf.actions.reshape(-1, 29)
    b_logp, b_ret = buf.log_probs.reshape(-1), returns.reshape(-1)
    b_adv, b_val = advs_n.reshape(-1), buf.values.reshape(-1)
    perms = [torch.randperm(batch, generator=g) for _ in range(epochs)]
    kl_sum = 0.0
    for ep in range(epochs):
        for start in range(0, batch, mb):
            j = perms[ep][start:start + mb]
            new_logp, values, entropy = ac.evaluate(b_obs[j], b_act[j])
            ratio = torch.exp(new_logp - b_logp[j])
            surr1 = ratio * b_adv[j]
            surr2 = torch.clamp(ratio, 1.0 - clip, 1.0 + clip) * b_adv[j]
            actor_loss = -torch.min(surr1, surr2).mean()
            vclip = b_val[j] + (values - b_val[j]).clamp(-clip, clip)
            critic_loss = torch.max((values - b_ret[j]).pow(2), (vclip - b_ret[j]).pow(2)).mean()
            loss = actor_loss + 1.0 * critic_loss - 0.01 * entropy.mean()
            opt.zero_grad()
            loss.backward()
            torch.nn.utils.clip_grad_norm_(ac.parameters(), max_grad_norm)
            opt.step()
            with torch.no_grad():
                kl_sum += (b_logp[j] - new_logp).mean().item()
    # the network before: rebuilt by the test from the same seed, so only a
    # fingerprint of each tensor is kept; after: up to 512 sampled entries
    # per tensor (indices and values), which keeps the fixture small
    out = {}
    for k, v in sd0.items():
        a = v.astype(np.float64).ravel()
        out[f"sd0/{k}"] = np.array([a.sum(), (a * a).sum()] + list(a[:8]) + [0.0] * (8 - min(8, a.size)))
    rs = np.random.default_rng(2)
    for k, v in ac.state_dict().items():
        a = v.detach().numpy().ravel()
        idx = np.sort(rs.choice(a.size, size=min(512, a.size), replace=False))
        out[f"sd1_idx/{k}"], out[f"sd1_val/{k}"] = idx, a[idx]
    out.update(obs=buf.obs.numpy(), actions=buf.actions.numpy(), log_probs=buf.log_probs.numpy(),
               rewards=buf.rewards.numpy(), dones=buf.dones.numpy(), values=buf.values.numpy(),
               next_value=next_value.numpy(), next_done=next_done.numpy(), returns=returns.numpy(),
               advs=advs.numpy(), perms=torch.stack(perms).numpy(), mean_kl=np.array(kl_sum / (epochs * 4)))
    np.savez_compressed(os.path.join(HERE, "ref_ppo.npz"), **out)
    print("ref_ppo.npz", os.path.getsize(os.path.join(HERE, "ref_ppo.npz")), "bytes; mean KL", kl_sum / (epochs * 4))


if __name__ == "__main__":
    main()
