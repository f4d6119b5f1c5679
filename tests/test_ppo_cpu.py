"""The PPO pieces of the training loop against the reference's own (CPU).

tests/golden/ref_ppo.npz (tests/golden/make_ppo_golden.py) was produced by
the reference's ActorCritic and RolloutBuffer (examples/train.py:16-141) and
its PPO update (train.py:330-373) with fixed minibatch order.  Here the
network is rebuilt from the same seed (checked against the fixture's
fingerprint), policy.gae must reproduce the reference's returns and
advantages, and policy.ppo_update, run with the same minibatch order, must
reproduce the reference's parameters after 5 epochs x 4 minibatches and its
mean KL.
"""
import os
import types

import numpy as np
import torch

from g1sim_b200 import policy as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gae_and_ppo_update_match_reference():
    g = np.load(os.path.join(ROOT, "tests", "golden", "ref_ppo.npz"))
    torch.manual_seed(0)
    ac = P.ActorCritic(99, 29)
    with torch.no_grad():
        ac.std.uniform_(-0.7, -0.3)
    ac.update_obs_norm(torch.randn(2048, 99) * 1.5 + 0.2)
    for k, v in ac.state_dict().items():
        a = v.detach().double().numpy().ravel()
        fp = np.array([a.sum(), (a * a).sum()] + list(a[:8]) + [0.0] * (8 - min(8, a.size)))
        assert np.allclose(fp, g[f"sd0/{k}"], rtol=1e-12, atol=1e-12), k
    t = lambda k: torch.tensor(g[k])  # noqa: E731
    returns, advs = P.gae(t("rewards"), t("values"), t("dones"), t("next_value"), t("next_done"))
    assert torch.allclose(returns, t("returns"), rtol=1e-6, atol=1e-6)
    assert torch.allclose(advs, t("advs"), rtol=1e-6, atol=1e-6)
    buf = types.SimpleNamespace(obs=t("obs"), actions=t("actions"), log_probs=t("log_probs"), values=t("values"))
    opt = torch.optim.Adam(ac.parameters(), lr=1e-3)
    kl = P.ppo_update(ac, opt, buf, returns, advs, perms=[torch.tensor(p) for p in g["perms"]])
    for k, v in ac.state_dict().items():
        got = v.detach().numpy().ravel()[g[f"sd1_idx/{k}"]]
        assert np.allclose(got, g[f"sd1_val/{k}"], rtol=1e-5, atol=1e-6), k
    assert abs(kl - float(g["mean_kl"])) <= 1e-5 * max(1.0, abs(float(g["mean_kl"])))
