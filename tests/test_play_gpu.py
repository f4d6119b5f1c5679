"""Headless playback (g1sim_b200.play) on the GPU: a saved policy.pt plays
for a few hundred policy steps and the trajectory file holds finite states
(needs a B200)."""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from g1sim_b200 import policy as P

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_play_writes_trajectory(tmp_path):
    ac = P.ActorCritic().xavier_(torch.Generator().manual_seed(0))
    pt = tmp_path / "policy.pt"
    torch.save(ac.state_dict(), pt)
    out = tmp_path / "traj.npz"
    r = subprocess.run([sys.executable, "-m", "g1sim_b200.play", "--policy", str(pt), "--steps", "100", "--nenv", "4",
                        "--out", str(out)], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    d = np.load(out)
    assert d["qpos"].shape == (101, 36, 4) and d["resets"].shape == (100, 4)
    assert np.isfinite(d["qpos"]).all()
    q = d["qpos"][:, 3:7]
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-4)
