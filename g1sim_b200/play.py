"""Headless policy playback: the reference's examples/play.py loop without
the MuJoCo viewer, writing the trajectory to a .npy file instead of drawing
it (no graphics stack is used or needed).

    python -m g1sim_b200.play --policy build/policy.pt --steps 500 --out traj.npz

Loop (reference examples/play.py:93-118): observation, deterministic actor
output, targets default + action * action_scale, `nsub` substeps of 1 ms,
reset when the base tilts beyond 70 degrees or the state blows up.  The file
holds qpos [steps + 1, 36, nenv] (the initial state first), the commands and
the reset flags per step.
"""
import argparse
import os

import numpy as np
import torch

from . import policy as P
from .g1sim import G1Sim


def play(ac, steps=500, nenv=1, nsub=20, command=(0.0, 0.0, 0.0), device=None):
    device = device or torch.device("cuda", 0)
    ac = ac.to(device).eval()
    env = G1Sim(nenv=nenv, device=device)
    env.reset_all(noise=0.0)
    for i in range(3):
        env.commands[i].fill_(float(command[i]))
    traj = np.zeros((steps + 1, 36, nenv), dtype=np.float32)
    resets = np.zeros((steps, nenv), dtype=bool)
    traj[0] = env.qpos.cpu().numpy()
    with torch.no_grad():
        for t in range(steps):
            obs = env.get_obs()
            action = ac.actor(ac.normalize_obs(obs))
            env.ctrl[:] = env.default_joint_pos + action.T * env.action_scale
            env.step(nsub=nsub)
            q = env.qpos[3:7]
            grav_z = -(1.0 - 2.0 * (q[1] * q[1] + q[2] * q[2]))
            tilt = torch.acos(torch.clamp(-grav_z, -1.0, 1.0)).abs()
            bad = torch.isnan(env.qpos).any(0) | (env.qpos.abs().amax(0) > 1000.0) | (tilt > 1.2217)
            if bool(bad.any()):
                resets[t] = bad.cpu().numpy()
                env.reset_done(bad.to(torch.uint8), noise=0.0)
            traj[t + 1] = env.qpos.cpu().numpy()
    return traj, resets


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--policy", default=os.path.join("build", "policy.pt"))
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--nenv", type=int, default=1)
    ap.add_argument("--nsub", type=int, default=20)
    ap.add_argument("--vx", type=float, default=0.0)
    ap.add_argument("--vy", type=float, default=0.0)
    ap.add_argument("--wz", type=float, default=0.0)
    ap.add_argument("--out", default="traj.npz")
    a = ap.parse_args()
    if os.path.exists(a.policy):
        ac = P.load_policy_pt(a.policy, device="cpu")
    else:
        print(f"no policy at {a.policy}: playing a Xavier-initialised network")
        ac = P.ActorCritic().xavier_(torch.Generator().manual_seed(0))
    traj, resets = play(ac, a.steps, a.nenv, a.nsub, (a.vx, a.vy, a.wz))
    np.savez_compressed(a.out, qpos=traj, resets=resets, command=np.array([a.vx, a.vy, a.wz], np.float32),
                        dt=np.float32(1e-3 * a.nsub))
    print(f"wrote {a.out}: qpos {traj.shape}, {int(resets.sum())} resets")


if __name__ == "__main__":
    main()
