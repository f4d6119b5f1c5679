#!/usr/bin/env python3
"""Benchmark of the B200 G1 step on the randomised 65,536-env workload.

Workload (per GPU): 65,536 envs, dt = 2 ms, decimation 10, 1,000 substeps
(100 policy steps) per bench step; PD targets stand + U(-0.3, 0.3) x range
redrawn on the device each policy step; per-env friction U[0.4, 1.0] and
base-mass offset U[-1, +3] kg; initial base height U[0.75, 0.85] m; envs
reset in the kernel when the base height drops below 0.3 m.  A bench step
replays one CUDA graph holding the 100 policy-step launches (state goes
through HBM between policy steps, as in an RL loop).

Metric: env-steps/s, one env-step = one physics substep of one env (the
reference's nenv * nsteps * nsub, src/g1_kernel.cu:238).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun); every rank runs its own 65,536
envs (independent replicas, no collective on the data path); the timed
region is bracketed by barriers and the max over ranks is reported.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic work per env-substep (FP32 flops, FMA = 2): the reference
# algorithm's counted add/sub/mul with its per-step recomputation of constant
# tree rotations, spatial inertias and hinge S vectors removed.
FLOPS_PER_ENV_STEP = 36600.0
# The same count with the reference's per-step recomputation kept (its code as
# written, 8 contacts active), reported alongside.
FLOPS_PER_ENV_STEP_AS_WRITTEN = 40544.0
# FP32 flops executed per env-substep by split_kernel (ncu: FFMA x 2 + FADD +
# FMUL thread instructions of one 16,384-env launch over its env-substeps).
FLOPS_EXECUTED_PER_ENV_STEP = 31385.0
# Algorithmic bytes per env per launch: SoA state in (qpos 36, qvel 35,
# anchor 16, ctrl 29, mu, dmass) and out (qpos, qvel, anchor, ctrl), float32.
BYTES_PER_ENV_LAUNCH = 4.0 * ((36 + 35 + 16 + 29 + 2) + (36 + 35 + 16 + 29))

# DRAM bytes per env of the bench step's launch (split_kernel, 100 policy steps
# = 1,000 substeps): dram__bytes_read.sum + dram__bytes_write.sum, mean of two
# ncu captures at 16,384 envs (6,554,880 and 6,892,032 B;
# profiles/split_kernel_65536env_launch_list.md), scaled by envs.  One
# policy-step launch moved 6,105,088 B at 16,384 envs
# (profiles/split_kernel_16384env_full.md).
NCU_DRAM_BYTES_PER_ENV_PERSISTENT = 6723456.0 / 16384

NENV = 65536
SUBSTEPS = 1000
DECIM = 10
DT = 2e-3


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nenv", type=int, default=NENV)
    p.add_argument("--npolicy", type=int, default=1, help="policy steps per launch with --part plain")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--surrogate-steps", type=int, default=3000, help="training steps of the surrogate (-1: skip)")
    p.add_argument("--part", default="all",
                   choices=["all", "plain", "policy", "adjoint", "gemm", "surrogate", "surtrain", "ppo"],
                   help="one sub-benchmark alone on --nenv envs (rows), one GPU (a small case for a profiler)")
    p.add_argument("--horizon", type=int, default=64, help="adjoint horizon with --part adjoint")
    return p.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------- distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# -------------------------------------------------------- CPU baseline
def _host_cpus():
    try:
        return sorted(os.sched_getaffinity(0))
    except AttributeError:
        return list(range(os.cpu_count() or 1))


def cpu_reference(seconds, nenv, precision=4):
    """The reference's own step (oracle/_ref/g1ref_rollout, built from the
    reference sources; g1ref_rollout64 for its FP64 host build) on this
    host's CPUs: one single-threaded process per CPU, pinned to it, each on
    its own contiguous slice of the nenv envs (all 1,000 substeps of each
    env), until its slice is done or `seconds` have passed.  Throughput =
    env-steps of all processes / the longest process time."""
    exe = os.path.join(ROOT, "oracle", "_ref", "g1ref_rollout" if precision == 4 else "g1ref_rollout64")
    if not os.path.exists(exe):
        return None
    cpus = _host_cpus()
    per = (nenv + len(cpus) - 1) // len(cpus)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    procs = []
    for i, c in enumerate(cpus):
        cmd = ["taskset", "-c", str(c), exe, "--nenv", str(nenv), "--env0", str(i * per), "--count", str(per),
               "--steps", str(SUBSTEPS), "--decim", str(DECIM), "--seconds", str(seconds), "--threads", "1"]
        procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, env=env))
    res = []
    for p in procs:
        out, _ = p.communicate(timeout=seconds * 10 + 120)
        if p.returncode != 0:
            return None
        res.append(json.loads(out.strip().splitlines()[-1]))
    steps = sum(r["env_steps"] for r in res)
    wall = max(r["seconds"] for r in res)
    envs = sum(r["envs"] for r in res)
    name = "FP32 g1_step" if precision == 4 else "FP64 host build of g1_step"
    return {"value": steps / wall, "unit": "env-steps/s", "cores": len(cpus), "kind": "reference",
            "sample": (f"{envs} of the {nenv} envs x {SUBSTEPS} substeps (dt 2 ms, decimation 10, target redraw, "
                       f"reset at z<0.3; nominal friction/mass: the reference has no per-env parameters), "
                       f"reference {name}, one pinned single-threaded process per host CPU "
                       f"({len(cpus)}) on its own env slice, {wall:.1f} s")}


def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    ws = []
    res = None
    for i in range(args.warmup + args.steps):
        r = cpu_reference(4.0, args.nenv)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/g1ref_rollout is not built "
                                                                  "(make -C oracle ref needs the reference sources)"}))
            return 0
        if i >= args.warmup:
            ws.append(r["value"])
            res = r
    v = statistics.mean(ws)
    line = {"impl": "reference", "metric": "env-steps/s", "value": v, "unit": "env-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"randomised plain step, {args.nenv} envs, dt 2 ms, decimation 10, "
                                   f"{SUBSTEPS} substeps", "envs": args.nenv, "substeps": SUBSTEPS,
                       "decimation": DECIM, "dt": DT},
            "cpu_baseline": {"value": v, "unit": "env-steps/s", "cores": res["cores"], "kind": "reference",
                             "sample": res["sample"]},
            "e2e": {"value": v, "unit": "env-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------- accuracy leg
ACC_ENVS = 1024


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    import parity
    return Oracle(), parity


def accuracy_plain(state, mu, dmass, device):
    """Checker, outside the timed region: 1,024 envs sampled evenly from the
    timed state (after its 1,000 substeps), stepped by the same kernels one
    substep at a time for one policy step (10 substeps, targets held) and
    compared with the FP64 oracle from the same float32 state each substep;
    then the 400-substep drift of a GPU rollout from the oracle's, both from
    that state."""
    import torch
    from g1sim_b200 import _lib
    from g1sim_b200 import g1sim as G
    o, parity = _oracle()
    n = state["qpos"].shape[1]
    idx = torch.arange(0, n, max(1, n // ACC_ENVS), device=device)[:ACC_ENVS]
    sub = {k: state[k][:, idx].contiguous() for k in ("qpos", "qvel", "anchor", "ctrl")}
    smu, sdm = mu[idx].contiguous(), dmass[idx].contiguous()
    gcfg = _lib.default_config(dt=DT)
    ocfg = o.config(dt=DT)
    h = lambda t: t.double().cpu().numpy()  # noqa: E731
    ctrl, mu64, dm64 = h(sub["ctrl"]), h(smu), h(sdm)

    def read():
        torch.cuda.synchronize()
        return h(sub["qpos"]), h(sub["qvel"]), h(sub["anchor"])

    def run(k):
        G.step(sub["qpos"], sub["qvel"], sub["anchor"], sub["ctrl"], k, config=gcfg, mu=smu, dmass=sdm)

    per = parity.per_substep(o, lambda: run(1), read, ocfg, ctrl, mu=mu64, dmass=dm64, substeps=DECIM)
    dr = parity.drift(o, run, read, ocfg, ctrl, mu=mu64, dmass=dm64, marks=(10, 100, 400))
    mapping, block, _ = _lib.get_launch()
    return {"envs": int(idx.numel()), "per_substep": per, "drift": dr,
            "kernel": f"g1b_step, launch shape mapping {mapping} block {block} (the timed kernel's physics)",
            "sample": f"every {max(1, n // ACC_ENVS)}th env of the timed state after {SUBSTEPS} substeps",
            "metric": "|x - x_fp64| / max(|x_fp64|, 1) per component, from the same float32 state; "
                      "env-substeps within FP32 rounding of a model switch (oracle margin < 1) excluded"}


def accuracy_policy(sim, packed, task, mu, dmass, device):
    """Checker, outside the timed region: one more policy step of the fused
    kernel over all envs with action sampling only (no pushes, resets or
    command redraws, so its 10 substeps run from the pre-step state with the
    targets the network chose); 1,024 sampled envs are compared with the
    FP64 oracle's 10 substeps from the same float32 state and targets, and
    the plain kernel's 10 substeps from that state the same way."""
    import torch
    from g1sim_b200 import _lib
    from g1sim_b200 import g1sim as G
    from g1sim_b200 import policy as P
    o, parity = _oracle()
    n = sim["qpos"].shape[1]
    idx = torch.arange(0, n, max(1, n // ACC_ENVS), device=device)[:ACC_ENVS]
    h = lambda t: t.double().cpu().numpy()  # noqa: E731
    pre = {k: sim[k][:, idx].contiguous() for k in ("qpos", "qvel", "anchor")}
    pre64 = {k: h(v) for k, v in pre.items()}
    pr = _lib.policy_default_params()
    pr.flags = _lib.SAMPLE
    buf = P.RolloutBuffers(1, n, device)
    P.policy_rollout(sim, packed, task, buf, 1, decim=DECIM, params=pr, mu=mu, dmass=dmass)
    torch.cuda.synchronize()
    ctrl = sim["ctrl"][:, idx].contiguous()
    fq, fv = h(sim["qpos"][:, idx]), h(sim["qvel"][:, idx])
    G.step(pre["qpos"], pre["qvel"], pre["anchor"], ctrl, DECIM, config=_lib.default_config(dt=DT),
           mu=mu[idx].contiguous(), dmass=dmass[idx].contiguous())
    torch.cuda.synchronize()
    pq, pv = h(pre["qpos"]), h(pre["qvel"])
    eq, ev, mg = parity.composed(o, pre64["qpos"], pre64["qvel"], pre64["anchor"], h(ctrl), fq, fv,
                                 o.config(dt=DT), DECIM, mu=h(mu[idx]), dmass=h(dmass[idx]))
    # the plain kernel against the oracle from the same start with the same targets
    eq2, ev2, _ = parity.composed(o, pre64["qpos"], pre64["qvel"], pre64["anchor"], h(ctrl), pq, pv,
                                  o.config(dt=DT), DECIM, mu=h(mu[idx]), dmass=h(dmass[idx]))
    st = lambda a: {"median": float(np.median(a)), "p99": float(np.percentile(a, 99)),  # noqa: E731
                    "max": float(a.max())}
    return {"envs": int(idx.numel()), "substeps": DECIM,
            "fused": {"qpos": st(eq), "qvel": st(ev)}, "plain_same_start": {"qpos": st(eq2), "qvel": st(ev2)},
            "fused_vs_plain_max_abs": float(max(np.abs(fq - pq).max(), np.abs(fv - pv).max())),
            "metric": "|x - x_fp64| / max(|x_fp64|, 1) after 10 compounded substeps (one policy step), "
                      "per env the max over components; both from the same float32 state and targets"}


# ------------------------------------------------- policy-fused rollout
# Actor and critic multiply-accumulates per env and policy step
# (99-512-256-128-29 and 99-512-256-128-1, unpadded).
ACTOR_MACS = 99 * 512 + 512 * 256 + 256 * 128 + 128 * 29
CRITIC_MACS = 99 * 512 + 512 * 256 + 256 * 128 + 128 * 1
POLICY_T = 25  # policy steps per launch (a PPO rollout's length); 4 launches = 1,000 substeps


def policy_fused_bench(n, rank, device, stream, steps, warmup, world, local, init):
    """The same 1,000 substeps per bench step, with the PPO actor and critic
    evaluated inside the step kernel on the tensor cores every 10 substeps:
    observation, sampling, targets, pushes, reward, termination and resets
    in the kernel; every output buffer (obs, actions, log-probs, values,
    rewards, dones) written."""
    import torch
    from g1sim_b200 import policy as P
    sim = {k: init[k].clone() for k in ("qpos", "qvel", "anchor", "ctrl")}
    for k, d in (("foot_pos", 6), ("foot_vel", 6), ("contact_forces", 8)):
        sim[k] = torch.zeros(d, n, device=device)
    sim0 = {k: v.clone() for k, v in sim.items()}
    ac = P.ActorCritic().xavier_(torch.Generator().manual_seed(0))
    packed = P.pack_policy(ac, device)
    task = P.TaskState(n, device, seed=rank)
    buf = P.RolloutBuffers(POLICY_T, n, device)
    nlaunch = SUBSTEPS // (DECIM * POLICY_T)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)  # 256 MB > L2

    def one():
        with torch.cuda.stream(stream):
            for k in sim:
                sim[k].copy_(sim0[k])
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for j in range(nlaunch):
                P.policy_rollout(sim, packed, task, buf, POLICY_T, decim=DECIM, step0=j * POLICY_T, seed=rank,
                                 mu=init["mu"], dmass=init["dmass"], stream=stream.cuda_stream,
                                 bootstrap=(j == nlaunch - 1))
            e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(warmup):
        one()
    barrier(world)
    times = [one() for _ in range(steps)]
    ms = max_over_ranks(statistics.mean(times), world, device)
    from g1sim_b200 import _lib
    status = _lib.policy_status()
    acc = accuracy_policy(sim, packed, task, init["mu"], init["dmass"], device) if rank == 0 else None
    env_steps = float(n) * SUBSTEPS
    net_flops = 2.0 * (ACTOR_MACS + CRITIC_MACS) * n * (SUBSTEPS // DECIM)
    return {"value": env_steps * world / (ms * 1e-3), "unit": "env-steps/s", "ms_per_step": ms,
            "kernel": f"policy_kernel (128 envs per CTA, {POLICY_T} policy steps per launch, {nlaunch} launches)",
            "network_tflops": net_flops / (ms * 1e-3) / 1e12,
            "network_flops_per_env_policy_step": 2.0 * (ACTOR_MACS + CRITIC_MACS),
            "outputs": "obs, actions, log-probs, values, rewards, dones, resets, bootstrap value",
            "status": status, "finite": bool(torch.isfinite(buf.rewards).all().item()), "accuracy": acc}


# -------------------------------------------- PPO iteration (config 3)
PPO_ENVS, PPO_T = 16384, 24


def policy_ppo_bench(device, iters=4, n=PPO_ENVS, T=PPO_T):
    """The policy-fused training workload end to end: per iteration one
    launch of the fused kernel for T = 24 policy steps of 16,384 envs
    (decimation 10: observation, critic and actor on the tensor cores,
    sampling, physics, reward, resets), the observation normaliser update,
    GAE (gamma 0.99, lambda 0.95) and the PPO update (5 epochs x 4
    minibatches, Adam, the reference's losses), then the weights repacked for
    the kernel.  Xavier-initialised network; velocity commands vx, yaw in
    U[-1, 1], vy in U[-0.5, 0.5].  Also the deviation of the kernel's BF16
    network from the reference's FP32 ActorCritic.forward on the first
    rollout's observations."""
    import torch
    from g1sim_b200 import g1sim as G
    from g1sim_b200 import policy as P
    torch.manual_seed(0)
    ac = P.ActorCritic().xavier_(torch.Generator().manual_seed(0)).to(device)
    opt = torch.optim.Adam(ac.parameters(), lr=1e-3)
    sim = {"qpos": torch.zeros(36, n, device=device), "qvel": torch.zeros(35, n, device=device),
           "anchor": torch.zeros(16, n, device=device), "ctrl": torch.zeros(29, n, device=device)}
    for k, d in (("foot_pos", 6), ("foot_vel", 6), ("contact_forces", 8)):
        sim[k] = torch.zeros(d, n, device=device)
    G.reset_done(sim["qpos"], sim["qvel"], sim["anchor"], torch.ones(n, dtype=torch.uint8, device=device), seed=42,
                 noise=0.1, drop=0.02)
    sim["ctrl"].copy_(sim["qpos"][7:])
    task = P.TaskState(n, device, seed=0)
    buf = P.RolloutBuffers(T, n, device, mean=True)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    rows, dev_stats = [], None
    for it in range(iters):
        packed = P.pack_policy(ac, device)
        e0, e1, e2, e3 = ev(), ev(), ev(), ev()
        e0.record()
        P.policy_rollout(sim, packed, task, buf, T, decim=DECIM, step0=it * T, seed=it, bootstrap=True)
        e1.record()
        if it == 0:
            with torch.no_grad():
                obs = buf.obs.reshape(-1, 99)
                mean32, _ = ac(obs)
                val32 = ac.critic(ac.normalize_obs(obs)).squeeze(-1)
                dm = (buf.mean.reshape(-1, 29) - mean32).abs()
                dv = (buf.values.reshape(-1) - val32).abs()
                dev_stats = {"samples": int(obs.shape[0]),
                             "actor_mean_abs_dev": {"median": float(dm.median()), "max": float(dm.max())},
                             "actor_mean_scale": float(mean32.abs().mean()),
                             "critic_value_abs_dev": {"median": float(dv.median()), "max": float(dv.max())},
                             "critic_value_scale": float(val32.abs().mean())}
        ac.update_obs_norm(buf.obs.reshape(-1, 99))
        returns, advs = P.gae(buf.rewards, buf.values, buf.dones, buf.last_value, buf.dones[-1])
        e2.record()
        kl = P.ppo_update(ac, opt, buf, returns, advs, epochs=5, minibatches=4)
        e3.record()
        torch.cuda.synchronize()
        rows.append({"rollout_ms": e0.elapsed_time(e1), "gae_ms": e1.elapsed_time(e2), "update_ms": e2.elapsed_time(e3),
                     "mean_reward": float(buf.rewards.mean()), "mean_kl": kl})
    it_ms = statistics.mean(r["rollout_ms"] + r["gae_ms"] + r["update_ms"] for r in rows[1:] or rows)
    return {"envs": n, "policy_steps_per_rollout": T, "decimation": DECIM, "iterations": iters,
            "iteration_ms": it_ms, "env_steps_per_s_with_update": n * T * DECIM / (it_ms * 1e-3),
            "rollout_ms": statistics.mean(r["rollout_ms"] for r in rows[1:] or rows),
            "update_ms": statistics.mean(r["update_ms"] for r in rows[1:] or rows),
            "per_iteration": rows, "bf16_network_vs_fp32_forward": dev_stats,
            "ppo": "5 epochs x 4 minibatches of 98,304 samples, clip 0.2, Adam lr 1e-3, max grad norm 1"}


# ------------------------------------------------------- horizon adjoint
ADJ_ENVS, ADJ_H, ADJ_C = 4096, 64, 8


def adjoint_bench(device, stream, steps, warmup, world, n=ADJ_ENVS, horizon=ADJ_H):
    """Loss and gradients over a 64-step horizon at dt 2 ms for 4,096 envs
    (targets 64 x 29 and per-env kp / kd scales U[0.8, 1.2]), checkpoints
    every 8 steps: forward rollout + reverse sweep, one g1b_adjoint call.
    n and horizon change the envs and the horizon (smaller profiler cases)."""
    import torch
    from g1sim_b200 import adjoint as A
    from g1sim_b200.model import g1_model_data as M
    rng = np.random.default_rng(0)
    H = horizon
    stand = np.asarray(M.qpos_stand)
    q0 = np.repeat(stand[:, None], n, axis=1)
    q0[2] = 0.79
    q0[7:] += rng.normal(0, 0.02, size=(29, n))
    f = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=torch.float32, device=device)  # noqa: E731
    tg = f(stand[7:][None, :, None] + rng.normal(0, 0.05, size=(H, 29, n)))
    kp, kd = f(rng.uniform(0.8, 1.2, n)), f(rng.uniform(0.8, 1.2, n))
    qp, qv, an = f(q0), f(np.zeros((35, n))), f(np.full((16, n), 1e30))
    scratch = torch.empty(A.scratch_size(n, H, ADJ_C), dtype=torch.float32, device=device)

    def one():
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = A.horizon_adjoint(tg, kp, kd, qp, qv, an, checkpoint=ADJ_C, scratch=scratch,
                                  stream=stream.cuda_stream)
            e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1), r

    for _ in range(max(1, warmup)):
        one()
    times, r = [], None
    with ClockSampler(device.index if device.index is not None else 0) as clk:
        for _ in range(max(3, steps)):
            t, r = one()
            times.append(t)
    ms = max_over_ranks(statistics.mean(times), world, device)
    # the plain step on the same envs for the same horizon (H substeps, one launch), for the cost ratio
    from g1sim_b200 import _lib
    from g1sim_b200 import g1sim as G
    pq, pv, pa, pc = qp.clone(), qv.clone(), an.clone(), tg[0].contiguous()
    cfg = _lib.default_config(dt=DT)
    with torch.cuda.stream(stream):
        G.step(pq, pv, pa, pc, H, config=cfg, kp_scale=kp, kd_scale=kd)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(5):
            G.step(pq, pv, pa, pc, H, config=cfg, kp_scale=kp, kd_scale=kd)
        e1.record(stream)
    stream.synchronize()
    plain_ms = e0.elapsed_time(e1) / 5
    return {"value": float(n) * H * world / (ms * 1e-3), "unit": "env-steps/s (horizon steps differentiated)",
            "ms_per_call": ms, "ms_per_call_each": times, "clocks": clk.summary(),
            "plain_step_same_envs": {"ms": plain_ms, "value": float(n) * H / (plain_ms * 1e-3),
                                     "note": f"g1b_step, {n} envs x {H} substeps in one launch"},
            "cost_vs_plain_same_envs": ms / plain_ms,
            "config": {"envs": n, "horizon": H, "checkpoint": ADJ_C, "dt": DT,
                                         "decision_variables": f"targets {H}x29 + kp/kd scale per env"},
            "kernels": "adj_kernel<float, 32> (one launch: forward rollout with checkpoints, then per segment the "
                       "recomputed states and the reverse-mode product of each step; tape in shared memory)",
            "finite": bool(torch.isfinite(r["grad_targets"]).all().item())}


def measured_bf16_peak(key="bf16_tflops"):
    """A measured dense BF16 figure of this pool's B200s: the burst one, or
    key="bf16_tflops_sustained" for work timed inside a long loop."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)[key])
    except (OSError, KeyError, ValueError):
        return None


# ------------------------------------------------------ dynamics surrogate
SUR_ENVS, SUR_GEN_STEPS, SUR_BATCH = 65536, 153, 65536  # 10.0M transitions


def surrogate_bench(device, train_steps, world):
    """Config of the learned dynamics surrogate: 10.0M transitions of the
    randomised workload's simulator (65,536 envs x 153 steps), MLP 4 x 512
    SiLU trained with batch 65,536 on the library's kernels (BF16 tcgen05
    GEMMs, FP32 accumulation), then a 50-step rollout of 65,536 envs with
    per-env fallback to the exact step where the one-step error exceeds 1e-3."""
    import torch
    from g1sim_b200 import surrogate as S
    sur = S.Surrogate(device, seed=0)
    t0 = time.perf_counter()
    F, A = S.generate_transitions(sur, SUR_ENVS, SUR_GEN_STEPS, device, seed=1)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    S.fit_normalisation(sur, F, A)
    X, T = S.normalise(sur, F, A)
    del F
    g = torch.Generator(device=device).manual_seed(0)
    idx = torch.randint(0, X.shape[0], (SUR_BATCH,), generator=g, device=device)
    xb, tb = X[idx].contiguous(), T[idx].contiguous()
    sur.forward(xb, keep=True)
    l0 = float(sur.backward(xb, tb).item())
    # timed training steps (the same minibatch each step keeps the timed region to the kernels):
    # the CUDA graph of the step the library's training loop replays, and the eager launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    tg = sur.capture_train_step(xb, tb, lr=1e-3)
    timed = {}
    for name, fn in (("graph", tg.step), ("eager", lambda: sur.train_step(xb, tb, lr=1e-3))):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(10):
            fn()
        e1.record()
        torch.cuda.synchronize()
        timed[name] = e0.elapsed_time(e1) / 10
    step_ms = timed["graph"]
    train_tflops = S.train_flops(SUR_BATCH) / (step_ms * 1e-3) / 1e12
    # inference throughput of the network alone (features in HBM)
    e0.record()
    for _ in range(10):
        sur.forward(xb)
    e1.record()
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / 10
    # the rest of the training budget on random minibatches (gathered into the graph's buffers)
    loss = None
    for k in range(train_steps):
        idx = torch.randint(0, X.shape[0], (SUR_BATCH,), generator=g, device=device)
        torch.index_select(X, 0, idx, out=xb)
        torch.index_select(T, 0, idx, out=tb)
        loss = tg.step(2e-3 * (0.05 ** (k / max(train_steps, 1))))
    torch.cuda.synchronize()
    l1 = float(loss.item()) if loss is not None else l0
    from g1sim_b200 import workloads
    w = workloads.randomized(nenv=SUR_ENVS, seed=7)
    st = {k: torch.tensor(w[k], dtype=torch.float32, device=device) for k in ("qpos", "qvel", "anchor", "ctrl")}
    mu, dm = (torch.tensor(w[k], dtype=torch.float32, device=device) for k in ("mu", "dmass"))
    from g1sim_b200 import g1sim as G
    G.rollout(st["qpos"], st["qvel"], st["anchor"], st["ctrl"], 20, DECIM, config=_cfg(), seed=7, mu=mu, dmass=dm)
    st_loose = {k: v.clone() for k, v in st.items()}
    frac, err = S.rollout_with_fallback(sur, st, 50, bound=1e-3, mu=mu, dmass=dm)
    frac_loose, _ = S.rollout_with_fallback(sur, st_loose, 50, bound=1e-1, mu=mu, dmass=dm)
    ref = refinement_bench(sur, device)
    peak, sustained = measured_bf16_peak(), measured_bf16_peak("bf16_tflops_sustained")
    return {"train_step_ms": step_ms, "train_step_eager_ms": timed["eager"], "train_tflops": train_tflops,
            "train_frac_of_bf16_peak": (train_tflops / peak) if peak else None,
            "train_frac_of_bf16_sustained": (train_tflops / sustained) if sustained else None,
            "bf16_peak_tflops": peak, "bf16_peak_source": "MEASURED_PEAKS.json bf16_tflops (burst), of measured",
            "train_flops_per_step": S.train_flops(SUR_BATCH),
            "inference": {"value": SUR_BATCH / (fwd_ms * 1e-3), "unit": "env-steps/s (network forward only)"},
            "transitions": int(X.shape[0]), "generation_s": gen_s, "train_steps": train_steps,
            "loss_start": l0, "loss_end": l1,
            "fallback_rollout": {"envs": SUR_ENVS, "steps": 50, "bound": 1e-3, "start": "after 20 policy steps",
                                 "fraction_surrogate": frac, "one_step_error": err,
                                 "second_bound": {"bound": 1e-1, "fraction_surrogate": frac_loose}},
            "refinement": ref,
            "gemm_status": S.gemm_status()}


def plain_bench(device, n, steps, warmup, npolicy=1):
    """The plain step alone: `npolicy` policy steps (10 substeps, target
    redraw, reset check each) of n randomised envs per launch, `warmup` +
    `steps` launches, CUDA-event timed (a small case for a profiler)."""
    import torch
    from g1sim_b200 import _lib, workloads
    from g1sim_b200 import g1sim as G
    w = workloads.randomized(nenv=n, seed=0)
    st = {k: torch.tensor(w[k], dtype=torch.float32, device=device)
          for k in ("qpos", "qvel", "anchor", "ctrl", "mu", "dmass")}
    run = lambda k: G.rollout(st["qpos"], st["qvel"], st["anchor"], st["ctrl"], npolicy, DECIM,  # noqa: E731
                              config=_cfg(), seed=0, step0=k * npolicy, mu=st["mu"], dmass=st["dmass"])
    for k in range(warmup):
        run(k)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(steps):
        run(warmup + k)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(steps, 1)
    mapping, block, _ = _lib.get_launch()
    return {"ms_per_launch": ms, "policy_steps_per_launch": npolicy,
            "env_steps_per_s": n * DECIM * npolicy / (ms * 1e-3),
            "tflops": FLOPS_PER_ENV_STEP * n * DECIM * npolicy / (ms * 1e-3) / 1e12, "mapping": mapping,
            "block": block}


def _cfg():
    from g1sim_b200 import _lib
    return _lib.default_config(dt=DT)


def refinement_bench(sur, device, n=4096, H=50, iters=10):
    """Short-horizon refinement of the targets a policy chose for standing
    envs (the drop test's stand + N(0, 0.1) targets, 200 substeps after the
    drop): J = sum over H substeps of (z - 0.78)^2 + 0.1 |u - u0|^2 with u
    held, `iters` normalised gradient steps per env, each judged by the exact
    step.  Gradients from the surrogate rollout alone, from the surrogate
    with fallback to the exact adjoint where its one-step error exceeds 5e-2,
    and from the exact adjoint alone."""
    import torch
    from g1sim_b200 import surrogate as S
    from g1sim_b200 import workloads
    from g1sim_b200 import g1sim as G
    w = workloads.drop_test(nenv=n, seed=9)
    s = {k: torch.tensor(w[k], dtype=torch.float32, device=device) for k in ("qpos", "qvel", "anchor", "ctrl")}
    G.step(s["qpos"], s["qvel"], s["anchor"], s["ctrl"], 200, config=_cfg())
    u0 = s["ctrl"].clone()
    J0 = S.exact_objective(s, u0, H, u0=u0, reg=0.1)
    out = {"envs": n, "horizon_substeps": H, "iterations": iters, "objective_unrefined": float(J0.mean())}
    for name, mode, bound in (("surrogate", "surrogate", None), ("surrogate_with_fallback", "surrogate", 5e-2),
                              ("exact", "exact", None)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, J, frac = S.refine_targets(sur, s, u0, H=H, iters=iters, mode=mode, bound=bound)
        torch.cuda.synchronize()
        out[name] = {"objective": float(J.mean()), "envs_improved": float((J < J0).float().mean()),
                     "seconds": time.perf_counter() - t0}
        if mode == "surrogate":
            out[name]["fraction_on_surrogate_gradient"] = frac
            out[name]["bound"] = bound
    return out


def gemm_bench(device, rows, steps, warmup):
    """The surrogate's layer products alone, rows x 512 x 512, each timed over
    `steps` calls with CUDA events: the plain product C = A W^T + b (FP32 C,
    g1b_gemm_bf16), the fused hidden layer of training (FP16 Z, BF16 H) and
    of inference (BF16 H only), the fused backward through SiLU (FP16 Z in;
    BF16 dZ, bias-gradient sums) and the weight gradient (K = rows split over
    tiles, atomic FP32 sums) from the row-major activations (MN-major tiles,
    the training step's form) and from transposed copies (K-major tiles).
    hbm_gbs: algorithmic bytes (operands read once, outputs written once) per
    call over its time."""
    import torch
    from g1sim_b200 import surrogate as S
    g = torch.Generator(device=device).manual_seed(0)
    bf = torch.bfloat16
    A_ = torch.randn(rows, 512, device=device, generator=g).to(bf)
    W = (torch.randn(512, 512, device=device, generator=g) / 512 ** 0.5).to(bf)
    b = torch.randn(512, device=device, generator=g)
    C_ = torch.empty(rows, 512, device=device)
    Z = torch.randn(rows, 512, device=device, generator=g).half()  # FP16 pre-activation
    H = torch.empty(rows, 512, dtype=bf, device=device)
    Ht = torch.empty(512, rows, dtype=bf, device=device)
    At = torch.randn(512, rows, device=device, generator=g).to(bf)
    db = torch.zeros(512, device=device)
    Cw = torch.empty(512, 512, device=device)
    splits = max(1, min(64, rows // 2048))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(max(1, warmup)):
            fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(max(1, steps)):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / max(1, steps)

    flops = 2.0 * rows * 512 * 512
    el = rows * 512
    cases = [("store", lambda: S.gemm(A_, W, C_, bias=b), el * (2 + 4)),
             ("silu_forward_training", lambda: S.linear_silu(A_, W, b, H, Z=Z), el * (2 + 2 + 2)),
             ("silu_forward_inference", lambda: S.linear_silu(A_, W, b, H), el * (2 + 2)),
             ("silu_backward", lambda: S.linear_silu_bwd(A_, W, Z, H, db=db), el * (2 + 2 + 2)),
             # the training step's form: MN-major tiles of the row-major activations
             ("weight_gradient", lambda: (Cw.zero_(), S.gemm_atb(A_, H, Cw)), el * (2 + 2)),
             # the same product from transposed copies (K-major tiles)
             ("weight_gradient_k_major", lambda: S.gemm(At, Ht, Cw, splits=splits), el * (2 + 2))]
    modes = {}
    for name, fn, nbytes in cases:
        ms = timed(fn)
        modes[name] = {"us_per_call": ms * 1e3, "tflops": flops / (ms * 1e-3) / 1e12,
                       "hbm_gbs": nbytes / (ms * 1e-3) / 1e9, "algorithmic_bytes": nbytes}
    return {"shape": [rows, 512, 512], "us_per_call": modes["store"]["us_per_call"],
            "tflops": modes["store"]["tflops"], "modes": modes, "weight_gradient_splits": splits,
            "status": S.gemm_status()}


def surtrain_bench(device, batch, steps, warmup):
    """One surrogate training step alone (forward, loss, backward, Adam) on a
    fixed synthetic minibatch of `batch` rows (normal BF16 features and
    targets), replayed from its CUDA graph `steps` times after `warmup`
    replays, timed with CUDA events."""
    import torch
    from g1sim_b200 import surrogate as S
    sur = S.Surrogate(device, seed=0)
    g = torch.Generator(device=device).manual_seed(0)
    xb = torch.randn(batch, S.NIN, device=device, generator=g).to(torch.bfloat16)
    tb = torch.randn(batch, 64, device=device, generator=g)
    tg = sur.capture_train_step(xb, tb, lr=1e-3)
    for _ in range(max(1, warmup)):
        tg.step()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(max(1, steps)):
        tg.step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(1, steps)
    return {"batch": batch, "train_step_ms": ms, "tflops": S.train_flops(batch) / (ms * 1e-3) / 1e12,
            "loss": float(tg.loss.item()), "status": S.gemm_status()}


def part_only(args, local):
    """One sub-benchmark alone on one GPU, printed as a diagnostic JSON line
    (not the bench line): the small cases the profiler captures run this way."""
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    stream = torch.cuda.Stream(device)
    if args.part == "plain":
        r = plain_bench(device, args.nenv, args.steps, args.warmup, args.npolicy)
    elif args.part == "policy":
        from g1sim_b200 import workloads
        w = workloads.randomized(nenv=args.nenv, seed=0)
        init = {k: torch.tensor(w[k], dtype=torch.float32, device=device)
                for k in ("qpos", "qvel", "anchor", "ctrl", "mu", "dmass")}
        r = policy_fused_bench(args.nenv, 0, device, stream, args.steps, args.warmup, 1, local, init)
    elif args.part == "ppo":
        r = policy_ppo_bench(device)
    elif args.part == "surrogate":
        r = surrogate_bench(device, args.surrogate_steps, 1)
    elif args.part == "surtrain":
        r = surtrain_bench(device, args.nenv, args.steps, args.warmup)
    elif args.part == "adjoint":
        r = adjoint_bench(device, stream, args.steps, args.warmup, 1, n=args.nenv, horizon=args.horizon)
    else:
        r = gemm_bench(device, args.nenv, args.steps, args.warmup)
    print(json.dumps({"part": args.part, "envs_or_rows": args.nenv, **r}))
    return 0


# ------------------------------------------------------------- our arm
def ours(args, world, rank, local):
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)

    from g1sim_b200 import _lib, workloads
    from g1sim_b200 import g1sim as G
    L = _lib.lib()

    n = args.nenv
    w = workloads.randomized(nenv=n, seed=rank)
    f32 = dict(dtype=torch.float32, device=device)
    init = {k: torch.tensor(w[k], **f32) for k in ("qpos", "qvel", "anchor", "ctrl", "mu", "dmass")}
    st = {k: init[k].clone() for k in ("qpos", "qvel", "anchor", "ctrl")}
    rc = torch.zeros(n, dtype=torch.int32, device=device)
    cfg = _lib.default_config(dt=DT)
    npolicy = SUBSTEPS // DECIM
    stream = torch.cuda.Stream(device)

    def launch_policy_steps(k0, count, counter):
        G.rollout(st["qpos"], st["qvel"], st["anchor"], st["ctrl"], count, DECIM, config=cfg, seed=rank,
                  step0=k0, mu=init["mu"], dmass=init["dmass"], reset_count=counter)

    def reset_state():
        for k in st:
            st[k].copy_(init[k])

    # the step: one persistent launch of the 100 policy steps (each CTA keeps its envs on chip
    # across all of them), captured in a CUDA graph; beside it the same work as a graph of 100
    # one-policy-step launches (the state goes back to memory between policy steps)
    rc_split = torch.zeros_like(rc)
    with torch.cuda.stream(stream):
        reset_state()
        launch_policy_steps(0, 1, rc_split)  # one eager launch before capture (kernel attributes, lazy loading)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            launch_policy_steps(0, npolicy, rc)
        graph_split = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph_split, stream=stream):
            for k in range(npolicy):
                launch_policy_steps(k, 1, rc_split)
    launches_per_step = 1

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)  # > 126 MB L2

    def timed_steps(count, g):
        times = []
        for _ in range(count):
            with torch.cuda.stream(stream):
                reset_state()
                flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                g.replay()
                e1.record(stream)
            stream.synchronize()
            times.append(e0.elapsed_time(e1))
        return times

    timed_steps(args.warmup, graph)
    barrier(world)
    torch.cuda.synchronize()
    rc0 = int(rc.sum().item())
    with ClockSampler(local) as clk:
        times = timed_steps(args.steps, graph)
    torch.cuda.synchronize()
    barrier(world)
    resets_per_step = (int(rc.sum().item()) - rc0) / max(args.steps, 1)
    accuracy = accuracy_plain(st, init["mu"], init["dmass"], device) if rank == 0 else None
    ms = max_over_ranks(statistics.mean(times), world, device)
    env_steps = float(n) * SUBSTEPS
    value = env_steps * world / (ms * 1e-3)
    # the same work as 100 one-policy-step launches (same warm-up and timing), reported alongside
    timed_steps(args.warmup, graph_split)
    ms_split = max_over_ranks(statistics.mean(timed_steps(args.steps, graph_split)), world, device)

    # ---- kernel-level roofline (dominant kernel: the persistent launch of 100 policy steps)
    launch_ms = ms / launches_per_step
    flops_launch = FLOPS_PER_ENV_STEP * n * SUBSTEPS
    achieved_tf = flops_launch / (launch_ms * 1e-3) / 1e12
    ffma_tf = C.c_float()
    ffma_ms = C.c_float()
    _lib.check(L.g1b_ffma_peak(20000, C.byref(ffma_tf), C.byref(ffma_ms)), "g1b_ffma_peak")
    peak_tf = float(ffma_tf.value)
    hbm_gbs = BYTES_PER_ENV_LAUNCH * n / (launch_ms * 1e-3) / 1e9
    mapping, block, _ = _lib.get_launch()
    kernel_name = {0: f"rollout_kernel<{block}> (1 thread per env)",
                   1: f"split_kernel<{block}, rollout> (2 threads per env)",
                   2: f"split3_kernel<{block}, rollout> (3 threads per env)"}.get(mapping, "?") + \
        f", {npolicy} policy steps per launch"

    # ---- end to end through the public API, host buffers in pinned memory
    host_in = {k: init[k].cpu().pin_memory() for k in init}
    host_out = {k: torch.empty_like(host_in[k]).pin_memory() for k in ("qpos", "qvel", "anchor", "ctrl")}
    dev_in = {k: torch.empty_like(init[k]) for k in init}
    h2d = sum(t.numel() * 4 for t in host_in.values())
    d2h = sum(t.numel() * 4 for t in host_out.values())

    def e2e_step():
        with torch.cuda.stream(stream):
            for k in host_in:
                dev_in[k].copy_(host_in[k], non_blocking=True)
            G.rollout(dev_in["qpos"], dev_in["qvel"], dev_in["anchor"], dev_in["ctrl"], npolicy, DECIM, config=cfg,
                      seed=rank, step0=0, mu=dev_in["mu"], dmass=dev_in["dmass"])
            for k in host_out:
                host_out[k].copy_(dev_in[k], non_blocking=True)
        stream.synchronize()

    e2e_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps, world, device)
    e2e_value = env_steps * world / e2e_s

    finite = bool(torch.isfinite(st["qpos"]).all().item())

    pol = policy_fused_bench(n, rank, device, stream, args.steps, args.warmup, world, local, init)
    ppo = policy_ppo_bench(device) if rank == 0 else None
    adj = adjoint_bench(device, stream, args.steps, args.warmup, world) if not args.no_adjoint else None
    sur = surrogate_bench(device, args.surrogate_steps, world) if args.surrogate_steps >= 0 else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference(args.cpu_seconds, n)
        fp64 = cpu_reference(args.cpu_seconds / 2, n, precision=8)
        if cpu is not None and fp64 is not None:
            cpu["fp64_host"] = {"value": fp64["value"], "unit": fp64["unit"], "cores": fp64["cores"],
                                "sample": fp64["sample"]}

    if rank == 0:
        line = {
            "metric": "env-steps/s", "value": value, "unit": "env-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"randomised plain step, {n} envs per GPU, dt 2 ms, decimation 10, "
                                   f"{SUBSTEPS} substeps per step (one persistent launch of {npolicy} policy steps, "
                                   f"in a CUDA graph)",
                       "envs_per_gpu": n, "substeps": SUBSTEPS, "decimation": DECIM, "dt": DT,
                       "parallelism": f"replicas x{world}", "l2": "flushed (256 MB write) between timed steps"},
            "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                         "frac": achieved_tf / peak_tf if peak_tf > 0 else None,
                         "traffic": NCU_DRAM_BYTES_PER_ENV_PERSISTENT * n,
                         "traffic_source": f"ncu DRAM bytes of one split_kernel launch of {npolicy} policy steps at "
                                           f"16,384 envs, scaled by envs",
                         "algorithmic_bytes": BYTES_PER_ENV_LAUNCH * n,
                         "peak_source": "measured FFMA microbenchmark (g1b_ffma_peak), this run",
                         "flops_per_env_step": FLOPS_PER_ENV_STEP,
                         "achieved_as_written": achieved_tf * FLOPS_PER_ENV_STEP_AS_WRITTEN / FLOPS_PER_ENV_STEP,
                         "flops_per_env_step_as_written": FLOPS_PER_ENV_STEP_AS_WRITTEN,
                         "achieved_executed": achieved_tf * FLOPS_EXECUTED_PER_ENV_STEP / FLOPS_PER_ENV_STEP,
                         "flops_per_env_step_executed": FLOPS_EXECUTED_PER_ENV_STEP, "kernel": kernel_name,
                         "kernel_ms": launch_ms, "hbm_gbs": hbm_gbs},
            "e2e": {"value": e2e_value, "unit": "env-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary(),
            "per_policy_step_launches": {"value": env_steps * world / (ms_split * 1e-3), "ms": ms_split,
                                         "form": f"CUDA graph of {npolicy} one-policy-step launches"},
            "resets_per_timed_step": resets_per_step, "finite": finite, "accuracy": accuracy,
            "policy_fused": pol,
            "policy_ppo": ppo,
        }
        if adj is not None:
            line["adjoint"] = adj
        if sur is not None:
            line["surrogate"] = sur
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        del graph
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        return reference_arm(args, world, rank)
    if args.part != "all":
        return part_only(args, local)
    return ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
