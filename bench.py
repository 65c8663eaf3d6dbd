#!/usr/bin/env python
"""Benchmark of the FP64 uniform-patch D-Claw step on B200.

Workload (default): the 4096 x 4096 random-field case -- dx 0.5 m, seeded
Gaussian random terrain (spectral slope -3, 5 m RMS) on a 20 deg tilt, 32
seeded paraboloid sources (~70% of cells dry), reference material
parameters, order 2 + transverse corrections + MC limiter, wall boundaries.
Synthetic data generated here from a seed.

A "step" is one full patch step (ghost fill, b4step2, step2 sweeps, update,
src2, Courant number, next dt). Metric: cell-updates/s (interior cells x
steps / time). `value` is measured with CUDA events on the launching stream
with the state resident in HBM (the 672 MB state is larger than L2, so no
flush is needed); `e2e` goes through the public patch-step API with host
buffers: each step copies the state from pinned host memory to the device,
runs the step and copies the new state and the Courant number back.

--impl reference times the CPU restatement of the reference Fortran
(oracle/, OpenMP over all host cores) on the same workload, one full step
per timed step.

Multi-GPU (torchrun): every rank advances its own patch (independent
replicas, weak scaling); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

BYTES_PER_CELL_UPDATE = 88  # read 5 state + 1 bed, write 5 state (FP64)
# One step over tile lists as ncu counts it (one launch of each kernel, after
# the warm-up steps): DRAM bytes read + written and warp instructions issued
# (smsp__inst_executed.sum), on the workload the numbers are quoted for
NCU_STEP = {
    "cells": 4096 * 4096,
    "command": "ncu --metrics gpu__time_duration.sum,smsp__inst_executed.sum,dram__bytes_read.sum,"
               "dram__bytes_write.sum --clock-control none -k regex:k_ python bench.py --size 4096 --steps 3 "
               "--warmup 3 --e2e-steps 0 --no-cpu-baseline --ensemble-members 0 --grad-steps 0 "
               "--bgrad-members 0 --full-steps 0 --variant-steps 0",
    "kernels": {  # name: (DRAM bytes, warp instructions) per launch, the mean of the 6 launches
        "k_scan_patch": (1295.4e6, 56.82e6),
        "k_list_patch": (0.4e6, 0.59e6),
        "k_records_list": (839.8e6, 276.57e6),
        "k_tile_list": (754.6e6, 1410.10e6),
        "k_src2_list": (325.6e6, 372.82e6),
    },
    # k_tile_list, --set full on the 2048^2 case: active lanes per warp
    # instruction, FP64 pipe active
    "k_tile_list_lanes": 20.74,
    "k_tile_list_fp64_pipe": 0.303,
}
SMS, SCHEDULERS_PER_SM = 148, 4
METRIC = "cell-updates/sec on 1 B200 (plain vs batched); gradient/forward time ratio"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--dx", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-steps", type=int, default=0,
                    help="timed oracle steps of the CPU baseline (0: --steps, the reference arm's sample)")
    ap.add_argument("--cpu-band-rows", type=int, default=256,
                    help="rows of the one-thread CPU sample (one step)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--json-out", default="")
    ap.add_argument("--ensemble-members", type=int, default=256,
                    help="members of the batched flume ensemble measured beside the plain step (0: skip)")
    ap.add_argument("--ensemble-steps", type=int, default=2000,
                    help="steps of the batched ensemble run (the case is defined over 2000)")
    ap.add_argument("--ensemble-window", type=int, default=10,
                    help="steps of the batched-vs-looped comparison windows (early and late in the run)")
    ap.add_argument("--grad-steps", type=int, default=500,
                    help="steps of the 512 x 512 gradient case measured beside the plain step (0: skip)")
    ap.add_argument("--checkpoint-block", type=int, default=0,
                    help="0: the smallest block whose checkpoints fit half of the free device memory")
    ap.add_argument("--bgrad-members", type=int, default=64,
                    help="members of the batched-gradient channel case (0: skip)")
    ap.add_argument("--bgrad-steps", type=int, default=800,
                    help="steps of the batched-gradient case (the case is defined over 800)")
    ap.add_argument("--full-steps", type=int, default=200,
                    help="steps of the whole-run leg of the plain case from its initial state "
                         "(the case is defined over 200; 0: skip)")
    ap.add_argument("--variant-steps", type=int, default=10,
                    help="timed steps of each option variant of the plain case (src2method 2, Manning, order 1, "
                         "the full state with segregation and entrainment); 0: skip")
    ap.add_argument("--slab-steps", type=int, default=0,
                    help="also step ONE patch of the case split into row slabs over the N ranks "
                         "(strong scaling; halo exchange + Courant max per step); 0: skip")
    ap.add_argument("--slab-count", type=int, default=8, help="slabs of the one-GPU slab measurement")
    ap.add_argument("--only", default="", choices=["", "batched", "gradient", "batched_gradient"],
                    help="run one side measurement alone and print its object (profiling runs)")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_case(args, rank=0):
    from dclaw_b200 import workloads as W

    from dclaw_b200.replicas import replica_seed

    return W.random_field_case(n=args.size, dx=args.dx, seed=replica_seed(args.seed, rank))


def workload_config(case, world=1):
    """The `config` object of both arms (the same keys and values)."""
    cells = case.mx * case.my
    return {"workload": f"random_field_{case.mx}x{case.my}_dx{case.dx}", "cells_per_gpu": cells,
            "parallelism": f"replicas{world}",
            "l2": f"state {40 * cells / 1e6:.0f} MB {'>' if 40 * cells > 126e6 else '<'} L2 (126 MB), no flush",
            "order": case.params.order, "transverse_waves": case.params.transverse_waves, "limiter": "MC"}


def oracle_sample(case, warmup, steps):
    """The CPU sample both arms time: the oracle (the CPU restatement of the
    reference Fortran, OpenMP over all host cores) advances the case by
    `warmup` untimed steps from its initial state, then `steps` timed full
    steps from there. Returns (cell-updates/s, seconds, cores, status)."""
    from oracle import Oracle

    o = Oracle()
    cores = o.threads(os.cpu_count() or 1)
    q, dt = case.q, case.dt_initial
    if warmup:
        r = o.run(case.params, case.q, case.b, case.dx, case.dy, warmup, case.dt_initial, parallel=True)
        # the timed steps continue from the warm-up state, starting at the
        # warm-up's last dt
        q, dt = r["q"], float(r["dt"][-1])
    t0 = time.perf_counter()
    r2 = o.run(case.params, q, case.b, case.dx, case.dy, steps, dt, parallel=True)
    el = time.perf_counter() - t0
    return case.mx * case.my * steps / el, el, cores, r2["status"]


def oracle_sample_text(case, warmup, steps, el):
    return (f"steps {warmup + 1}..{warmup + steps} of the {case.mx}x{case.my} workload ({warmup} untimed warm-up "
            f"steps from its initial state, then {steps} timed full steps, {el:.1f} s; oracle/dclaw_oracle.cpp, "
            f"OpenMP)")


def cpu_baseline(args, case, warmup, steps):
    """The reference arm's sample (oracle_sample) timed on this box, and a
    one-thread figure on a band of rows of the same field beside it."""
    import numpy as np

    from oracle import Oracle

    v, el, cores, status = oracle_sample(case, warmup, steps)
    out = {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port",
           "sample": oracle_sample_text(case, warmup, steps, el), "status": status}
    o = Oracle()
    band = min(case.my, max(1, args.cpu_band_rows))
    qb, bb = np.ascontiguousarray(case.q[:, :band, :]), np.ascontiguousarray(case.b[:band, :])
    timing = {}
    for n in (1, cores):
        o.threads(n)
        t0 = time.perf_counter()
        o.run(case.params, qb, bb, case.dx, case.dy, 1, case.dt_initial, parallel=True)
        timing[n] = time.perf_counter() - t0
    o.threads(cores)
    out["one_thread"] = {"value": case.mx * band / timing[1], "unit": "cell-updates/s", "cores": 1,
                         "all_threads_same_sample": case.mx * band / timing[cores],
                         "sample": f"1 step of rows 1..{band} of the same field ({case.mx}x{band}, walls at the "
                                   f"band's edges; {timing[1]:.1f} s on 1 thread, {timing[cores]:.2f} s on {cores})"}
    return out


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    case = make_case(args)
    v, el, cores, status = oracle_sample(case, args.warmup, args.steps)
    line = {"metric": METRIC, "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(case, args.gpus),
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                             "sample": oracle_sample_text(case, args.warmup, args.steps, el)},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "status": status}
    print(json.dumps(line), flush=True)


def ensemble_bench(args, dev):
    """Batched flume ensemble (uneven channels, per-member parameters and dt)
    over its whole run (--ensemble-steps, 2000 by default, from the initial
    state), replayed from one captured CUDA graph of the persistent ensemble
    kernels after autotuning. Beside it, two windows of --ensemble-window
    steps -- the first steps of the run and the last ones, where the flows
    have spread -- are also run by looping the plain patch step over the
    members from the same states and clocks (eagerly, and captured into one
    CUDA graph of all its launches)."""
    import torch

    from dclaw_b200 import workloads as W
    from dclaw_b200.ensemble import EnsembleStepper, Member
    from dclaw_b200.params import CLOCK_DOUBLES
    from dclaw_b200.solver import PatchStepper

    K = max(2, args.ensemble_window + args.ensemble_window % 2)
    nrep = max(2, -(-args.ensemble_steps // K))
    N = nrep * K
    cases = W.flume_ensemble(n=args.ensemble_members, seed=args.seed)
    members = [Member(c.q, c.b, c.params, c.dx, c.dy, c.dt_initial) for c in cases]
    cells = sum(c.mx * c.my for c in cases)
    ens = EnsembleStepper(members, dev)
    tune = ens.autotune(steps=2)      # leaves the state and clocks at the start
    ens.capture(K)
    torch.cuda.synchronize()

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def snapshot():
        return ([ens.state(k).clone() for k in range(ens.n)], ens.clocks.view(ens.n, CLOCK_DOUBLES).clone())

    snap_early = snapshot()
    ms_early = timed(lambda: ens.replay(1))
    ms_mid = timed(lambda: ens.replay(nrep - 2))
    snap_late = snapshot()
    ms_late = timed(lambda: ens.replay(1))
    status_b = ens.status()
    ms_run = ms_early + ms_mid + ms_late
    beds = [torch.from_numpy(m.b).to(dev) for m in members]
    del ens
    torch.cuda.empty_cache()

    def looped(snap):
        states, clocks = snap
        steppers = []
        for k, m in enumerate(members):
            ps = PatchStepper(states[k], beds[k], m.params, m.dx, m.dy)
            ps.clock.copy_(clocks[k])
            steppers.append(ps)

        def reset():
            for k, ps in enumerate(steppers):
                ps.qa.copy_(states[k])
                ps.clock.copy_(clocks[k])

        def loop_eager():
            for _ in range(K):
                for ps in steppers:
                    ps.step(1)

        ms_le = timed(loop_eager)
        reset()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                for _ in range(K // 2):
                    for ps in steppers:
                        ps._launch(ps.qa, ps.qb)
                    for ps in steppers:
                        ps._launch(ps.qb, ps.qa)
        torch.cuda.current_stream().wait_stream(s)
        reset()
        ms_lg = timed(g.replay)
        del g, steppers
        torch.cuda.empty_cache()
        return ms_le, ms_lg

    def window(first, ms_b, snap):
        ms_le, ms_lg = looped(snap)
        return {"steps": [first + 1, first + K], "batched_ms_per_step": ms_b / K,
                "batched_value": cells * K / (ms_b / 1000.0),
                "looped_eager_ms_per_step": ms_le / K, "looped_graph_ms_per_step": ms_lg / K,
                "vs_looped_eager": ms_le / ms_b, "vs_looped_graph": ms_lg / ms_b}

    early = window(0, ms_early, snap_early)
    late = window(N - K, ms_late, snap_late)
    return {"workload": f"flume_ensemble_{len(members)}_dx0.05", "members": len(members), "cells": cells,
            "steps": N, "value": cells * N / (ms_run / 1000.0), "unit": "cell-updates/s", "ms_per_step": ms_run / N,
            "note": "the whole run from the initial state, one graph of the ensemble step replayed",
            "early_window": early, "late_window": late,
            "autotune": {k: tune[k] for k in ("tile_shape", "tile_ctas_per_sm", "ms")},
            "gpu_launches": 6 * N, "status_nonzero": sum(1 for x in status_b if x)}


def gradient_bench(args, dev):
    """Gradient of a gauge loss over a 500-step run of the 512 x 512 case
    with respect to (phi, kref, m0, alpha_c) and the initial depth of every
    cell, by the hand-written step adjoint with time checkpointing (every
    state kept when the run fits the memory budget),
    against the forward solve of the same run. Both are timed with CUDA
    events on the launching stream; the gradient's time covers its forward
    pass (with checkpoints), the loss and the whole backward pass."""
    import torch

    from dclaw_b200 import workloads as W
    from dclaw_b200.adjoint import checkpoint_block_of, initial_state, rollout_states, theta_of
    from dclaw_b200.solver import PatchStepper

    c = W.gradient_case(nsteps=args.grad_steps)
    p = c.params
    b = torch.tensor(c.b, device=dev)
    gj = torch.tensor(c.gauges[:, 0], device=dev)
    gi = torch.tensor(c.gauges[:, 1], device=dev)
    h0 = torch.tensor(c.h0, device=dev)
    blk = args.checkpoint_block or None

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        return e

    sel = gj * c.b.shape[1] + gi            # depth plane entries of the gauge cells

    used_k = []

    def gauges(h, m0, theta, block=blk):
        q0 = initial_state(h, m0, p)
        out = rollout_states(q0, theta, b, p, c.dx, c.dx, c.nsteps, c.out_steps, c.dt_initial,
                             checkpoint_block=block, select=sel)
        if out.grad_fn is not None:
            used_k.append(checkpoint_block_of(out))
        return out

    with torch.no_grad():
        target = gauges(h0, torch.tensor(c.m0, dtype=torch.float64, device=dev), theta_of(c.true_params, dev))
    # forward solve of the same run (plain fused steps)
    q0 = initial_state(h0, torch.tensor(c.m0, dtype=torch.float64, device=dev), p)
    fwd_ms = []
    for _ in range(2):
        st = PatchStepper(q0, b, p, c.dx, c.dx)
        st.init_clock(c.dt_initial)
        torch.cuda.synchronize()
        e0 = ev()
        st.step(c.nsteps)
        e1 = ev()
        torch.cuda.synchronize()
        fwd_ms.append(e0.elapsed_time(e1))
    del st
    grad_ms = []
    for _ in range(3):
        h = h0.clone().requires_grad_(True)
        m0 = torch.tensor(c.m0, dtype=torch.float64, device=dev, requires_grad=True)
        theta = theta_of(p, dev).requires_grad_(True)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats(dev)
        e0 = ev()
        loss = ((gauges(h, m0, theta) - target) ** 2).sum()
        loss.backward()
        e1 = ev()
        torch.cuda.synchronize()
        grad_ms.append(e0.elapsed_time(e1))
    f, g = min(fwd_ms), min(grad_ms)
    k = used_k[-1]
    # the same gradient with two-level sqrt(N) checkpoints (the memory
    # minimum: every block's states recomputed once in the backward pass)
    ksq = max(1, math.ceil(math.sqrt(c.nsteps)))
    sq_ms = []
    for _ in range(3):
        hs = h0.clone().requires_grad_(True)
        ms0 = torch.tensor(c.m0, dtype=torch.float64, device=dev, requires_grad=True)
        ths = theta_of(p, dev).requires_grad_(True)
        torch.cuda.synchronize()
        e0 = ev()
        ((gauges(hs, ms0, ths, ksq) - target) ** 2).sum().backward()
        e1 = ev()
        torch.cuda.synchronize()
        sq_ms.append(e0.elapsed_time(e1))
    same = bool(torch.equal(ths.grad, theta.grad) and torch.equal(hs.grad, h.grad))
    mx, my = c.b.shape[1], c.b.shape[0]
    return {"workload": f"gauge_loss_{mx}x{my}_dx{c.dx}_{c.nsteps}steps", "gauges": len(c.gauges),
            "output_times": len(c.out_steps), "checkpoint_block": k, "forward_ms": f, "gradient_ms": g,
            "gradient_over_forward": g / f, "loss": float(loss.detach()),
            "sqrt_n_checkpoints": {"checkpoint_block": ksq, "gradient_ms": min(sq_ms),
                                   "gradient_over_forward": min(sq_ms) / f, "same_gradient_bits": same},
            "grad": {"phi_deg": float(theta.grad[0]), "kref": float(theta.grad[1]), "m0": float(m0.grad),
                     "alpha_c": float(theta.grad[2]), "h0_l2": float(h.grad.norm())},
            "peak_mem_gb": torch.cuda.max_memory_allocated(dev) / 1e9,
            "gpu_launches": {"adjoint_per_step": 21, "recompute_per_step": 3, "forward_per_step": 3},
            "note": "dt of each step chosen by the tick rule in the forward pass and replayed, not differentiated"}


def batched_gradient_bench(args, dev):
    """Per-member gradients over an ensemble of uneven channels: each member's
    gauge loss (16 centreline gauges x 50 output times against a target run
    at its own perturbed parameters) differentiated with respect to its four
    material parameters, its solid fraction m0 and its release-block volume,
    by the batched step adjoint with sqrt(N) checkpointing. Timed against the
    batched forward solve of the same run; both with CUDA events. The
    unbatched reference times rollout_states gradients of the first two
    members one after the other."""
    import torch

    from dclaw_b200 import workloads as W
    from dclaw_b200.adjoint import (checkpoint_block_of, ensemble_rollout_states, initial_state, rollout_states,
                                    theta_of)
    from dclaw_b200.ensemble import EnsembleStepper, Member

    c = W.batched_gradient_case(n=args.bgrad_members, nsteps=args.bgrad_steps)
    n = len(c.members)
    members = [Member(m.q, m.b, m.params, m.dx, m.dy, m.dt_initial) for m in c.members]
    ens = EnsembleStepper(members, dev)
    total = ens.qa.numel()
    offs = [int(ens.cm[k].q_off) for k in range(n)]
    masks = [torch.tensor(mk, device=dev) for mk in c.block_masks]
    gidx = []
    for k, m in enumerate(c.members):
        mx = m.q.shape[2]
        gidx += [offs[k] + int(j) * mx + int(i) for j, i in c.gauges[k]]
    gidx = torch.tensor(gidx, device=dev)

    def arena(H, m0):
        pieces, pos = [], 0
        for k, m in enumerate(c.members):
            if offs[k] > pos:
                pieces.append(torch.zeros(offs[k] - pos, dtype=torch.float64, device=dev))
            qk = initial_state(H[k] * masks[k], m0[k], m.params)
            pieces.append(qk.reshape(-1))
            pos = offs[k] + qk.numel()
        if pos < total:
            pieces.append(torch.zeros(total - pos, dtype=torch.float64, device=dev))
        return torch.cat(pieces)

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        return e

    ones = torch.ones(n, dtype=torch.float64, device=dev)
    m0s = torch.tensor([m.params.m0 for m in c.members], dtype=torch.float64, device=dev)
    th_true = torch.stack([theta_of(p, dev) for p in c.true_params])
    with torch.no_grad():
        target = ensemble_rollout_states(arena(ones, m0s), th_true, members, c.nsteps, c.out_steps, select=gidx)
    # forward solve of the same run (batched fused steps)
    q0 = arena(ones, m0s).detach()
    fwd = []
    for _ in range(2):
        st = EnsembleStepper(members, dev)
        st.qa.copy_(q0)
        torch.cuda.synchronize()
        e0 = ev()
        st.step(c.nsteps)
        e1 = ev()
        torch.cuda.synchronize()
        fwd.append(e0.elapsed_time(e1))
        del st
    H = ones.clone().requires_grad_(True)
    m0 = m0s.clone().requires_grad_(True)
    theta = torch.stack([theta_of(m.params, dev) for m in c.members]).requires_grad_(True)
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats(dev)
    e0 = ev()
    out = ensemble_rollout_states(arena(H, m0), theta, members, c.nsteps, c.out_steps, select=gidx)
    loss = ((out - target) ** 2).sum()
    loss.backward()
    e1 = ev()
    torch.cuda.synchronize()
    grad_ms = e0.elapsed_time(e1)
    peak = torch.cuda.max_memory_allocated(dev) / 1e9
    # unbatched: the first two members' gradients, one patch at a time
    unb = 0.0
    for k in range(min(2, n)):
        m = c.members[k]
        b = torch.tensor(m.b, device=dev)
        tk = theta_of(m.params, dev).requires_grad_(True)
        qk = initial_state(masks[k].clone(), torch.tensor(m.params.m0, dtype=torch.float64, device=dev), m.params)
        selk = torch.tensor([int(j) * m.q.shape[2] + int(i) for j, i in c.gauges[k]], device=dev)
        tgt = target[:, k * 16:(k + 1) * 16]
        torch.cuda.synchronize()
        f0 = ev()
        ok = rollout_states(qk, tk, b, m.params, m.dx, m.dy, c.nsteps, c.out_steps, m.dt_initial, select=selk)
        ((ok - tgt) ** 2).sum().backward()
        f1 = ev()
        torch.cuda.synchronize()
        unb += f0.elapsed_time(f1)
    cells = sum(m.q.shape[1] * m.q.shape[2] for m in c.members)
    area = torch.tensor(c.block_area, dtype=torch.float64, device=dev)
    return {"workload": f"channels_{n}x1024_w128-256_dx0.05_{c.nsteps}steps", "members": n, "cells": cells,
            "steps": c.nsteps, "checkpoint_block": checkpoint_block_of(out), "forward_ms": min(fwd),
            "gradient_ms": grad_ms,
            "gradient_over_forward": grad_ms / min(fwd), "unbatched_first2_gradient_ms": unb,
            "batched_gradient_ms_per_member": grad_ms / n, "peak_mem_gb": peak,
            "grad_member0": {"phi_deg": float(theta.grad[0, 0]), "kref": float(theta.grad[0, 1]),
                             "alpha_c": float(theta.grad[0, 2]), "mu": float(theta.grad[0, 3]),
                             "m0": float(m0.grad[0]), "block_volume": float(H.grad[0] / area[0])},
            "gpu_launches": {"adjoint_per_step": 20, "recompute_per_step": 6, "forward_per_step": 6},
            "note": "every member's dt from its own tick rule, recorded and replayed, not differentiated"}


def variants_bench(args, dev, case, plain_ms):
    """The plain case's state under option variants of the step, each from
    the case's initial state: `warmup` untimed steps, then `--variant-steps`
    timed ones (CUDA events on the launching stream). The full-state variant
    steps the seven-field state (dclaw_step_full) with segregation (chi0 =
    0.5, beta_seg 0.3) and entrainment (ent_dclaw4, method 0) over an
    erodible layer of 0.5 m under every cell."""
    import torch

    from dclaw_b200 import workloads as W
    from dclaw_b200.solver import PatchStepper

    cells = case.mx * case.my
    b = torch.tensor(case.b, device=dev)
    out = {"steps": args.variant_steps, "warmup": args.warmup, "unit": "cell-updates/s",
           "plain_ms_per_step": plain_ms}
    runs = {"src2method2": (dict(src2method=2, alphamethod=1), False),
            "manning": (dict(friction_forcing=True, manning_coefficient=0.03), False),
            "order1_no_transverse": (dict(order=1, transverse_waves=0), False),
            "full_state_segregation_entrainment": (dict(segregation=1, beta_seg=0.3, entrainment=1,
                                                        entrainment_method=0), True)}
    for name, (kw, full) in runs.items():
        p = case.params.replace(**kw)
        if full:
            q = torch.tensor(W.full_state(case.q, p), device=dev)
            he = torch.full((case.my, case.mx), 0.5, dtype=torch.float64, device=dev)
            st = PatchStepper(q, b, p, case.dx, case.dy, h_e=he)
        else:
            st = PatchStepper(torch.tensor(case.q, device=dev), b, p, case.dx, case.dy)
        st.init_clock(case.dt_initial)
        st.step(args.warmup)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        st.step(args.variant_steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.variant_steps
        out[name] = {"ms_per_step": ms, "value": cells / (ms / 1000.0), "vs_plain_time": ms / plain_ms,
                     "launches_per_step": 7 if full else 5, "status": st.status()}
        del st
        torch.cuda.empty_cache()
    return out


def slab_bench(args, dev, rank, world, barrier):
    """ONE patch of the case (the same on every rank) split into row slabs
    over the ranks: halo exchange, own rows, Courant max, tick per step
    (strong scaling). On one rank, the patch as `--slab-count` slabs stepped
    one after another on the one GPU: the work the halos add."""
    import torch

    from dclaw_b200 import _lib
    from dclaw_b200.replicas import max_over_ranks
    from dclaw_b200.slabs import DistSlabs, LocalSlabs

    case = make_case(args, 0)
    q = torch.tensor(case.q, device=dev)
    b = torch.tensor(case.b, device=dev)
    if world > 1:
        sl = DistSlabs(q, b, case.params, case.dx, case.dy)
        nslab = world
    else:
        sl = LocalSlabs(q, b, case.params, case.dx, case.dy, args.slab_count)
        nslab = args.slab_count
    del q, b
    sl.init_clock(case.dt_initial)
    sl.step(args.warmup)
    barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sl.step(args.slab_steps)
    e1.record(stream)
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    cells = case.mx * case.my
    return {"workload": f"random_field_{case.mx}x{case.my}_dx{case.dx}", "slabs": nslab, "ranks": world,
            "halo_rows": _lib.load().dclaw_rows_granule(), "steps": args.slab_steps, "ms_per_step": ms / args.slab_steps,
            "value": cells * args.slab_steps / (ms / 1000.0), "unit": "cell-updates/s",
            "scaling": "strong" if world > 1 else "one GPU, slabs in turn",
            "gpu_launches_per_step_per_slab": 5}


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_info()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    from dclaw_b200.replicas import max_over_ranks
    from dclaw_b200.solver import PatchStepper

    case = make_case(args, rank)
    q = torch.tensor(case.q, device=dev)
    b = torch.tensor(case.b, device=dev)
    st = PatchStepper(q, b, case.params, case.dx, case.dy)
    st.init_clock(case.dt_initial)
    cells = case.mx * case.my

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up (also advances the flow past its first, mostly static, steps)
    st.step(args.warmup)
    barrier()
    sampler = ClockSampler(dev.index)
    sampler.start()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    st.step(args.steps)
    e1.record(stream)
    barrier()
    clocks = sampler.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    status = st.status()
    value = cells * args.steps * world / (ms / 1000.0)

    # ---- end to end through the public patch-step API with host buffers ----
    e2e_ms = e2e_serial_ms = None
    h2d = d2h = 0
    if args.e2e_steps > 0:
        qh = st.state().cpu().pin_memory()
        from dclaw_b200.params import CLOCK_DOUBLES

        cfl_h = torch.zeros(CLOCK_DOUBLES, dtype=torch.float64).pin_memory()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        # the host-buffer step: the state stays in pinned host memory and
        # every step uploads it, steps it and downloads the result, the
        # copies pipelined against the compute band by band
        st.step_host(qh)
        barrier()
        f0.record(stream)
        for _ in range(args.e2e_steps):
            st.step_host(qh)                             # host state in, new host state out
            cfl_h.copy_(st.clock, non_blocking=True)     # Courant number and next dt
        f1.record(stream)
        barrier()
        e2e_ms = max_over_ranks(f0.elapsed_time(f1), dev)
        # the same with whole-state copies around the device step, for comparison
        barrier()
        f0.record(stream)
        for _ in range(args.e2e_steps):
            st.qa.copy_(qh, non_blocking=True)
            st.step(1)
            qh.copy_(st.state(), non_blocking=True)
            cfl_h.copy_(st.clock, non_blocking=True)
        f1.record(stream)
        barrier()
        e2e_serial_ms = max_over_ranks(f0.elapsed_time(f1), dev)
        # a lower bound: the state's upload alone and its download alone,
        # whole-state copies with nothing else running; the step moves both,
        # so it cannot take less than the slower of the two
        qh2 = torch.empty_like(qh).pin_memory()
        one_way = {}
        for name, fn in (("h2d", lambda: st.qb.copy_(qh, non_blocking=True)),
                         ("d2h", lambda: qh2.copy_(st.qb, non_blocking=True))):
            fn()
            barrier()
            f0.record(stream)
            for _ in range(args.e2e_steps):
                fn()
            f1.record(stream)
            barrier()
            one_way[name] = max_over_ranks(f0.elapsed_time(f1), dev) / args.e2e_steps
        del qh2
        h2d = qh.numel() * 8
        d2h = qh.numel() * 8 + cfl_h.numel() * 8

    # ---- the case over its whole stated run, from its initial state ----
    full = None
    if args.full_steps > 0:
        fs = PatchStepper(torch.tensor(case.q, device=dev), b, case.params, case.dx, case.dy)
        fs.init_clock(case.dt_initial)
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        fs.step(args.full_steps)
        f1.record(stream)
        barrier()
        full_ms = max_over_ranks(f0.elapsed_time(f1), dev)
        full = {"steps": args.full_steps, "value": cells * args.full_steps * world / (full_ms / 1000.0),
                "unit": "cell-updates/s", "ms_per_step": full_ms / args.full_steps,
                "t_end": fs.read_clock().t, "wet_fraction_end": float((fs.state()[0] > 0).double().mean()),
                "status": fs.status(),
                "note": "steps 1..N of the case from its initial state (no warm-up steps on the state)"}
        del fs

    peak, peak_kind = load_peaks()
    step_s = ms / 1000.0 / args.steps
    achieved = BYTES_PER_CELL_UPDATE * cells / step_s / 1e9
    scale = cells / NCU_STEP["cells"]
    traffic = sum(v[0] for v in NCU_STEP["kernels"].values()) * scale
    # the issue ceiling: every scheduler issuing one warp instruction per
    # cycle at the SM clock sampled during the timed region
    inst = sum(v[1] for v in NCU_STEP["kernels"].values()) * scale
    sm_hz = (clocks.get("sm_mhz") or 1965.0) * 1e6
    issue_peak = SMS * SCHEDULERS_PER_SM * sm_hz
    lanes = NCU_STEP["k_tile_list_lanes"]
    issue = {"bound": "issue", "achieved": inst / step_s / 1e9, "peak": issue_peak / 1e9,
             "unit": "G warp-instructions/s", "frac": inst / step_s / issue_peak, "inst_per_step": inst,
             "peak_note": f"{SMS} SMs x {SCHEDULERS_PER_SM} schedulers x 1 warp instruction per cycle at the "
                          f"sampled SM clock",
             "lane_frac": inst * lanes / step_s / (32 * issue_peak),
             "lane_note": f"thread instructions (k_tile_list's {lanes:.2f} active lanes per warp instruction "
                          f"applied to the step) over 32 lanes per issue slot",
             "k_tile_list_fp64_pipe": NCU_STEP["k_tile_list_fp64_pipe"],
             "source": "smsp__inst_executed.sum per kernel from ncu at "
                       f"{int(NCU_STEP['cells'] ** 0.5)}^2, scaled by cells (x1 on that workload)"}
    out = None
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": workload_config(case, world),
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic,
                            "traffic_note": f"DRAM bytes read + written per step from ncu at "
                                            f"{int(NCU_STEP['cells'] ** 0.5)}^2, scaled by cells (x1 on that "
                                            f"workload)",
                            "algorithmic_bytes": BYTES_PER_CELL_UPDATE * cells,
                            "kernel": "the step over tile lists: k_scan_patch + k_list_patch + k_records_list + "
                                      "k_tile_list + k_src2_list (88 B/cell-update algorithmic)",
                            "peak_source": peak_kind},
               "issue_roofline": issue,
               "clocks": clocks, "gpu_launches": 5 * args.steps, "status": status}
        if full is not None:
            out["full_run"] = full
        if e2e_ms is not None:
            out["e2e"] = {"value": cells * args.e2e_steps * world / (e2e_ms / 1000.0), "unit": "cell-updates/s",
                          "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms / args.e2e_steps,
                          "api": "PatchStepper.step_host (dclaw_step_host): pinned host state in and out every "
                                 "step, copies pipelined by bands of tile rows",
                          "serial_copies_value": cells * args.e2e_steps * world / (e2e_serial_ms / 1000.0),
                          "serial_copies_note": "whole-state copy in, PatchStepper.step, whole-state copy out",
                          "copy_bound_ms_per_step": max(one_way.values()),
                          "h2d_alone_ms": one_way["h2d"], "d2h_alone_ms": one_way["d2h"],
                          "frac_of_copy_bound": max(one_way.values()) / (e2e_ms / args.e2e_steps),
                          "copy_bound_note": "the slower of the state's upload alone and its download alone "
                                             "(whole-state copies, nothing else running): a lower bound on a "
                                             "step that moves both"}
    if args.slab_steps > 0:
        sl = slab_bench(args, dev, rank, world, barrier)
        if rank == 0:
            out["one_patch_slabs"] = sl
    if world > 1:
        dist.barrier()
    if rank == 0 and world == 1 and args.variant_steps > 0:
        out["variants"] = variants_bench(args, dev, case, ms / args.steps)
    if rank == 0 and world == 1 and args.ensemble_members > 0:
        del st
        torch.cuda.empty_cache()
        out["batched"] = ensemble_bench(args, dev)
    if rank == 0 and world == 1 and args.grad_steps > 0:
        out["gradient"] = gradient_bench(args, dev)
    if rank == 0 and world == 1 and args.bgrad_members > 0 and args.bgrad_steps > 0:
        out["batched_gradient"] = batched_gradient_bench(args, dev)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, case, args.warmup, args.cpu_steps or args.steps)
    if rank == 0:
        print(json.dumps(out), flush=True)
        if args.json_out:
            Path(args.json_out).write_text(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


def run_only(args):
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    fn = {"batched": ensemble_bench, "gradient": gradient_bench, "batched_gradient": batched_gradient_bench}
    out = fn[args.only](args, dev)
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.only:
        run_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
