"""Benchmark: cells/s of one GCM chemistry call on the 69-species network, 1,048,576 cells per GPU.

Workload: the seeded synthetic 69-species C-H-N-O network (390 reactions, 48 photolysis branches) on a column grid of
64 log-P levels (1e-2 to 1e8 dyn cm^-2) x 16,384 columns, T a smooth 400-2200 K profile with +-100 K noise, upper-layer
J log-uniform in 1e-10..1e-3 s^-1 where P < 1e3. Four untimed 300 s calls from a solar-like start settle the gas; a
step is then the fifth 300 s call (x, T, P, dt, h, J resident in HBM), repeated on the same inputs. The inputs
(552 MB of x alone) exceed L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--cells B] [--impl ours|reference]
  python bench.py --derivative jvp|vjp [--directions D] [--frozen] [--cells B]   (the derivative calls)
  python bench.py --workload uneven [--network N] [--calls C]                    (a call loop with cold starts)
  python bench.py --workload mlp [--cells B]           (the surrogate network's forward and training step alone)

--impl reference times the CPU implementation of the same solve (the oracle, a C restatement of the reference's
kernels, on all host threads) on a bounded sample of the same cells; rank 0 alone runs it.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path
from typing import Any

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cells/s per GCM call (69-sp, 1M cells): FP64 Rodas3 vs mixed/learned @rtol 1e-3"
NETWORK = "chno69"
LEVELS = 64
SPINUP_CALLS = 4
DT = 300.0
# DRAM bytes of one call-kernel launch per cell: ncu's dram__bytes_read.sum + dram__bytes_write.sum of the timed call
# at 262,144 cells (411.78 MB), divided by its cells; a launch's traffic grows with its cells.
TRAFFIC_PER_CELL = 411.78e6 / 262144
HBM_GBS = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"] if (ROOT / "MEASURED_PEAKS.json").exists() else 6650.0


def parse() -> argparse.Namespace:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--cells", type=int, default=1 << 20, help="cells per GPU")
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--cpu-sample", type=int, default=262144, help="cells of the CPU baseline sample")
    p.add_argument("--ref-sample", type=int, default=32768,
                   help="cells of the reference arm's sample (its four spin-up calls run on the CPU too)")
    p.add_argument("--workload", choices=("column", "uneven", "mlp"), default="column",
                   help="uneven: 262,144 cells, half at night, a quarter cold starts, a loop of --calls calls; "
                        "mlp: the surrogate network's forward pass and training step on --cells rows")
    p.add_argument("--calls", type=int, default=100, help="calls of the uneven workload's loop")
    p.add_argument("--network", choices=("cho41", "chno69", "sncho91"), default=NETWORK,
                   help="the synthetic network (the metric is quoted on chno69)")
    p.add_argument("--dt", type=float, default=DT, help="the call's dt, s (300; the sulfur configuration uses 600)")
    p.add_argument("--derivative", choices=("jvp", "vjp"), default=None,
                   help="time the call with its tangent (jvp, --directions of them) or its adjoint (vjp) instead")
    p.add_argument("--directions", type=int, default=1, help="tangent directions of --derivative jvp")
    p.add_argument("--frozen", action="store_true", help="--derivative with adapt=False (the accepted steps held)")
    p.add_argument("--arms", default="fp64,learned,mixed",
                   help="comma list of fp64, learned (the surrogate's gated call), mixed (FP32 factors)")
    p.add_argument("--train-cells", type=int, default=1 << 20, help="cells of the surrogate's training pairs")
    p.add_argument("--train-calls", type=int, default=10,
                   help="chained calls of the training pairs (10 x 1,048,576 cells: the 10 M pairs of the surrogate's "
                        "configuration)")
    p.add_argument("--epochs", type=int, default=20, help="training epochs of the surrogate")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    return p.parse_args()


def inputs(net, cells: int, seed: int):
    from maxichem_b200 import synthetic

    return synthetic.workload(net, "column", cells, seed=seed)


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int) -> None:
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)  # fmt: skip
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([q.strip() for q in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = [r for r in self.rows if len(r) == 7]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = [n for k, n in enumerate(names) if any(r[3 + k].lower() == "active" for r in rows)]
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(rows[0][1]) if rows[0][1] else None,
                "reasons": reasons, "samples": len(rows)}  # fmt: skip


def run_reference(args) -> None:
    """The CPU implementation of the same solve on the host's cores, one bounded sample per step."""
    import oracle
    from maxichem_b200 import synthetic, tables

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    net = synthetic.network(NETWORK)
    tab = tables.build(net, True)
    ref = oracle.Oracle(tab)
    sample = min(args.ref_sample, args.cells)
    # the GPU arm's own cells (rank 0's seed, the full batch's column grid), the first `sample` of them (whole columns)
    w = inputs(net, args.cells, seed=1000)
    w.dt[:] = args.dt
    T, P, dt, J = w.T[:sample], w.P[:sample], w.dt[:sample], w.J[:sample]
    x, h = w.x[:sample], w.h[:sample]
    for _ in range(SPINUP_CALLS):
        r = ref.call(x, T, P, dt, h, J=J)
        x, h = r["x"], r["h"]
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ref.call(x, T, P, dt, h, J=J)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = sample / float(np.mean(times))
    cores = oracle.threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{NETWORK}: call {SPINUP_CALLS + 1} of {args.dt:g} s calls on a {LEVELS}-level "
                               "column grid",
                   "cells": sample, "species": tab.ns, "reactions": tab.nr,
                   "sample_of": f"the first {sample} of the GPU arm's {args.cells} cells (seed 1000, whole columns)"},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "port",
                         "sample": f"the first {sample} cells of the same call (its four spin-up calls also on the "
                                   f"CPU), all {cores} host threads (OpenMP)"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def launch_ranks(args) -> None:
    """--gpus N > 1 outside torchrun: start N ranks of this script under torch.distributed.run (one per GPU) and exit
    with their status; inside torchrun, the world size must be N. Fails clearly when fewer GPUs are visible."""
    from maxichem_b200 import replicas

    if replicas.under_launcher():
        world = int(os.environ["WORLD_SIZE"])
        if world != args.gpus:
            sys.exit(f"bench.py --gpus {args.gpus} runs under a launcher of {world} ranks: they must agree")
        return
    if args.gpus <= 1:
        return
    import torch

    visible = torch.cuda.device_count() if torch.cuda.is_available() else 0
    if visible < args.gpus:
        sys.exit(f"bench.py --gpus {args.gpus}: only {visible} CUDA devices are visible; one rank per GPU needs "
                 f"{args.gpus}")  # fmt: skip
    os.environ.setdefault("NCCL_DEBUG", "INFO")  # the ranks' NCCL init lines show the communicator's size
    os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    sys.exit(replicas.relaunch(args.gpus, str(Path(__file__).resolve()), sys.argv[1:]))


def main() -> None:
    args = parse()
    if args.gpus < 1:
        sys.exit(f"bench.py --gpus: at least 1 expected, got {args.gpus}")
    if args.impl == "reference":
        run_reference(args)
        return
    launch_ranks(args)
    if args.workload == "uneven":
        run_uneven(args)
        return
    if args.workload == "mlp":
        run_mlp(args)
        return
    if args.derivative:
        run_derivative(args)
        return
    run_call(args)


def timed_steps(fn, steps: int, warmup: int, stream, name: str | None = None) -> tuple[float, Any]:
    """W untimed calls, then K calls between CUDA events on the launching stream: ms per call and the last output.
    `name` marks the K calls as an NVTX range (ncu --nvtx --nvtx-include "<name>/" then profiles just them)."""
    import torch

    out = None
    for _ in range(warmup):
        out = fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if name:
        torch.cuda.nvtx.range_push(name)
    e0.record(stream)
    for _ in range(steps):
        out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    if name:
        torch.cuda.nvtx.range_pop()
    return e0.elapsed_time(e1) / steps, out


def accuracy(ref: dict, got: dict) -> dict:
    """Per-species relative error of `got`'s x against the plain FP64 call's (species above 1e-20), over the call."""
    import torch

    from maxichem_b200.surrogate import quantile

    big = ref["x"] > 1e-20
    rel = ((got["x"] - ref["x"]).abs() / ref["x"])[big]
    rel = torch.nan_to_num(rel, nan=float("inf"))
    return {"p50": quantile(rel, 0.5), "p99": quantile(rel, 0.99), "p999": quantile(rel, 0.999),
            "max": float(rel.max()), "share_above_rtol": float((rel > 1e-3).double().mean()),
            "done_all": bool(got["done"].bool().all())}  # fmt: skip


def train_surrogate(solver, args, dev) -> tuple[Any, dict]:
    """The learned part, trained on the GPU by the library's kernels on pairs from the plain solver (other cells than
    the timed ones: the uneven column workload, seeds 2000/3000), its gate calibrated on held-out pairs."""
    from maxichem_b200 import surrogate as sg

    t0 = time.perf_counter()
    train = sg.pairs(solver, args.train_cells, args.train_calls, seed=2000, cold_share=0.1, dt=args.dt)
    val = sg.pairs(solver, 131072, args.train_calls, seed=3000, cold_share=0.1, dt=args.dt)
    gen_s = time.perf_counter() - t0
    sur = sg.Surrogate(solver.ns, solver.nj, solver.tab.atoms, dev, seed=1)
    t0 = time.perf_counter()
    fit = sur.fit(train, epochs=args.epochs, batch=16384, lr=2e-3)
    torch_sync()
    fit_s = time.perf_counter() - t0
    cal = max((sg.calibrate(sur, val, target=1e-3, proj_max=pm) for pm in (1e-3, 1e-2, 1e-1)),
              key=lambda c: c["accept"])  # fmt: skip
    info = {"pairs": len(train), "held_out": len(val), "generate_s": round(gen_s, 2), "fit_s": round(fit_s, 2),
            "epochs": args.epochs, "final_loss": fit["loss"][-1], "adam_steps": fit["steps"], "calibration": cal,
            "network": f"{sur.kin} -> {sur.layers} x {sur.hidden} SiLU -> {sur.heads} heads x {sur.nt} (BF16)"}  # fmt: skip
    return sur, info


def torch_sync() -> None:
    import torch

    torch.cuda.synchronize()


def run_call(args) -> None:
    """The call on 1,048,576 cells of the settled column grid, by arm: "fp64" (the plain Rodas3 path), "learned" (the
    BF16 surrogate's gated call with the FP64 path solving what it rejects, and a 1/64 audit), "mixed" (FP32 factors
    with FP64 refinement). The headline value is the fastest arm whose call meets the bar against the FP64 arm's
    result on the same inputs (per-species error within rtol 1e-3 at the 99.9th percentile, every cell done)."""
    import torch
    import torch.distributed as dist

    from maxichem_b200 import abi, replicas, synthetic
    from maxichem_b200 import surrogate as sg
    from maxichem_b200.solver import CudaSolver, check_inputs

    rank, local, world = replicas.rank_from_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    arms = [a for a in args.arms.split(",") if a]
    net = synthetic.network(args.network)
    B = args.cells
    w = inputs(net, B, seed=replicas.seed(1000, rank))  # each rank its own batch of columns (weak scaling)
    w.dt[:] = args.dt
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)  # noqa: E731
    solver = CudaSolver(net, dev, photo=True)
    tab = solver.tab
    x, T, P, dt, h, J = t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), t(w.J)
    spin = []
    for _ in range(SPINUP_CALLS):
        t0 = time.perf_counter()
        x, h, _, steps = solver(x, T, P, dt, h, J=J)
        spin.append({"s": round(time.perf_counter() - t0, 3), "steps_mean": float(steps.mean())})
    check_inputs(dev, tab.ns, x, T, P, dt, h, 1e-3, 1e-25, 4000)
    lib = abi.library()
    stream = torch.cuda.current_stream(dev)
    kw = dict(rtol=1e-3, atol=1e-25, max_steps=4000, J=J)
    report: dict[str, Any] = {}
    runners: dict[str, Any] = {}
    gated = sur_info = mixed = None
    if "learned" in arms:
        sur, sur_info = train_surrogate(solver, args, dev)
        cal = sur_info["calibration"]
        gated = sg.GatedSolver(solver, sur, spread_max=cal["spread_max"], proj_max=cal["proj_max"], audit_every=64,
                               seed=7)  # fmt: skip
        runners["learned"] = lambda: gated.launch_raw(x, T, P, dt, h, **kw)  # noqa: E731
    if "mixed" in arms:
        mixed = CudaSolver(net, dev, photo=True, precision="mixed")
        runners["mixed"] = lambda: mixed.launch_raw(x, T, P, dt, h, **kw)  # noqa: E731
    tries = torch.zeros(3, dtype=torch.int64, device=dev)
    lib.mx_set_try_counter(solver._handle, tries.data_ptr())
    outs: dict[str, Any] = {}
    with Clocks(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        ms64, outs["fp64"] = timed_steps(lambda: solver.launch_raw(x, T, P, dt, h, **kw), args.steps, args.warmup,
                                         stream, "fp64")  # fmt: skip
        nt = tries.cpu().tolist()
        tries.zero_()
        report["fp64"] = {"ms_per_step": replicas.max_over_ranks(ms64, dev), "counts": solver.fallback,
                          "fresh_tries": nt[0] - nt[1], "retries": nt[1]}  # fmt: skip
        for arm, fn in runners.items():
            if gated is not None and arm == "learned":
                gated.stats.zero_()
            steps_arm = args.steps if arm != "mixed" else max(1, min(args.steps, 3))
            ms, outs[arm] = timed_steps(fn, steps_arm, min(args.warmup, 3), stream, arm)
            report[arm] = {"ms_per_step": replicas.max_over_ranks(ms, dev), "steps": steps_arm,
                           "accuracy_vs_fp64": accuracy(outs["fp64"], outs[arm])}  # fmt: skip
        if world > 1:
            dist.barrier()
    lib.mx_set_try_counter(solver._handle, None)
    if gated is not None:
        n_calls = args.steps + min(args.warmup, 3)
        c = gated.counts()
        report["learned"].update(
            {"accepted_share": c["accepted"] / (n_calls * B), "audit": gated.audit(), "surrogate": sur_info,
             "gate_counts_per_call": {k: v / n_calls for k, v in c.items()}, "counts": solver.fallback,
             "cpu_reads_per_call": 0})  # fmt: skip
    if mixed is not None:
        report["mixed"]["escalated_per_call"] = int(mixed.escalated.item()) / (report["mixed"]["steps"] + 3)
        report["mixed"]["counts"] = mixed.fallback
    # the library's launches in each arm's timed region: the FP64 call (call, recovery, counts); the learned call
    # (features, the network's layers per 65,536-row chunk, gate, audit, the list-mode call, recovery, counts); the
    # mixed call (mixed kernel, its hand-back list call, recovery, counts, escalation count)
    per_call = {"fp64": 3, "mixed": 5}
    if gated is not None:
        per_call["learned"] = 6 + (gated.sur.layers + 1) * -(-B // 65536)
    launches = {arm: per_call[arm] * report[arm].get("steps", args.steps) for arm in report}
    for arm in report:
        report[arm]["cells_per_s"] = replicas.throughput(B, world, report[arm]["ms_per_step"] * 1e-3)
        report[arm]["gpu_launches"] = launches[arm]
    bar = lambda r: ("accuracy_vs_fp64" not in r or  # noqa: E731
                     (r["accuracy_vs_fp64"]["p999"] <= 1e-3 and r["accuracy_vs_fp64"]["done_all"]))
    headline = max((a for a in report if bar(report[a])), key=lambda a: report[a]["cells_per_s"])
    ms = report[headline]["ms_per_step"]
    value = report[headline]["cells_per_s"]
    counts = replicas.sum_counts(solver.total).cpu().tolist()
    phases = phase_shares(solver, lib, x, T, P, dt, h, J, dev)
    steps_mean = float(outs["fp64"]["steps"].mean())
    # roofline: the FP64 call kernel, the dominant kernel of every arm (the learned arm's fallback is this kernel on
    # the cells the gate rejects): algorithmic FP64 work of its tries / the plain arm's time per call
    f = tab.flops
    fresh, retry = report["fp64"]["fresh_tries"], report["fp64"]["retries"]
    flop_step = (fresh * f["fresh_try"] + retry * f["retry"] + (args.steps + args.warmup) * B * f["rates"]) / (
        args.steps + args.warmup)
    peak = ctypes_probe(lib, local)
    achieved = flop_step / (report["fp64"]["ms_per_step"] * 1e-3) / 1e12
    io_bytes = B * (8 * (2 * tab.ns + tab.nj + 6) + 12)
    line = {
        "metric": METRIC if (args.network, args.dt) == (NETWORK, DT) else
                  f"cells/s per GCM call ({tab.ns}-sp, {B * world} cells, dt {args.dt:g} s): FP64 Rodas3",
        "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if headline == "fp64" else ("bf16+f64" if headline == "learned" else "f32+f64"),
        "data": "synthetic (seeded 69-species network and column grid; the VULCAN networks are absent)",
        "config": {"workload": f"{args.network}: call {SPINUP_CALLS + 1} of {args.dt:g} s calls on a {LEVELS}-level "
                               "column grid",
                   "headline_arm": headline, "arms": report,
                   "cells_per_gpu": B, "species": tab.ns, "reactions": tab.nr, "photolysis": tab.nj,
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (no flush)",
                   "accepted_steps_mean": steps_mean, "tries_per_cell": (fresh + retry) / (args.steps + args.warmup) / B,
                   "us_per_cell_call": ms * 1e3 / B,  # per GPU: the unit of the reference's timings (its README.md:201)
                   "counts": dict(zip(["queue", *abi_counts()], counts)), "spinup": spin, "layout": solver.info,
                   "phase_shares": phases},
        "roofline": {"bound": "fp64", "kernel": "call_kernel (the plain arm)", "achieved": achieved,
                     "peak": peak / 1e3, "unit": "TFLOP/s", "frac": achieved / (peak / 1e3) if peak else None,
                     "traffic": TRAFFIC_PER_CELL * B,
                     "traffic_source": "ncu DRAM bytes of the call kernel at 262,144 cells, scaled by cells",
                     "algorithmic_bytes": io_bytes, "hbm_gbs": io_bytes / (report["fp64"]["ms_per_step"] * 1e-3) / 1e9,
                     "hbm_frac_of_measured": io_bytes / (report["fp64"]["ms_per_step"] * 1e-3) / 1e9 / HBM_GBS,
                     "peak_source": "measured in-process: FP64 fma chains on every SM (mx_probe_fp64)",
                     "flops_per_step": flop_step},
        "gpu_launches": sum(launches.values()),
        "clocks": clocks.summary(),
    }  # fmt: skip
    if gated is not None:
        line["roofline_mlp"] = mlp_roofline(gated.sur, x, T, P, dt, h, J, stream)
    if not args.no_e2e:
        if headline == "learned":
            line["e2e"] = e2e_gated(gated, x, h, w, dev, args)
        else:
            line["e2e"] = e2e(solver, x, h, w, dev, args)
        line["e2e"]["ms_per_step"] = replicas.max_over_ranks(line["e2e"]["ms_per_step"], dev)
        line["e2e"]["value"] = replicas.throughput(B, world, line["e2e"]["ms_per_step"] * 1e-3)
        line["e2e"]["arm"] = headline
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(tab, x, h, w, args)
    if gated is not None:
        gated.sur.close()
    if mixed is not None:
        mixed.close()
    solver.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def mlp_roofline(sur, x, T, P, dt, h, J, stream) -> dict:
    """The surrogate network's forward pass on the timed cells: its tcgen05 GEMMs' FLOPs over their time, against the
    measured sustained BF16 peak."""
    import torch

    feat, _ = sur.features(x, T, P, dt, h, J)
    ms, _ = timed_steps(lambda: sur.forward(feat), 5, 2, stream)
    flop = 2.0 * feat.shape[0] * useful_macs(sur)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak, sustained = peaks.get("bf16_tflops", 1590.0), peaks.get("bf16_tflops_sustained", 1400.0)
    torch.cuda.synchronize()
    return {"bound": "tensor", "kernel": "gemm_kernel (the network's 5 layers)", "achieved": flop / ms / 1e9,
            "peak": peak, "unit": "TFLOP/s", "frac": flop / ms / 1e9 / peak, "frac_of_sustained": flop / ms / 1e9 /
            sustained, "ms_per_forward": ms, "flops_per_forward": flop,
            "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst: the forward's launches timed alone)"}  # fmt: skip


def useful_macs(sur) -> int:
    """Multiply-adds per row of the network's forward pass on its real sizes: the features (not their padding to a
    multiple of 64) into the first layer, the heads' real outputs (not their padding to a 128- or 192-wide tile)."""
    sizes = [(r, c) for r, c in sur.shapes]
    sizes[0] = (sizes[0][0], sur.nf)
    sizes[-1] = (sur.heads * sur.nt, sizes[-1][1])
    return sum(r * c for r, c in sizes)


def run_mlp(args) -> None:
    """The surrogate network alone (69-species network's shapes: 4 x 512 SiLU layers, 4 heads, BF16 on the tcgen05
    GEMM): rows/s of its forward pass and of one training step (forward, Huber loss, backward, Adam) on --cells rows of
    seeded standard-normal features, weights at their seeded initial values. A step is one forward pass (K of them
    between CUDA events after W warm-up ones); the forward's activations (--cells x 512 x 2 bytes per layer) exceed L2
    from 131,072 rows up. The roofline is the GEMMs' FLOPs over the forward's time against the measured BF16 peak
    (burst: the forward's launches are timed back to back for well under a second)."""
    import torch

    from maxichem_b200 import surrogate as sg
    from maxichem_b200 import synthetic
    from maxichem_b200.solver import CudaSolver

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    net = synthetic.network(args.network)
    with CudaSolver(net, dev, photo=True) as solver:
        ns, nj, atoms = solver.ns, solver.nj, solver.tab.atoms
    rows = max(64, args.cells // 64 * 64)
    sur = sg.Surrogate(ns, nj, atoms, dev, seed=1)
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    feat = torch.randn(rows, sur.kin, device=dev, generator=g).to(torch.bfloat16)
    tgt = torch.randn(rows, sur.nt, device=dev, generator=g)
    wts = torch.ones(rows, sur.heads, device=dev)
    stream = torch.cuda.current_stream(dev)
    clock = Clocks(0)
    with clock:
        ms_fwd, _ = timed_steps(lambda: sur.forward(feat), args.steps, args.warmup, stream, "forward")
        ms_train, _ = timed_steps(lambda: sur.train_step(feat, tgt, wts, 1e-4, delta=1.0), args.steps, args.warmup,
                                  stream)  # fmt: skip
    sur.check()
    flop = 2.0 * rows * useful_macs(sur)  # the padding's multiply-adds are done but not counted
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("bf16_tflops", 1590.0)
    achieved = flop / ms_fwd / 1e9
    line = {"metric": f"rows/s of the surrogate's forward pass ({ns}-sp network's shapes, {rows} rows)",
            "value": rows / ms_fwd * 1e3, "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_fwd, "higher_is_better": True, "dtype": "bf16", "data": "synthetic (seeded features)",
            "config": {"workload": f"surrogate forward, {sur.kin} -> {sur.layers} x {sur.hidden} SiLU -> "
                                   f"{sur.heads} x {sur.nt} heads (padded to {sur.kout})", "rows": rows},
            "gpu_launches": (sur.layers + 1) * args.steps,
            "roofline": {"bound": "tensor", "kernel": "gemm_kernel", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "frac_of_sustained": achieved / peaks.get("bf16_tflops_sustained", 1400.0),
                         "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback 1590"},
            "train_step": {"ms": ms_train, "rows_per_s": rows / ms_train * 1e3,
                           "gemm_tflops": 3 * flop / ms_train / 1e9,
                           "note": "forward, loss, backward (6 more GEMMs, transposes, column sums), Adam"},
            "clocks": clock.summary()}  # fmt: skip
    sur.close()
    print(json.dumps(line), flush=True)


def run_derivative(args) -> None:
    """cells/s of the call with its tangent (ADSolver.jvp along --directions seeded directions of every input class)
    or its adjoint (ADSolver.vjp of seeded cotangents of x and h), on the settled column workload of the default line;
    the plain call is timed beside it on the same inputs."""
    import torch

    from maxichem_b200 import replicas, synthetic
    from maxichem_b200.ad import ADSolver

    rank, local, world = replicas.rank_from_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    net = synthetic.network(args.network)
    B = args.cells
    w = inputs(net, B, seed=replicas.seed(1000, rank))
    w.dt[:] = args.dt
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    solver = ADSolver(net, dev, photo=True)
    x, T, P, dt, h, J = t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), t(w.J)
    for _ in range(SPINUP_CALLS):
        x, h, _, _ = solver(x, T, P, dt, h, J=J)
    rng = np.random.default_rng(7)
    ns, nr, nj, D = solver.ns, solver.nr, solver.nj, args.directions
    adapt = not args.frozen
    if args.derivative == "jvp":
        xs = x.cpu().numpy()
        dx = xs * rng.standard_normal((D, B, ns))
        dx -= xs * dx.sum(2, keepdims=True)
        tan = [t(dx)] + [t(rng.standard_normal((D, B)) * s) for s in (w.T * 0.01, w.P, w.dt, h.cpu().numpy())]
        extra = dict(dlm=t(rng.standard_normal((D, B, nr))), dJ=t(w.J * rng.standard_normal((D, B, nj))))
        run = lambda: solver.jvp(x, T, P, dt, h, *tan, J=J, adapt=adapt, **extra)  # noqa: E731
    else:
        gx = t(rng.standard_normal((B, ns)) / np.maximum(x.cpu().numpy(), 1e-20))
        gh = t(rng.standard_normal(B)) if adapt else None
        run = lambda: solver.vjp(x, T, P, dt, h, gx, gh=gh, J=J, adapt=adapt)  # noqa: E731
    stream = torch.cuda.current_stream(dev)

    def timed(fn) -> float:
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    with Clocks(local) as clocks:
        ms = timed(run)
    flags = np.bincount(solver.flag.cpu().numpy(), minlength=3).tolist()
    ms_call = timed(lambda: solver.launch(x, T, P, dt, h, J=J))
    what = f"its tangent along {D} direction{'s' if D > 1 else ''}" if args.derivative == "jvp" else "its adjoint"
    line = {
        "metric": f"cells/s per GCM call with {what} ({solver.ns}-sp, {B * world} cells, dt {args.dt:g} s): FP64",
        "value": replicas.throughput(B, world, ms * 1e-3), "unit": "cells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded network and column grid)",
        "config": {"workload": f"{args.network}: call {SPINUP_CALLS + 1} of {args.dt:g} s calls on a {LEVELS}-level "
                               "column grid", "derivative": args.derivative,
                   "directions": D if args.derivative == "jvp" else None,
                   "contract": "adaptive" if adapt else "frozen", "cells_per_gpu": B, "flags": flags},
        "call_ms_per_step": ms_call, "cost_vs_call": ms / ms_call, "clocks": clocks.summary(),
    }  # fmt: skip
    solver.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_uneven(args) -> None:
    """Uneven batching: 262,144 cells of the column grid, the night half dark, settled by four 300 s calls, then a
    quarter turned into cold starts (h 1e-10 s, x perturbed log-normally); a loop of --calls 300 s calls, each from
    the previous call's x and h. Reports the per-call latency (p50, p99) of the loop run call by call with the
    autotuned mapping (2 or 4 warps per cell) and persistent grid and with one CTA per cell, and cells/s of the loop
    captured in one CUDA graph. --network picks the network (the configuration's is the 69-species one)."""
    import torch

    from maxichem_b200 import autotune, graph, synthetic
    from maxichem_b200.solver import CudaSolver

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    net = synthetic.network(args.network)
    B = min(args.cells, 262144)
    w = synthetic.workload(net, "uneven", B, seed=11)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    spin = CudaSolver(net, dev, photo=True)
    x, T, P, dt, h, J = t(w.x), t(w.T), t(w.P), t(w.dt), t(w.h), t(w.J)
    for _ in range(SPINUP_CALLS):
        x, h, _, _ = spin(x, T, P, dt, h, J=J)
    spin.close()
    xc, hc, cold = synthetic.cold_start(x.cpu().numpy(), h.cpu().numpy(), seed=12)
    x0, h0 = t(xc), t(hc)
    solver, tuned = autotune.tune(net, dev, x0, T, P, dt, h0, J=J)
    tuned["best"] = tuned["grid"]
    stream = torch.cuda.current_stream(dev)

    def loop(grid: int) -> dict:
        solver.set_grid(grid)
        xs, hs, times, out = x0, h0, [], None
        steps = None
        for k in range(args.calls):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = solver.launch_raw(xs, T, P, dt, hs, rtol=1e-3, atol=1e-25, max_steps=4000, J=J)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            if k == 0:
                steps = out["steps"].cpu().numpy()
            xs, hs = out["x"], out["h"]
        ms = np.array(times)
        return {"ctas_per_sm": grid, "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
                "first_call_ms": float(ms[0]), "cells_per_s": B * len(ms) / (ms.sum() * 1e-3),
                "first_call_steps": {"cold_mean": float(steps[cold].mean()), "warm_mean": float(steps[~cold].mean()),
                                     "max": float(steps.max()), "min": float(steps.min())}}  # fmt: skip

    persistent = loop(tuned["best"] if tuned["best"] > 0 else solver.info["call_ctas_per_sm"])
    static = loop(0)
    solver.set_grid(tuned["best"])
    cl = graph.CallLoop(solver, x0, T, P, dt, h0, J=J, calls=args.calls)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    last = cl.run(check=False)
    e1.record(stream)
    e1.synchronize()
    graph_ms = e0.elapsed_time(e1)
    done_all = bool(last["done"].bool().all())
    cl.close()
    line = {
        "metric": f"cells/s of a GCM call loop with uneven step counts ({solver.ns}-sp, {B} cells)", "unit": "cells/s",
        "workload": "uneven", "cells": B, "calls": args.calls, "cold_cells": int(cold.sum()),
        "autotune_ms": {f"{k[0]} warps, {k[1]} ctas/sm": v for k, v in tuned["ms"].items()},
        "autotune_best": {"warps_per_cell": tuned["warps"], "ctas_per_sm": tuned["grid"]},
        "persistent": persistent, "static_one_cta_per_cell": static,
        "graph": {"ms": graph_ms, "cells_per_s": B * args.calls / (graph_ms * 1e-3), "last_call_all_done": done_all},
        "data": "synthetic (seeded 69-species network, column grid, night half dark, quarter cold starts)",
    }  # fmt: skip
    solver.close()
    print(json.dumps(line), flush=True)


PHASES = ("rates", "rhs_jacobian", "lu", "stages12", "stage3", "stage4", "control", "output_guard")


def phase_shares(solver, lib, x, T, P, dt, h, J, dev) -> dict:
    """One untimed call through the call kernel's clock64-instrumented variant: the share of SM cycles per phase."""
    import torch

    cycles = torch.zeros(8, dtype=torch.int64, device=dev)
    lib.mx_set_phase_counter(solver._handle, cycles.data_ptr())
    solver.launch_raw(x, T, P, dt, h, rtol=1e-3, atol=1e-25, max_steps=4000, J=J)
    torch.cuda.synchronize(dev)
    lib.mx_set_phase_counter(solver._handle, None)
    c = cycles.cpu().double()
    return {k: round(float(v), 4) for k, v in zip(PHASES, (c / c.sum()).tolist())}


def abi_counts():
    from maxichem_b200.constants import COUNTS

    return [*COUNTS, "recovery_queue"]


def ctypes_probe(lib, device: int) -> float:
    import ctypes

    g = ctypes.c_double()
    lib.mx_probe_fp64(device, 20000, ctypes.byref(g))
    return g.value


def e2e(solver, x, h, w, dev, args) -> dict:
    """The same call through the public API from pinned host buffers (CudaSolver.call_host): H2D, the call with its
    count read-back, D2H, overlapped over four pieces of the batch."""
    import torch

    pin = lambda a: torch.as_tensor(a, dtype=torch.float64).pin_memory()
    hx, hT, hP, hdt, hh, hJ = (pin(a) for a in (x.cpu(), w.T, w.P, w.dt, h.cpu(), w.J))
    ox, oh, ost = (torch.empty_like(a).pin_memory() for a in (hx, hh, hh))
    odone = torch.empty(hh.shape, dtype=torch.bool).pin_memory()
    stream = torch.cuda.current_stream(dev)

    oflag, ostatus = (torch.empty(hh.shape, dtype=torch.int32).pin_memory() for _ in range(2))
    out = {"x": ox, "h": oh, "steps": ost, "done": odone, "flag": oflag, "status": ostatus}

    def step():  # the call on host buffers: copies in, kernels and copies out overlapped over pieces of the batch
        solver.call_host(hx, hT, hP, hdt, hh, J=hJ, out=out)

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    h2d = sum(a.numel() * a.element_size() for a in (hx, hT, hP, hdt, hh, hJ))
    d2h = sum(a.numel() * a.element_size() for a in (ox, oh, odone, ost, oflag, ostatus))
    return {"value": hx.shape[0] / (ms * 1e-3), "unit": "cells/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms}  # fmt: skip


def e2e_gated(gated, x, h, w, dev, args) -> dict:
    """The learned arm through its public API from pinned host buffers (GatedSolver.call_host): H2D of x, T, P, dt, h,
    J, the gated call with its refusal check, D2H of x, h, steps, done, flag, status."""
    import torch

    pin = lambda a: torch.as_tensor(a, dtype=torch.float64).pin_memory()  # noqa: E731
    hx, hT, hP, hdt, hh, hJ = (pin(a) for a in (x.cpu(), w.T, w.P, w.dt, h.cpu(), w.J))
    B = hx.shape[0]
    out = {"x": torch.empty_like(hx).pin_memory(), "h": torch.empty_like(hh).pin_memory(),
           "steps": torch.empty_like(hh).pin_memory(),
           **{k: torch.empty(B, dtype=torch.int32).pin_memory() for k in ("done", "flag", "status")}}  # fmt: skip
    stream = torch.cuda.current_stream(dev)
    ms, _ = timed_steps(lambda: gated.call_host(hx, hT, hP, hdt, hh, J=hJ, out=out), args.steps, max(1, args.warmup),
                        stream)  # fmt: skip
    h2d = sum(a.numel() * a.element_size() for a in (hx, hT, hP, hdt, hh, hJ))
    d2h = sum(a.numel() * a.element_size() for a in out.values())
    return {"value": B / (ms * 1e-3), "unit": "cells/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": ms}  # fmt: skip


def cpu_baseline(tab, x, h, w, args) -> dict:
    """The oracle on the host's cores on a bounded sample of the same call (the first cells of the batch)."""
    import oracle

    n = min(args.cpu_sample, x.shape[0])
    xs, hs = x[:n].cpu().numpy(), h[:n].cpu().numpy()
    ref = oracle.Oracle(tab)
    t0 = time.perf_counter()
    ref.call(xs, w.T[:n], w.P[:n], w.dt[:n], hs, J=w.J[:n])
    dt = time.perf_counter() - t0
    cores = oracle.threads()
    return {"value": n / dt, "unit": "cells/s", "cores": cores, "kind": "port",
            "sample": f"first {n} cells of the timed call, {dt:.1f} s on {cores} host threads"}  # fmt: skip


if __name__ == "__main__":
    main()
