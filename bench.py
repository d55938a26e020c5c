"""Benchmark of the REMC docking path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]
                    [--workload ensemble_4000x40]

Workload (default): the full replica ensemble of the plain form -- a 4,000
point protein with 11 conformations, a 40-atom ligand with 50 conformations,
16 temperatures (0.004..0.08), i.e. 8,800 replicas; move sizes 0.02 A /
0.08 rad; exchange every 20 MC steps.  One bench step is one exchange
interval: 20 MC steps of every replica followed by one temperature exchange.
Metric: replica-MC-steps/s (n_rep x MC steps / time; the reference's "MC
sweeps per second", util.C:1120-1123).

value     device time (CUDA events on the library's stream) of K steps with
          everything resident; L2 flushed (256 MiB write) before every step.
e2e       the same metric through gd_run (the Run() counterpart): every step
          uploads the complex from host memory, initialises, runs 20 MC steps
          + exchange and copies the results back.
roofline  the MC-interval kernel: 36 algorithmic FP32 flops per ligand-protein
          pair x pairs per launch / mean launch time (CUDA events), against the
          FP32 FMA peak measured live on this GPU.
cpu_baseline  the CPU oracle (C port of the reference kernels, OpenMP) on a
          bounded sample of the same workload on this host.

--impl reference times the reference's CPU path (the oracle port; the
reference's own code is CUDA-4/sm_20 only) on all host cores.
Multi-GPU: one process per GPU, each with its own independent 8,800-replica
ensemble (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOP_PER_PAIR = 36  # algorithmic FP32 flops per ligand-protein pair


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--workload", default="ensemble_4000x40")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        load = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def build_workload(name, seed):
    from gpudock_b200 import synth
    w = synth.WORKLOADS[name]
    cx = synth.make_complex(w.spec, seed=seed)
    _, mb = synth.temperatures(w)
    return w, cx, mb


def cpu_baseline(w, cx, mb, budget_s=15.0, native=True):
    """Times the CPU oracle (MC steps of a replica sample, OpenMP) on this host."""
    from gpudock_b200 import abi
    from oracle import oracle as orc
    params, _keep = abi.mc_params(w.steps, w.steps_per_exchange, mb, w.move_scale, seed=1)
    try:
        orc.build(native=native)
    except Exception:
        native = False
    threads = orc.max_threads(native)
    n_rep_total = cx.n_prt * cx.n_lig * w.n_tmp
    # calibrate with one step of `threads` replicas
    t0 = time.perf_counter()
    orc.mc_sample(cx, params, 0, threads, 1, threads, native)
    t1 = time.perf_counter() - t0
    per = max(t1, 1e-4)  # seconds for `threads` replica-steps
    n_steps = max(1, min(50, int(budget_s / per / 4)))
    n_rep = min(n_rep_total, threads * 4)
    t0 = time.perf_counter()
    done = orc.mc_sample(cx, params, 0, n_rep, n_steps, threads, native)
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "replica-MC-steps/s", "cores": threads,
            "kind": "port",
            "sample": f"{n_rep} of {n_rep_total} replicas x {n_steps} MC steps "
                      f"({done} energy evaluations, {dt:.1f} s, "
                      f"{'-march=native' if native else 'x86-64'} OpenMP build)"}


def run_reference(args):
    """--impl reference: the reference's CPU path (oracle port) on all cores."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    w, cx, mb = build_workload(args.workload, args.seed)
    from gpudock_b200 import abi
    from oracle import oracle as orc
    native = True
    try:
        orc.build(native=True)
    except Exception:
        native = False
    threads = orc.max_threads(native)
    params, _keep = abi.mc_params(w.steps, w.steps_per_exchange, mb, w.move_scale, seed=1)
    n_rep_total = cx.n_prt * cx.n_lig * w.n_tmp
    # each step: a replica sample x 2 MC steps sized to about 4 s of CPU work
    t0 = time.perf_counter()
    orc.mc_sample(cx, params, 0, threads, 1, threads, native)
    per_rep_step = max(time.perf_counter() - t0, 1e-4) / threads
    n_rep = int(min(n_rep_total, max(threads, 4.0 / (2 * per_rep_step))))
    for _ in range(args.warmup):
        orc.mc_sample(cx, params, 0, threads, 1, threads, native)
    t0 = time.perf_counter()
    done = 0
    for k in range(args.steps):
        done += orc.mc_sample(cx, params, (k * n_rep) % max(1, n_rep_total - n_rep), n_rep, 2,
                              threads, native)
    dt = time.perf_counter() - t0
    val = done / dt
    line = {
        "impl": "reference", "metric": "replica-MC-steps/s", "value": val,
        "unit": "replica-MC-steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w.name, "n_rep": n_rep_total, "lna": cx.lna, "pnp": cx.pnp,
                   "steps_per_exchange": w.steps_per_exchange},
        "cpu_baseline": {"value": val, "unit": "replica-MC-steps/s", "cores": threads,
                         "kind": "port",
                         "sample": f"per step {n_rep} replicas x 2 MC steps (C oracle, OpenMP)"},
        "e2e": {"value": val, "unit": "replica-MC-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    from gpudock_b200 import abi, lib

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist

    w, cx, mb = build_workload(args.workload, args.seed + 7919 * rank)
    n_rep = cx.n_prt * cx.n_lig * w.n_tmp
    spe = w.steps_per_exchange
    # a dedicated (non-default) stream shared by torch and the library, so the
    # CUDA events and the L2 flush are ordered with the library's kernels
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = lib.Context(local, stream.cuda_stream)
    dcx = lib.DeviceComplex(ctx, cx)
    total_steps = spe * (args.warmup + args.steps + 2)
    remc = lib.Remc(dcx, total_steps, spe, mb, w.move_scale, seed=args.seed + rank)
    remc.init()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        remc.run(spe)
    torch.cuda.synchronize()

    # ---- timed region: K exchange intervals, device-timed -----------------
    clocks = Clocks(local)
    clocks.start()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    remc.set_profiling(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(stream)
        remc.run(spe)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    gpu_launches = ctx.launches - launches0
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    mc_ms, mc_n, ex_ms, ex_n = remc.kernel_times()
    remc.set_profiling(False)
    if pg:
        t = torch.tensor([ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    out = remc.read()  # also checks the kernels' error word

    value = ws * n_rep * spe * args.steps / (ms * 1e-3)
    pairs_per_launch = n_rep * spe * cx.lna * cx.pnp
    mean_launch_s = mc_ms * 1e-3 / max(mc_n, 1)
    achieved = FLOP_PER_PAIR * pairs_per_launch / mean_launch_s / 1e12

    # ---- FP32 peak, measured on this GPU -------------------------------------
    peak = lib.fma_peak(ctx) / 1e12

    # ---- e2e through gd_run (host buffers) -----------------------------------
    e2e = None
    if not args.no_e2e:
        h2d = dcx.device_bytes + 4 * len(mb)
        d2h = n_rep * (4 * abi.NTERM + 4 * 6 + 4 + 4) + 4 * w.n_tmp
        for _ in range(1):
            lib.run(cx, spe, spe, mb, move_scale=w.move_scale, seed=args.seed)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        for k in range(args.steps):
            lib.run(cx, spe, spe, mb, move_scale=w.move_scale, seed=args.seed + k)
        dt = time.perf_counter() - t0
        if pg:
            t = torch.tensor([dt], device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            dt = float(t.item())
        e2e = {"value": ws * n_rep * spe * args.steps / dt, "unit": "replica-MC-steps/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "path": "gd_run: upload + init + 20 MC steps + exchange + read-back per step"}

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline(w, cx, mb)
            except Exception as exc:  # reported, not fatal
                cpu = {"value": None, "error": str(exc)}
        peaks = measured_peaks()
        line = {
            "metric": "replica-MC-steps/s", "value": value, "unit": "replica-MC-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name, "n_rep": n_rep, "n_prt": cx.n_prt,
                       "n_lig": cx.n_lig, "n_tmp": w.n_tmp, "lna": cx.lna, "pnp": cx.pnp,
                       "steps_per_exchange": spe, "step": "one exchange interval",
                       "l2": "flushed (256 MiB write) before every step",
                       "parallelism": f"replicas, {ws} independent ensemble(s)"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                         "kernel": "dock_kernel<REMC> (MC interval)",
                         "flops_per_launch": FLOP_PER_PAIR * pairs_per_launch,
                         "mean_launch_ms": mean_launch_s * 1e3, "launches": mc_n,
                         "peak_source": "measured live: FP32 FMA probe kernel on this GPU",
                         "exchange_kernel_ms": ex_ms / max(ex_n, 1)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": gpu_launches,
            "clocks": clk,
            "accept_rate": out.ac_mc / float(n_rep * spe * (args.warmup + args.steps)),
            "exchange_rate": out.ac_temp_exchg / float(
                max(1, n_rep * (args.warmup + args.steps))),
            "measured_peaks_file": {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops")},
        }
        print(json.dumps(line), flush=True)
    remc.close()
    dcx.close()
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
