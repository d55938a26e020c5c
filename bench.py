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
          bounded sample of the same workload on this host, on all cores
          (value) and on one thread (value_1_thread).

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
# The serving form runs one stream per launch shape; with the driver's
# default of 8 hardware work queues, launches of unrelated streams that map
# to one queue wait for each other.  32 queues (the maximum) must be asked
# for before the CUDA context exists.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

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
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the plain / batched / served / pose-sweep measurements")
    ap.add_argument("--tile", default=None,
                    help="launch shape A,P,NA of the headline workload instead of the "
                         "autotuner's (e.g. 4,3,10)")
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


def build_workload(name, seed, oracle_tables=False):
    """(workload, complex, minus_beta).  oracle_tables: derive the kernel
    tables and the temperature ladder with the oracle's restatements of
    OptimizeEnepara / SetTemperature (bit-identical to the library's), so
    that the reference arm never loads the library."""
    from gpudock_b200 import synth
    w = synth.WORKLOADS[name]
    if oracle_tables:
        from oracle import oracle as orc
        ff = orc.enepara_optimize(synth.raw_ff()[1])
        cx = synth.make_complex(w.spec, seed=seed, ff=ff)
        _, mb = synth.temperatures(w, orc.set_temperature)
    else:
        cx = synth.make_complex(w.spec, seed=seed)
        _, mb = synth.temperatures(w)
    return w, cx, mb


def workload_config(w, cx, ws):
    """The `config` object of both arms' JSON lines."""
    return {"workload": w.name, "n_rep": cx.n_prt * cx.n_lig * w.n_tmp, "n_prt": cx.n_prt,
            "n_lig": cx.n_lig, "n_tmp": w.n_tmp, "lna": cx.lna, "pnp": cx.pnp,
            "steps_per_exchange": w.steps_per_exchange,
            "step": f"one exchange interval ({w.steps_per_exchange} MC steps of every replica "
                    "+ one temperature exchange)",
            "l2": "GPU arm: flushed (256 MiB write) before every step",
            "parallelism": f"replicas, {ws} independent ensemble(s)"}


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
    n_steps = max(1, min(2000, int(budget_s / per / 4)))
    n_rep = min(n_rep_total, threads * 4)
    t0 = time.perf_counter()
    done = orc.mc_sample(cx, params, 0, n_rep, n_steps, threads, native)
    dt = time.perf_counter() - t0
    # one thread as well, on about a fifth of the budget
    n_steps1 = max(1, min(2000, int(budget_s / 5 / per)))
    t0 = time.perf_counter()
    done1 = orc.mc_sample(cx, params, 0, 1, n_steps1, 1, native)
    dt1 = time.perf_counter() - t0
    return {"value": done / dt, "unit": "replica-MC-steps/s", "cores": threads,
            "kind": "port", "value_1_thread": done1 / dt1,
            "sample": f"{n_rep} of {n_rep_total} replicas x {n_steps} MC steps "
                      f"({done} energy evaluations, {dt:.1f} s, "
                      f"{'-march=native' if native else 'x86-64'} OpenMP build); "
                      f"1 thread: 1 replica x {n_steps1} MC steps ({dt1:.1f} s)"}


def cpu_rate(cxs, mb, move_scale, spe, budget_s=3.0):
    """The oracle's replica-MC-steps/s on a sample of complexes (each complex's
    replicas in parallel), on all host cores and on one thread: a bounded
    sample sized to about budget_s seconds per leg."""
    from gpudock_b200 import abi
    from oracle import oracle as orc
    native = True
    try:
        orc.build(native=True)
    except Exception:
        native = False
    threads = orc.max_threads(native)
    params = [abi.mc_params(1000, spe, mb, move_scale, seed=1) for _ in cxs]
    out = {}
    for leg, nt in (("all_cores", threads), ("one_thread", 1)):
        # calibrate on one step of the first complex's replicas
        n_rep0 = cxs[0].n_prt * cxs[0].n_lig * len(mb)
        n_rep0 = min(n_rep0, nt * 4) if nt > 1 else 1
        t0 = time.perf_counter()
        orc.mc_sample(cxs[0], params[0][0], 0, n_rep0, 1, nt, native)
        per = max(time.perf_counter() - t0, 1e-5) / n_rep0 * nt  # s per replica-step per thread
        done, t_used = 0, 0.0
        for cx, (pa, _keep) in zip(cxs, params):
            n_rep = cx.n_prt * cx.n_lig * len(mb)
            n_rep = min(n_rep, max(nt, 1) * 2) if nt > 1 else 1
            n_steps = max(1, int(budget_s / len(cxs) / (per * n_rep / nt)))
            t0 = time.perf_counter()
            done += orc.mc_sample(cx, pa, 0, n_rep, n_steps, nt, native)
            t_used += time.perf_counter() - t0
        out[leg] = done / t_used
    return {"value": out["all_cores"], "unit": "replica-MC-steps/s", "cores": threads,
            "kind": "port", "value_1_thread": out["one_thread"],
            "sample": f"{len(cxs)} complex(es) of the form, a replica sample each, "
                      f"about {budget_s:g} s per leg (C oracle, OpenMP, "
                      f"{'-march=native' if native else 'x86-64'})"}


def profile_metric(workload, key):
    """(value, unit) of one metric row of the committed ncu summary of the
    headline kernel of this workload, or None."""
    import re
    path = os.path.join(ROOT, "profiles", f"dock_kernel_remc_{workload}.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"`" + re.escape(key) + r"`\) \| ([0-9.]+) ?([%\w]*)", open(path).read())
    return (float(m.group(1)), m.group(2)) if m else None


def profile_traffic(workload):
    """DRAM bytes per launch of the headline kernel from the committed ncu
    summary of this workload (dram__bytes_read.sum + dram__bytes_write.sum),
    or None without one."""
    import re
    path = os.path.join(ROOT, "profiles", f"dock_kernel_remc_{workload}.md")
    if not os.path.exists(path):
        return None
    scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    total = 0.0
    for key in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
        m = re.search(r"`" + re.escape(key) + r"`\) \| ([0-9.]+) (\w+)", open(path).read())
        if not m:
            return None
        total += float(m.group(1)) * scale.get(m.group(2), 1)
    return total


def _event_ms(stream, fn):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def form_plain(ctx, stream, seed, flush):
    """Plain form of the single-complex workload: 1,500 points x 24 atoms,
    8 temperatures (8 replicas, one CTA), exchange every 10 steps."""
    from gpudock_b200 import lib
    w, cx, mb = build_workload("plain_1500x24", seed)
    n_rep = cx.n_prt * cx.n_lig * w.n_tmp
    d = lib.DeviceComplex(ctx, cx)
    steps = 200
    r = lib.Remc(d, 4 * steps, w.steps_per_exchange, mb, w.move_scale, seed=seed)
    r.init()
    r.run(steps)
    flush.fill_(1)
    ms = _event_ms(stream, lambda: r.run(steps))
    r.read()
    r.close()
    d.close()
    return {"workload": w.name, "n_rep": n_rep, "mc_steps": steps,
            "value": n_rep * steps / (ms * 1e-3), "unit": "replica-MC-steps/s",
            "ms_per_mc_step": ms / steps,
            "cpu_baseline": cpu_rate([cx], mb, w.move_scale, w.steps_per_exchange)}


def form_batched(ctx, stream, seed, flush, n_steps=50):
    """Batched form: 512 ligands of 12..96 atoms x 4 conformations x 8
    temperatures (16,384 replicas) against one 6,000-point protein with 4
    conformations; launch shapes autotuned per ligand-size bucket; the
    exchange cadence chosen by the cadence autotuner among the divisors of
    the configuration's 10 steps (the most frequent exchange whose MC-step
    cost is within 2% of the cheapest, so it never exchanges less often than
    the configuration) and used for the timed run; timed over n_steps MC
    steps (a sample of the 3,000), median of 3."""
    import dataclasses
    from gpudock_b200 import abi, lib, synth
    w = synth.WORKLOADS["batched_512"]
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    prt = synth.make_protein(rng, w.spec, 9.0, raw)
    lo, hi = w.extra["lna_range"]
    lnas = rng.integers(lo, hi + 1, size=w.extra["n_ligand"])
    cxs = [synth.make_complex(dataclasses.replace(w.spec, lna=int(n), n_prt=w.spec.n_prt),
                              seed=seed + 100 + i, protein=prt) for i, n in enumerate(lnas)]
    _, mb = synth.temperatures(w)
    base = lib.DeviceComplex(ctx, cxs[0])
    dcxs = [lib.DeviceComplex(ctx, cx, share=base, prt_conf0=i % w.spec.n_prt, n_prt=1)
            for i, cx in enumerate(cxs)]
    t0 = time.perf_counter()
    tuned = lib.autotune_buckets(dcxs)
    tune_s = time.perf_counter() - t0
    # exchange cadence: candidates at least as frequent as the configuration's
    cands = tuple(c for c in (1, 2, 5, 10) if w.steps_per_exchange % c == 0)
    cad, table = lib.autotune_cadence(ctx, dcxs[:148], mb, candidates=cands, steps=40,
                                      move_scale=w.move_scale, seed=seed, flags=abi.MC_EXCHANGE)
    params = [abi.mc_params(w.steps, cad, mb, w.move_scale, seed=seed, stream_id=i,
                            flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY)
              for i in range(len(dcxs))]
    b = lib.Batch(ctx, dcxs, params)
    b.init()
    b.run(2 * w.steps_per_exchange)
    times = []
    launches = 0
    for _ in range(3):
        flush.fill_(2)
        launches0 = ctx.launches
        times.append(_event_ms(stream, lambda: b.run(n_steps)))
        launches = ctx.launches - launches0
    ms = statistics.median(times)
    b.set_profiling(True)
    b.run(n_steps)
    mc_ms, mc_n, ex_ms, ex_n = b.kernel_times()
    b.set_profiling(False)
    pairs = sum(4 * w.n_tmp * int(n) for n in lnas) * w.spec.pnp * n_steps
    out = {"workload": w.name, "n_rep": b.n_rep, "n_ligand": len(cxs),
           "lna_range": [int(lnas.min()), int(lnas.max())], "mc_steps_timed": n_steps,
           "value": b.n_rep * n_steps / (ms * 1e-3), "unit": "replica-MC-steps/s",
           "ms_per_mc_step": ms / n_steps, "timing": "median of 3 runs of n_steps",
           "launch_shapes": b.n_shapes, "gpu_launches": launches,
           "fp32_tflops": FLOP_PER_PAIR * pairs / (mc_ms * 1e-3) / 1e12 if mc_ms else None,
           "autotune_s": tune_s,
           "tiles": {f"lna<={k[0]},tiles={k[1]}": list(v[0]) for k, v in tuned.items()},
           "steps_per_exchange": cad,
           "cadence": {"chosen_steps_per_exchange": cad, "applied": True,
                       "candidates": list(cands),
                       "ms_per_mc_step": {str(k): v for k, v in table.items()},
                       "rule": "the most frequent exchange whose MC-step cost is within 2% of "
                               "the cheapest candidate",
                       "sample": "148 of the 512 ligands, 40 MC steps per candidate"}}
    b.close()
    pick = np.random.Generator(np.random.PCG64(seed + 9)).choice(len(cxs), 8, replace=False)
    out["cpu_baseline"] = cpu_rate([cxs[i] for i in pick], mb, w.move_scale, cad)
    out["cpu_baseline"]["sample"] = "8 of the 512 ligands; " + out["cpu_baseline"]["sample"]
    for d in dcxs:
        d.close()
    base.close()
    return out


def form_served(seed, rate=50.0, n_request=2000, steps=2000, budget_gb=120, pool=512,
                cpu=True, steps_per_launch=None, split=None, max_active=0):
    """Serving form: Poisson arrivals at `rate` req/s; ligand sizes log-normal
    (median 30, clipped to 8..120); each request 4 ligand conformations x 8
    temperatures (32 replicas) x `steps` MC steps against one of 4 resident
    proteins (2,000 / 4,000 / 7,000 / 10,000 points); admission by an HBM
    budget.  The requests cycle through a pool of `pool` distinct synthetic
    complexes, each submission with its own random stream.  Latency = submit
    -> result, measured by the server; the queue is sampled every 0.5 s."""
    import dataclasses
    from gpudock_b200 import abi, lib, synth
    w = synth.WORKLOADS["serving"]
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(seed + 2))
    prots = [synth.make_protein(rng, dataclasses.replace(w.spec, pnp=p), 10.0, raw)
             for p in w.extra["proteins"]]
    lo, hi = w.extra["lna_clip"]
    n_pool = min(n_request, pool)
    lnas = np.clip(np.round(np.exp(rng.normal(np.log(w.extra["lna_median"]), 0.5,
                                              n_pool))), lo, hi).astype(int)
    which = rng.integers(0, len(prots), n_pool)
    gaps = rng.exponential(1.0 / rate, n_request)
    cxs = [synth.make_complex(dataclasses.replace(w.spec, lna=int(n),
                                                  pnp=w.extra["proteins"][k]),
                              seed=seed + 1000 + i, protein=prots[k])
           for i, (n, k) in enumerate(zip(lnas, which))]
    _, mb = synth.temperatures(w)
    steps_per_launch = steps_per_launch or w.steps_per_exchange * 2
    srv = lib.Server(0, hbm_budget_bytes=int(budget_gb) << 30, max_active=max_active,
                     steps_per_launch=steps_per_launch)
    if split is not None:
        srv.set_split(split)
    pids = [srv.add_protein(cxs[int(np.nonzero(which == k)[0][0])]) if (which == k).any()
            else None for k in range(len(prots))]
    n_rep = 32
    pairs = 0.0
    series = []
    ids, pending = [], {}
    lat = np.zeros(n_request)
    svc = np.zeros(n_request)

    def sample(t0):
        st = srv.stats()
        series.append([round(time.perf_counter() - t0, 2), st.queued, st.active,
                       int(st.completed)])

    def collect():
        for i in list(pending):
            out = srv.poll(pending[i])
            if out is not None:
                lat[i] = out.log.t_wall
                svc[i] = out.log.t_compute
                del pending[i]

    t0 = time.perf_counter()
    t_next = t0
    t_sample = t0
    for i in range(n_request):
        k = i % n_pool
        t_next += gaps[i]
        while True:
            now = time.perf_counter()
            if now >= t_sample:
                sample(t0)
                collect()
                t_sample += 0.5
            if now >= t_next:
                break
            time.sleep(min(t_next - now, max(0.0, t_sample - now), 0.01))
        rid = srv.submit(pids[which[k]], cxs[k], steps, w.steps_per_exchange, mb, n_prt=1,
                         seed=seed, stream_id=i, flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY)
        ids.append(rid)
        pending[i] = rid
        pairs += n_rep * steps * int(lnas[k]) * w.extra["proteins"][which[k]]
    t_submitted = time.perf_counter() - t0
    while pending:
        if time.perf_counter() >= t_sample:
            sample(t0)
            t_sample += 0.5
        collect()
        time.sleep(0.01)
    wall = time.perf_counter() - t0
    sample(t0)
    st = srv.stats()
    srv.close()
    n_sm = 148
    try:
        import torch
        n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    except Exception:
        pass
    skip = n_request // 5  # the first fifth fills the GPU: not steady state
    out = {"workload": w.name, "n_request": n_request, "rate_req_s": rate,
           "mc_steps": steps, "replicas_per_request": n_rep,
           "value": n_request * n_rep * steps / wall, "unit": "replica-MC-steps/s",
           "requests_per_s": n_request / wall,
           "fp32_tflops": FLOP_PER_PAIR * pairs / wall / 1e12,
           "submitted_in_s": t_submitted, "wall_s": wall,
           "p50_latency_s": float(np.percentile(lat[skip:], 50)),
           "p99_latency_s": float(np.percentile(lat[skip:], 99)),
           "p50_latency_all_s": float(np.percentile(lat, 50)),
           "p99_latency_all_s": float(np.percentile(lat, 99)),
           "p50_service_s": float(np.percentile(svc[skip:], 50)),
           "p99_service_s": float(np.percentile(svc[skip:], 99)),
           "latency_window": f"requests {skip}..{n_request - 1} (after the first fifth)",
           "sm_occupancy": st.cta_busy_s / (n_sm * wall),
           "host_launch_s": st.host_launch_s,
           "busy_s": st.busy_s, "launches": st.launches,
           "steps_per_launch": steps_per_launch,
           "queue_series": {"every_s": 0.5, "columns": ["t_s", "queued", "active", "completed"],
                            "rows": series[::4]},
           "sample": f"{n_request} requests of the 10,000-request trace at {rate:g} req/s, "
                     f"cycling through {n_pool} distinct synthetic complexes"}
    if cpu:
        pick = np.random.Generator(np.random.PCG64(seed + 4)).choice(n_pool, 8, replace=False)
        out["cpu_baseline"] = cpu_rate([cxs[i] for i in pick], mb, w.move_scale,
                                       w.steps_per_exchange)
        out["cpu_baseline"]["sample"] = ("8 of the requests (throughput only); "
                                         + out["cpu_baseline"]["sample"])
    return out


def form_poses(ctx, stream, seed, n_pose=1 << 20):
    """Energy-only sweep: n_pose random rigid poses of a 48-atom ligand against
    proteins of 2,000 / 4,000 / 8,000 / 16,000 points (pose-energies/s)."""
    import dataclasses
    import torch
    from gpudock_b200 import abi, lib, synth
    w = synth.WORKLOADS["poses_48"]
    rng = np.random.default_rng(seed + 3)
    poses_h = synth.random_poses(rng, n_pose, box=w.extra["box"])
    poses = torch.from_numpy(poses_h).cuda()
    terms = torch.empty((n_pose, 10), dtype=torch.float32, device="cuda")
    out = {}
    for pnp in w.extra["pnp_sweep"]:
        cx = synth.make_complex(dataclasses.replace(w.spec, pnp=pnp), seed=seed + pnp)
        d = lib.DeviceComplex(ctx, cx)
        run = lambda: d.energy_poses_dev(n_pose, poses.data_ptr(), terms.data_ptr())
        # the other shapes that cover 48 atoms, timed on the sweep itself,
        # beside the autotuner's choice (which is timed on MC steps)
        alt = {}
        for t in ((5, 2, 10), (6, 2, 8), (8, 1, 6), (12, 1, 4)):
            lib.check(ctx._lib.gd_ctx_set_tile(ctx.h, cx.lna, pnp, abi.GdTile(*t)),
                      "gd_ctx_set_tile")
            run()
            alt[",".join(map(str, t))] = _event_ms(stream, run)
        tile, _ = d.autotune()
        run()
        ms = _event_ms(stream, run)
        out[str(pnp)] = {"value": n_pose / (ms * 1e-3), "unit": "pose-energies/s",
                         "fp32_tflops": FLOP_PER_PAIR * n_pose * cx.lna * pnp / (ms * 1e-3)
                         / 1e12, "tile": list(tile),
                         "ms_by_tile_A_P_NA": alt,
                         "cpu_baseline": cpu_poses_rate(cx, poses_h)}
        d.close()
    return {"workload": w.name, "n_pose": n_pose, "by_protein_points": out}


def cpu_poses_rate(cx, poses, budget_s=2.0):
    """The oracle's pose-energies/s on a prefix of the sweep's poses, on all
    host cores and on one thread (about budget_s seconds per leg)."""
    from oracle import oracle as orc
    native = True
    try:
        orc.build(native=True)
    except Exception:
        native = False
    threads = orc.max_threads(native)
    out = {}
    for leg, nt in (("all_cores", threads), ("one_thread", 1)):
        n = nt
        t0 = time.perf_counter()
        orc.energy_poses(cx, poses[:n], n_threads=nt, native=native)
        per = max(time.perf_counter() - t0, 1e-5) / n * nt
        n = int(min(4096, max(nt, budget_s / per * nt)))
        t0 = time.perf_counter()
        orc.energy_poses(cx, poses[:n], n_threads=nt, native=native)
        out[leg] = (n / (time.perf_counter() - t0), n)
    return {"value": out["all_cores"][0], "unit": "pose-energies/s", "cores": threads,
            "kind": "port", "value_1_thread": out["one_thread"][0],
            "sample": f"{out['all_cores'][1]} poses on all cores, {out['one_thread'][1]} on one "
                      f"thread (C oracle, {'-march=native' if native else 'x86-64'})"}


def form_similarity(ctx, cx, seed, n_conf=4096):
    """Contact-mode similarity matrix of n_conf conformations of the headline
    complex (random protein / ligand conformations, moves of ~1.5 A and
    ~0.3 rad about the pocket), through gd_similarity_matrix with host
    buffers: matrix entries per second of the whole call."""
    from gpudock_b200 import lib
    rng = np.random.Generator(np.random.PCG64(seed + 5))
    confs = np.zeros((n_conf, 8), np.float32)
    confs[:, 0] = rng.integers(0, cx.n_prt, n_conf)
    confs[:, 1] = rng.integers(0, cx.n_lig, n_conf)
    confs[:, 2:5] = rng.normal(0.0, 1.5, (n_conf, 3))
    confs[:, 5:8] = rng.normal(0.0, 0.3, (n_conf, 3))
    import torch
    d = lib.DeviceComplex(ctx, cx)
    d.similarity_matrix(confs)  # warm-up: grows the stream-ordered pool to this size
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        S = d.similarity_matrix(confs)
        times.append(time.perf_counter() - t0)
    dt = statistics.median(times)
    # the matrix left in device memory (gd_similarity_matrix_dev), on ctx's device
    out = torch.empty((n_conf, n_conf), dtype=torch.float32, device=f"cuda:{ctx.device}")
    torch.cuda.synchronize()
    d.similarity_matrix_dev(confs, out.data_ptr())
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        d.similarity_matrix_dev(confs, out.data_ptr())
        times.append(time.perf_counter() - t0)
    dt_dev = statistics.median(times)
    d.close()
    return {"workload": f"similarity_{n_conf}", "n_conf": n_conf,
            "value": n_conf * n_conf / dt, "unit": "contact-MCC entries/s", "ms": dt * 1e3,
            "ms_device_output": dt_dev * 1e3,
            "median_entry": float(np.median(S)), "timing": "median of 3 calls each",
            "path": "gd_similarity_matrix: host conformations in, host matrix out "
                    "(ms_device_output: gd_similarity_matrix_dev, matrix left on the GPU)"}


def run_reference(args):
    """--impl reference: the reference's CPU path (oracle port) on all cores."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    w, cx, mb = build_workload(args.workload, args.seed, oracle_tables=True)
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
        "config": workload_config(w, cx, ws),
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
    if args.tile:
        tile = tuple(int(v) for v in args.tile.split(","))
        lib.check(ctx._lib.gd_ctx_set_tile(ctx.h, cx.lna, cx.pnp, abi.GdTile(*tile)),
                  "gd_ctx_set_tile")
    else:
        tile, _ = dcx.autotune()  # launch shape of this size class, kept in ctx
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

    forms = None
    if ws == 1 and not args.no_forms:
        forms = {}
        for name, fn in (("plain", lambda: form_plain(ctx, stream, args.seed, flush)),
                         ("batched", lambda: form_batched(ctx, stream, args.seed, flush)),
                         ("poses", lambda: form_poses(ctx, stream, args.seed)),
                         ("similarity", lambda: form_similarity(ctx, cx, args.seed)),
                         ("served", lambda: form_served(args.seed)),
                         # the top of the trace's rate range: the requests arrive
                         # faster than they finish, so this measures capacity
                         ("served_400", lambda: form_served(args.seed, rate=400.0,
                                                            cpu=False))):
            try:
                forms[name] = fn()
            except Exception as exc:  # reported, not fatal
                forms[name] = {"error": f"{type(exc).__name__}: {exc}"}

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline(w, cx, mb)
            except Exception as exc:  # reported, not fatal
                cpu = {"value": None, "error": str(exc)}
        peaks = measured_peaks()
        traffic = profile_traffic(w.name)
        hbm_peak = peaks.get("hbm_gbs")
        hbm = {"achieved_gbs": traffic / mean_launch_s / 1e9 if traffic else None,
               "peak_gbs": hbm_peak,
               "frac": traffic / mean_launch_s / 1e9 / hbm_peak if traffic and hbm_peak
               else None,
               "note": "DRAM bytes per launch (ncu) / mean launch time, against the measured "
                       "copy bandwidth of MEASURED_PEAKS.json: the kernel is not HBM-bound"}
        line = {
            "metric": "replica-MC-steps/s", "value": value, "unit": "replica-MC-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(w, cx, ws),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": traffic, "hbm": hbm,
                         "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per "
                                           "launch, ncu capture summarised in profiles/",
                         "ncu_pipe_util_pct": {
                             "fma": profile_metric(
                                 w.name,
                                 "sm__pipe_fma_cycles_active.avg.pct_of_peak_sustained_active"),
                             "xu": profile_metric(
                                 w.name,
                                 "sm__inst_executed_pipe_xu.avg.pct_of_peak_sustained_active"),
                             "note": "FP32 (FMA) and MUFU (XU) pipe utilisation of the same "
                                     "kernel from the committed ncu capture; frac counts the 36 "
                                     "algorithmic flops per pair against the FFMA peak"},
                         "kernel": "dock_kernel<REMC> (MC interval)",
                         "tile_A_P_NA": list(tile),
                         "flops_per_launch": FLOP_PER_PAIR * pairs_per_launch,
                         "mean_launch_ms": mean_launch_s * 1e3, "launches": mc_n,
                         "peak_source": "measured live: FP32 FMA probe kernel on this GPU",
                         "exchange_kernel_ms": ex_ms / max(ex_n, 1)},
            "cpu_baseline": cpu,
            "forms": forms,
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
