#!/usr/bin/env python
"""Benchmark: split-step wavefront propagation throughput on B200.

Workload (one bench step): the three-grating Talbot-Lau interferometer at
N = 2^24 complex128 (dx = 2 nm), 32 energies 20-70 keV weighted by a filtered
Kramers spectrum, G2 stepped over 8 phase steps -> 102 split steps per energy,
3264 split steps per bench step, detector intensity accumulated in FP64.
Inputs are seeded synthetic (plane-wave illumination, tabulated materials).

Metric: propagated complex samples * split steps per second (whole job, all
ranks). One split step = one transmission + FFT + transfer function + iFFT
of the reference's schedule (big-wave/wavesim.py:84-298).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rsw|reference]

Multi-GPU (torchrun, one rank per GPU): weak scaling, each rank runs its own
32 energies of a 32*N-energy spectrum; the FP64 detector accumulators are
summed with one NCCL all-reduce per step.
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

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "propagated complex samples*steps/s"
UNIT = "samples*steps/s"
PROFILE_TRAFFIC = ROOT / "profiles" / "ncu_traffic.txt"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="rsw", choices=["rsw", "reference"])
    ap.add_argument("--dtype", default="c16", choices=["c16", "c8"])
    ap.add_argument("--logn", type=int, default=24)
    ap.add_argument("--energies", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end measurement")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic(kernel: str, dtype: str, logn: int):
    """dram bytes per launch from the committed ncu summary (scaled to 2^logn)."""
    if not PROFILE_TRAFFIC.exists():
        return None
    for line in PROFILE_TRAFFIC.read_text().splitlines():
        f = line.split()
        if len(f) >= 4 and not line.startswith("#") and f[0] == kernel and f[1] == dtype:
            cap_logn, by = int(f[2]), float(f[3])
            return by * 2.0 ** (logn - cap_logn)
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms (own process)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", gpu_id], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                rows.append((float(c[1]), float(c[2]), float(c[3]), c[5:9]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "reasons": reasons}


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return rank, ws, local


# ----------------------------------------------------------- CPU baselines
def cpu_split_steps(logn, dtype, n_steps, workers):
    """Time ``n_steps`` split steps of the oracle port (FP64 numpy/scipy
    restatement of big-wave): G0 grating sub-steps (mask multiply + propagate)
    at the workload's N. Returns (samples*steps/s, seconds)."""
    import scipy.fft as spfft

    from oracle import bigwave_np as bw
    from rave_sim_b200 import workloads

    case = workloads.talbot_lau(n=1 << logn, dtype=dtype)
    sim = bw.make_sim(case)
    el = dict(case["elements"][0])
    el["nr_steps"] = n_steps
    el["thickness"] = el["thickness"] * n_steps / case["elements"][0]["nr_steps"]
    u = np.ones(sim.N, np.complex128 if dtype == "c16" else np.complex64)
    with spfft.set_workers(workers):
        t = time.perf_counter()
        bw.apply_grating(u, None, sim, el, case["db"], np.sin(case["cutoff_angles"][1]) / sim.wl, 0)
        dt = time.perf_counter() - t
    return sim.N * n_steps / dt, dt


def reference_arm(args, rank, ws):
    """--impl reference: the reference's CPU path (the oracle port of big-wave's
    FP64 NumpyVector path; big-wave itself is not installable on the GPU host)
    on all host cores, rank 0 only."""
    if rank != 0:
        return
    workers = os.cpu_count() or 1
    rates = []
    for i in range(args.warmup + args.steps):
        r, _ = cpu_split_steps(args.logn, args.dtype, 1, workers)
        if i >= args.warmup:
            rates.append(r)
    v = float(np.mean(rates))
    n = 1 << args.logn
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": n / v * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.dtype == "c16" else "f32",
        "data": "synthetic",
        "config": {"workload": f"talbot_lau_3g_N2^{args.logn}_{args.dtype}", "sample": "1 split step per bench step"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": f"1 grating split step (mask + FFT + transfer + iFFT) at N=2^{args.logn}, "
                                   f"scipy.fft workers={workers}"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ main
def main():
    args = parse()
    rank, ws, local = dist_init(args)
    if args.impl == "reference":
        reference_arm(args, rank, ws)
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    import torch

    import rave_sim_b200 as rsw
    from rave_sim_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = rsw.load_library()
    n = 1 << args.logn
    case = workloads.talbot_lau(n=n, dtype=args.dtype)
    from rave_sim_b200.sharding import reduce_detector, shard_sources

    all_e, all_w = workloads.config2_energies(args.energies * ws)
    mine = shard_sources([1.0] * len(all_e), ws)[rank]  # equal cost: same N and schedule per energy
    my_e, my_w = all_e[mine], all_w[mine]
    sim = rsw.Simulation(case, dtype=args.dtype)
    acc = torch.zeros((sim.nr_phase_steps, sim.n_pix), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    def run_step(source, field=None):
        sim.reset()
        for e, w in zip(my_e, my_w):
            sim.run_source(energy=float(e), db_table=workloads.db_table(float(e)), source=source,
                           weight=float(w), field=field)
        sim.detected_device(acc)
        reduce_detector(acc)

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    plane = case["source"]
    s0 = sim.split_steps
    run_step(plane)
    steps_per_bench_step = sim.split_steps - s0
    for _ in range(args.warmup - 1):
        run_step(plane)

    # ---- timed region (device resident)
    gpu_id = str(getattr(torch.cuda.get_device_properties(dev), "uuid", local))
    if gpu_id and not gpu_id.startswith("GPU-") and len(gpu_id) > 8:
        gpu_id = "GPU-" + gpu_id
    clocks = ClockSampler(gpu_id)
    barrier()
    l0 = lib.rsw_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        run_step(plane)
    ev1.record(stream)
    barrier()
    t_wall = time.perf_counter() - t_wall
    launches = lib.rsw_launch_count() - l0
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1)) / args.steps
    total_samples = float(n) * steps_per_bench_step * ws
    value = total_samples / (ms * 1e-3)

    # ---- end to end through the public API with host buffers
    npd = np.complex128 if args.dtype == "c16" else np.complex64
    h_field = torch.from_numpy(np.ones(n, npd)).pin_memory()
    d_field = torch.empty(n, dtype=h_field.dtype, device=dev)
    h_out = torch.empty((sim.nr_phase_steps, sim.n_pix), dtype=torch.float64).pin_memory()
    vec = {"type": "vector", "z": plane["z"]}

    def e2e_step():
        d_field.copy_(h_field, non_blocking=True)
        run_step(vec, field=d_field)
        h_out.copy_(acc, non_blocking=True)

    e2e_ms = e2e_value = None
    if not args.no_e2e:
        e2e_step()
        barrier()
        ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2e_steps = max(1, min(args.steps, 2))
        ev2.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        ev3.record(stream)
        barrier()
        e2e_ms = max_over_ranks(ev2.elapsed_time(ev3)) / e2e_steps
        e2e_value = total_samples / (e2e_ms * 1e-3)

    # ---- per-kernel device time (CUDA events on the launch stream), one energy
    sim.set_timing(True)
    sim.run_source(energy=float(my_e[0]), db_table=workloads.db_table(float(my_e[0])), source=plane, weight=0.0)
    kinds = {}
    for k, name in ((0, "row_pass"), (1, "col_pass"), (2, "detect")):
        t, cnt = sim.timing(k)
        kinds[name] = {"ms_total": t, "launches": cnt, "ms_avg": t / cnt if cnt else None}
    sim.set_timing(False)
    s_bytes = 16 if args.dtype == "c16" else 8
    dom = max(("row_pass", "col_pass"), key=lambda k: kinds[k]["ms_total"])
    avg_ms = kinds[dom]["ms_avg"]
    algo_bytes = 2.0 * n * s_bytes  # read + write of the field per pass launch
    peak, peak_kind = measured_peak_hbm()
    achieved = algo_bytes / (avg_ms * 1e-3) / 1e9
    for k in ("row_pass", "col_pass"):
        if kinds[k]["ms_avg"]:
            kinds[k]["GBps"] = algo_bytes / (kinds[k]["ms_avg"] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_launch": algo_bytes,
                "traffic": ncu_traffic(dom, args.dtype, args.logn), "kernels": kinds}

    # ---- CPU baseline (rank 0, N=1): oracle port on a bounded sample
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        k = 3
        v, dt = cpu_split_steps(args.logn, args.dtype, k, 1)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{k} grating split steps (mask + FFT + transfer + iFFT) at N=2^{args.logn} "
                         f"{args.dtype}, FP64 numpy/scipy oracle, 1 thread, {dt:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.dtype == "c16" else "f32+f64",
            "data": "synthetic (seeded plane wave, tabulated gratings)",
            "config": {"workload": f"talbot_lau_3g_N2^{args.logn}_{args.dtype}",
                       "n": n, "energies_per_rank": len(my_e), "phase_steps": sim.nr_phase_steps,
                       "split_steps_per_bench_step": steps_per_bench_step * ws,
                       "field_bytes": n * s_bytes, "l2_policy": "inputs larger than L2 (field 2^24 c128 = 256 MiB)",
                       "parallelism": f"dp{ws} (energies sharded, detector all-reduce)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * s_bytes,
                    "d2h_bytes_per_step": sim.nr_phase_steps * sim.n_pix * 8, "ms_per_step": e2e_ms},
            "gpu_launches": int(launches),
            "wall_s": t_wall,
            "clocks": clk,
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
