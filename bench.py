#!/usr/bin/env python
"""Benchmark: split-step wavefront propagation throughput on B200.

Default workload (one bench step): the three-grating Talbot-Lau
interferometer at N = 2^24 complex128 (dx = 2 nm), 32 energies 20-70 keV
weighted by a filtered Kramers spectrum, G2 stepped over 8 phase steps ->
102 split steps per energy, 3264 split steps per bench step, detector
intensity accumulated in FP64. Inputs are seeded synthetic (plane-wave
illumination, tabulated materials).

Other workloads (--workload):
  batched       128 energies on fields of 2^20..2^25 samples over one
                window (one field length per group of ~21 energies, groups on
                separate streams), complex64 by default
  thick_sample  the interferometer with a 200-slice cracked aluminium
                cylinder between G1 and G2, N = 2^26 (--energies per step)
  large_field   the interferometer on 2^31 complex64 / 2^30 complex128 samples
--compare-fp64 adds the detector error of a complex64 run against the
complex128 run of the same step (rel-L2 and max-abs / max).

Metric: propagated complex samples * split steps per second (whole job, all
ranks). One split step = one transmission + FFT + transfer function + iFFT
of the reference's schedule (big-wave/wavesim.py:84-298).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rsw|reference]
                    [--workload talbot_lau|batched|thick_sample|large_field]

Multi-GPU (torchrun, one rank per GPU): weak scaling, each rank runs its own
share of an N-times larger energy list (longest-processing-time sharding);
the FP64 detector accumulators are summed with one NCCL all-reduce per step.
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
    ap.add_argument("--workload", default="talbot_lau",
                    choices=["talbot_lau", "batched", "thick_sample", "large_field"])
    ap.add_argument("--dtype", default=None, choices=["c16", "c8"],
                    help="default: c16 for talbot_lau, c8 otherwise")
    ap.add_argument("--logn", type=int, default=None, help="field length (talbot_lau 24, thick_sample 26, "
                    "large_field 31 for c8 / 30 for c16)")
    ap.add_argument("--energies", type=int, default=None,
                    help="energies per rank and bench step (talbot_lau 32, batched 128, thick_sample 8, "
                         "large_field 1)")
    ap.add_argument("--compare-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end measurement")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the built-in schedule instead of timing the candidates first")
    ap.add_argument("--no-gpu-baseline", action="store_true",
                    help="skip the reference's cuFFT fast-wave path on the same workload")
    ap.add_argument("--no-batch", action="store_true",
                    help="run the sources of a field length one after the other instead of in lockstep "
                         "(one launch per pass for all of them)")
    a = ap.parse_args()
    if a.dtype is None:
        a.dtype = "c16" if a.workload == "talbot_lau" else "c8"
    if a.logn is None:
        a.logn = {"talbot_lau": 24, "batched": 25, "thick_sample": 26,
                  "large_field": 31 if a.dtype == "c8" else 30}[a.workload]
    if a.energies is None:
        a.energies = {"talbot_lau": 32, "batched": 128, "thick_sample": 8, "large_field": 1}[a.workload]
    return a


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
    """(dram bytes per launch, how) from the committed ncu summary: the
    capture at this size when there is one, else the 2^24 capture scaled by
    the samples per launch."""
    if not PROFILE_TRAFFIC.exists():
        return None, None
    lines = {}
    for line in PROFILE_TRAFFIC.read_text().splitlines():
        f = line.split()
        if len(f) >= 4 and not line.startswith("#") and f[0] == kernel and f[1] == dtype:
            lines[int(f[2])] = float(f[3])
    if logn in lines:
        return lines[logn], f"ncu capture at 2^{logn}"
    if 24 in lines:
        return lines[24] * 2.0 ** (logn - 24), f"ncu capture at 2^24 scaled by 2^{logn - 24}"
    return None, None


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
    lg = min(args.logn, CPU_SAMPLE_MAX_LOGN)
    rates = []
    for i in range(args.warmup + args.steps):
        r, _ = cpu_split_steps(lg, args.dtype, 1, workers)
        if i >= args.warmup:
            rates.append(r)
    v = float(np.mean(rates))
    n = 1 << lg
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": n / v * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.dtype == "c16" else "f32",
        "data": "synthetic",
        "config": {"workload": workload_name(args), "sample": f"1 split step at N=2^{lg} per bench step"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": f"1 grating split step (mask + FFT + transfer + iFFT) at N=2^{lg}, "
                                   f"scipy.fft workers={workers}"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def gpu_baseline(args, value, det):
    """The reference's GPU path (fast-wave's kernels and cuFFT, compiled
    unmodified, on fast-wave's schedule) timed on the same workload and
    energies in its own process (baseline/fastwave). Never falls back to the
    engine's kernels: without the prebuilt library the block says why."""
    lib = ROOT / "baseline" / "_ref" / "libfastwave_harness.so"
    if args.workload not in ("talbot_lau", "thick_sample"):
        return {"unavailable": f"no fast-wave baseline for the {args.workload} workload"}
    if args.logn > 30:
        return {"unavailable": "fast-wave indexes fields with int (N > 2^30 is out of its range)"}
    if not lib.exists():
        return {"unavailable": "baseline/_ref/libfastwave_harness.so is not built (needs the reference checkout)"}
    with tempfile.TemporaryDirectory() as td:
        out = Path(td) / "det.npy"
        cmd = [sys.executable, "-m", "baseline.fastwave.run", "--workload", args.workload, "--dtype", args.dtype,
               "--logn", str(args.logn), "--energies", str(args.energies), "--repeats", "1", "--warmup", "1",
               "--detector", str(out)]
        r = subprocess.run(cmd, cwd=str(ROOT), capture_output=True, text=True)
        if r.returncode != 0 or not r.stdout.strip():
            tail = (r.stderr or r.stdout).strip().splitlines()[-1:] or ["no output"]
            return {"unavailable": f"fast-wave run failed (exit {r.returncode}): {tail[0][:200]}"}
        b = json.loads(r.stdout.strip().splitlines()[-1])
        fw = np.load(out)
    b["ratio"] = value / b["value"]
    if det is not None and fw.shape == det.shape and np.linalg.norm(det) > 0:
        # fast-wave follows its own discrete rules (grating coordinates, cutoff,
        # binning): information, not a parity figure
        b["detector_rel_l2_vs_engine"] = float(np.linalg.norm(fw - det) / np.linalg.norm(det))
    return b


# ------------------------------------------------------------------ jobs
CPU_SAMPLE_MAX_LOGN = 24  # the oracle port times its sample at most at 2^24 (host memory and time)


def workload_name(args):
    return {"talbot_lau": f"talbot_lau_3g_N2^{args.logn}_{args.dtype}",
            "batched": f"batched_128E_N2^20-2^25_{args.dtype}",
            "thick_sample": f"thick_sample_200slices_N2^{args.logn}_{args.dtype}",
            "large_field": f"large_field_N2^{args.logn}_{args.dtype}"}[args.workload]


def build_groups(args, ws, rank, dtype):
    """This rank's work: a list of dicts (case, grids, energies, weights, db),
    one per field length; the energies of all ranks are sharded by cost."""
    from rave_sim_b200 import workloads
    from rave_sim_b200.sharding import shard_sources

    items = []  # (group index, energy, weight)
    groups = []
    if args.workload == "batched":
        count = args.energies * ws
        for g, (case, e, w) in enumerate(workloads.batched_energies(count=count, dtype=dtype)):
            groups.append({"case": case, "grids": None, "db": workloads.db_table})
            items += [(g, float(x), float(y)) for x, y in zip(e, w)]
    else:
        grids = None
        db = workloads.db_table
        if args.workload == "talbot_lau":
            case = workloads.talbot_lau(n=1 << args.logn, dtype=dtype)
        elif args.workload == "thick_sample":
            case, grids = workloads.thick_sample(n=1 << args.logn, dtype=dtype)
            db = workloads.db_table_sample
        else:
            case = workloads.large_field(dtype=dtype, n=1 << args.logn)
        count = args.energies * ws
        e, w = workloads.config2_energies(count)
        groups.append({"case": case, "grids": grids, "db": db})
        items = [(0, float(x), float(y)) for x, y in zip(e, w)]
    costs = [float(groups[g]["case"]["sim_params"]["N"]) for g, _, _ in items]
    mine = shard_sources(costs, ws)[rank]
    for g in groups:
        g["energies"], g["weights"] = [], []
    for i in mine:
        g, e, w = items[i]
        groups[g]["energies"].append(e)
        groups[g]["weights"].append(w)
    return [g for g in groups if g["energies"]] or groups[:1]


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
    from rave_sim_b200.sharding import reduce_detector

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = rsw.load_library()
    s_bytes = 16 if args.dtype == "c16" else 8
    groups = build_groups(args, ws, rank, args.dtype)
    tuning = {}
    if not args.no_autotune:
        # the schedule of each field length chosen by timing (registered for
        # the simulations created below), on batches of that length's fields
        # when its sources run in lockstep (up to 4 GiB of fields)
        from rave_sim_b200 import autotune

        for g in groups:
            n_g = int(g["case"]["sim_params"]["N"])
            fields = 1
            if not args.no_batch and len(g["energies"]) > 1:
                fields = max(1, min(len(g["energies"]), (4 << 30) // (n_g * s_bytes)))
            r = autotune.tune(n_g, args.dtype, reps=3 if fields > 1 else 5, save=False, fields=fields)
            tuning[str(n_g)] = {"choice": r["best"], "ms_per_split_step": r["ms_per_split_step"],
                                "fields": fields, "candidates": len(r["tried"])}
    for g in groups:
        g["sim"] = rsw.Simulation(g["case"], grids=g["grids"], dtype=args.dtype)
        g["n"] = int(g["case"]["sim_params"]["N"])
    main_stream = torch.cuda.current_stream()
    for g in groups:
        g["stream"] = torch.cuda.Stream() if len(groups) > 1 else main_stream
    sim0 = groups[0]["sim"]
    batch = not args.no_batch
    acc = torch.zeros((sim0.nr_phase_steps, sim0.n_pix), dtype=torch.float64, device=dev)
    accs = [torch.zeros_like(acc) for _ in groups]

    def run_step(fields=None):
        for i, g in enumerate(groups):
            g["stream"].wait_stream(main_stream)
            with torch.cuda.stream(g["stream"]):
                sim = g["sim"]
                sim.reset()
                src = g["case"]["source"] if fields is None else {"type": "vector", "z": g["case"]["source"]["z"]}
                f = None if fields is None else fields[i]
                if batch:
                    sim.run_sources([{"energy": e, "db_table": g["db"](e), "weight": w}
                                     for e, w in zip(g["energies"], g["weights"])], source=src, field=f)
                else:
                    for e, w in zip(g["energies"], g["weights"]):
                        sim.run_source(energy=e, db_table=g["db"](e), source=src, weight=w, field=f)
                sim.detected_device(accs[i])
        for g in groups:
            main_stream.wait_stream(g["stream"])
        torch.sum(torch.stack(accs), dim=0, out=acc)
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

    s0 = [g["sim"].split_steps for g in groups]
    run_step()
    torch.cuda.synchronize()
    steps_g = [g["sim"].split_steps - a for g, a in zip(groups, s0)]
    samples_step = float(sum(g["n"] * k for g, k in zip(groups, steps_g)))
    for _ in range(args.warmup - 1):
        run_step()

    # ---- timed region (device resident)
    gpu_id = str(getattr(torch.cuda.get_device_properties(dev), "uuid", local))
    if gpu_id and not gpu_id.startswith("GPU-") and len(gpu_id) > 8:
        gpu_id = "GPU-" + gpu_id
    clocks = ClockSampler(gpu_id)
    barrier()
    l0 = lib.rsw_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall = time.perf_counter()
    ev0.record(main_stream)
    for _ in range(args.steps):
        run_step()
    ev1.record(main_stream)
    barrier()
    t_wall = time.perf_counter() - t_wall
    launches = lib.rsw_launch_count() - l0
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1)) / args.steps
    total_samples = samples_step * ws  # weak scaling: every rank runs an equal share
    value = total_samples / (ms * 1e-3)

    # ---- end to end through the public API with host buffers: each group's
    # input field uploaded from pinned memory every step (fields above 4 GiB:
    # plane-wave source, nothing uploaded), detector read back
    e2e_ms = e2e_value = None
    h2d = 0
    h_out = torch.empty_like(acc, device="cpu").pin_memory()
    if not args.no_e2e:
        npd = np.complex128 if args.dtype == "c16" else np.complex64
        upload = all(g["n"] * s_bytes <= (4 << 30) for g in groups)
        if upload:
            h_fields = [torch.from_numpy(np.ones(g["n"], npd)).pin_memory() for g in groups]
            d_fields = [torch.empty(g["n"], dtype=h.dtype, device=dev) for g, h in zip(groups, h_fields)]
            h2d = sum(g["n"] * s_bytes for g in groups)

        def e2e_step():
            if upload:
                for d, h in zip(d_fields, h_fields):
                    d.copy_(h, non_blocking=True)
            run_step(d_fields if upload else None)
            h_out.copy_(acc, non_blocking=True)

        e2e_step()
        barrier()
        ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2e_steps = args.steps
        ev2.record(main_stream)
        for _ in range(e2e_steps):
            e2e_step()
        ev3.record(main_stream)
        barrier()
        e2e_ms = max_over_ranks(ev2.elapsed_time(ev3)) / e2e_steps
        e2e_value = total_samples / (e2e_ms * 1e-3)

    # ---- per-kernel device time (CUDA events on the launch stream): the
    # largest field's sources as the timed region runs them (a lockstep batch
    # of all of them, or one energy)
    gd = max(groups, key=lambda g: g["n"])
    n = gd["n"]
    sim = gd["sim"]
    sim.set_timing(True)
    steps0 = sim.split_steps
    if batch:
        sim.run_sources([{"energy": e, "db_table": gd["db"](e), "weight": 0.0} for e in gd["energies"]],
                        source=gd["case"]["source"])
    else:
        e = gd["energies"][0]
        sim.run_source(energy=e, db_table=gd["db"](e), source=gd["case"]["source"], weight=0.0)
    # fields per pass launch: split steps of all sources over row launches (a
    # batch that the engine runs source by source launches once per field)
    row_t, row_n = sim.timing(0)
    per_launch = max(1, int(round((sim.split_steps - steps0) / row_n))) if row_n else 1
    kinds = {}
    for k, name in ((0, "row_pass"), (1, "col_pass"), (2, "detect"), (3, "mid_pass")):
        t, cnt = sim.timing(k)
        if cnt or k < 3:
            kinds[name] = {"ms_total": t, "launches": cnt, "ms_avg": t / cnt if cnt else None}
    sim.set_timing(False)
    passes = [k for k in ("row_pass", "col_pass", "mid_pass") if k in kinds and kinds[k]["launches"]]
    dom = max(passes, key=lambda k: kinds[k]["ms_total"])
    avg_ms = kinds[dom]["ms_avg"]
    algo_bytes = 2.0 * n * s_bytes * per_launch  # read + write of the fields per pass launch
    peak, peak_kind = measured_peak_hbm()
    achieved = algo_bytes / (avg_ms * 1e-3) / 1e9
    for k in passes:
        kinds[k]["GBps"] = algo_bytes / (kinds[k]["ms_avg"] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_launch": algo_bytes,
                "kernels": kinds}
    roofline["traffic"], roofline["traffic_source"] = ncu_traffic(dom, args.dtype, int(round(math.log2(n))))
    if roofline["traffic"] is not None and per_launch > 1:
        roofline["traffic"] *= per_launch
        roofline["traffic_source"] += f", times the {per_launch} fields of a batched launch"
    roofline["fields_per_launch"] = per_launch
    if not batch or len(gd["energies"]) == 1:
        sources_mode = "one source after the other"
    elif per_launch > 1:
        sources_mode = "lockstep batch per field length (one launch per pass for all its energies)"
    else:
        sources_mode = ("one source after the other (the engine's choice for this plan: its batched kernels "
                        "hold fewer CTAs per SM)")

    # ---- mixed precision against the complex128 run of the same step
    precision = None
    if args.compare_fp64 and args.dtype == "c8":
        ref = torch.zeros_like(acc)
        for g, a in zip(groups, accs):
            s16 = rsw.Simulation(g["case"], grids=g["grids"], dtype="c16")
            s16.reset()
            s16.run_sources([{"energy": e, "db_table": g["db"](e), "weight": w}
                             for e, w in zip(g["energies"], g["weights"])], source=g["case"]["source"])
            ref += s16.detected_device()
            s16.close()
        run_step()
        reduce_detector(ref)
        d = (acc - ref).double()
        precision = {"rel_l2": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(ref)),
                     "max_abs_over_max": float(d.abs().max() / ref.abs().max()),
                     "reference": "complex128 run of the same energies and phase steps"}

    # ---- CPU baseline (rank 0, N=1): oracle port on a bounded sample
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        k = 3
        lg = min(int(round(math.log2(n))), CPU_SAMPLE_MAX_LOGN)
        v, dt = cpu_split_steps(lg, args.dtype, k, 1)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{k} grating split steps (mask + FFT + transfer + iFFT) at N=2^{lg} "
                         f"{args.dtype}, FP64 numpy/scipy oracle, 1 thread, {dt:.1f} s"}

    gpu_base = None
    if rank == 0 and ws == 1 and not args.no_gpu_baseline:
        gpu_base = gpu_baseline(args, value, acc.cpu().numpy() if len(groups) == 1 else None)

    if rank == 0:
        cfg = {"workload": workload_name(args),
               "fields": [{"n": g["n"], "energies": len(g["energies"]), "split_steps": k}
                          for g, k in zip(groups, steps_g)],
               "phase_steps": sim0.nr_phase_steps,
               "split_steps_per_bench_step": int(sum(steps_g)) * ws,
               "l2_policy": "inputs larger than L2" if n * s_bytes > (126 << 20) else
                            "field smaller than L2 (no flush)",
               "parallelism": f"dp{ws} (energies sharded, detector all-reduce)",
               "sources": sources_mode,
               "schedule": {"autotuned": tuning} if tuning else "built-in"}
        if args.workload == "talbot_lau":
            cfg.update({"n": n, "energies_per_rank": len(gd["energies"]), "field_bytes": n * s_bytes,
                        "l2_policy": "inputs larger than L2 (field 2^24 c128 = 256 MiB)"
                        if n * s_bytes > (126 << 20) else "field smaller than L2 (no flush)"})
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.dtype == "c16" else "f32+f64",
            "data": "synthetic (seeded plane wave, tabulated gratings"
                    + (", seeded cracked-cylinder phantom)" if args.workload == "thick_sample" else ")"),
            "config": cfg,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": int(acc.numel()) * 8, "ms_per_step": e2e_ms},
            "gpu_launches": int(launches),
            "wall_s": t_wall,
            "clocks": clk,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "gpu_baseline": gpu_base,
        }
        if precision is not None:
            line["precision"] = precision
        print(json.dumps(line), flush=True)
    for g in groups:
        g["sim"].close()
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
