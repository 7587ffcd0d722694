#!/usr/bin/env python
"""Spin-flip attempts/s of the B200 annealer on the muon-tomography pyramid.

Workload (one step): the 306,328-bit, 75,594-ray pyramid QUBO (11.2 M bit-ray
entries, kappa = ln 999, lambda = 2), 16 branches annealed T 50 -> 1 over 200
sweeps then held 50 sweeps at T = 1 (the reference's default posterior
schedule, ising_recon.hpp:81-86), fp64 residual refresh every 50 sweeps; the
branches' fp64 energies and per-bit void fractions are computed on the device.
attempts per step = 16 * 250 * 306,328.

  value   -- device-resident problem, CUDA events on the solve's stream, L2
             flushed (256 MB write) before every timed step, outside the events;
  e2e     -- the public C ABI from pinned host buffers every step: upload and
             plan the problem, solve, read the void fractions back;
  --impl reference -- the reference's own CPU branch_fractions
             (oracle/_ref, compiled from the reference sources) on this host.

Multi-GPU: one process per GPU (torchrun); every rank solves its own copy of
the workload (branches are independent: weak scaling, no collective on the
data path); the timed region is bracketed by barriers and the slowest rank's
time is reported.
"""
import argparse
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

WORKLOAD = "muon-tomography pyramid: 306,328 bits, 75,594 rays, 16 branches, T 50->1 (200 sweeps) + 50 at T=1"
METRIC = "spin-flip attempts/s"
BRANCHES = 16
# DRAM bytes (read + write) per sweep of resid_lockstep_kernel from the
# committed ncu capture of a 10-sweep launch on the same pyramid and 16
# branches (profiles/resid_lockstep_pyramid.md): 1.924 GB + 6.3 MB over 10
# sweeps. The bit->ray structure streams from DRAM once per sweep, so the
# traffic of a full launch is this figure times its sweeps.
NCU_TRAFFIC_PER_SWEEP = (1.924285e9 + 6.321408e6) / 10


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu_id), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(a, R, sweeps, refresh, accepted):
    """Bytes one launch of the lockstep residual sweep must move: the residual
    form's per-sweep figure with a replica tile of 16 branches (one stream
    of the bit->ray CSR -- ray id + a, 8 B per entry -- serves 16 branches),
    each branch's residuals read and written once per sweep (rays x 2 x 4 B),
    its bits read and written (2 x 1/8 B each), the prior's neighbour lists
    once per tile (4 B per entry), plus every accepted flip's residual
    read-modify-write (entries of the bit x 2 x 4 B, from the device's
    accept count, at the mean entries per bit) and the fp64 refreshes
    (ray-major CSR, 8 B per entry, once per tile)."""
    nnz = int(a["ray"].size)
    n = int(a["row_ptr"].size - 1)
    rays = int(a["d"].size)
    nbr = int(a["nbr"].size)
    tiles = (R + 15) // 16
    per_sweep = nnz * 8 * tiles + R * (rays * 2 * 4 + n * 2 / 8) + nbr * 4 * tiles
    refreshes = (sweeps - 1) // refresh if refresh > 0 else 0
    return per_sweep * sweeps + refreshes * tiles * nnz * 8 + accepted * (nnz / n) * 2 * 4


def cpu_baseline(a, sched, threads, branches):
    """The reference's branch_fractions (oracle/_ref) on a bounded sample."""
    from oracle import oracle as O
    n = int(a["row_ptr"].size - 1)
    if O.ref_available():
        rp = O.RefProblem(a)
        _, _, wall = rp.branch_fractions(sched.t_hot, sched.t_cold, sched.anneal_sweeps, sched.hold_sweeps,
                                         branches, threads, 0, keep=False)
        kind = "reference"
    else:
        from concurrent.futures import ThreadPoolExecutor
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda b: O.anneal_branch(a, sched.t_hot, sched.t_cold, sched.anneal_sweeps,
                                                  sched.hold_sweeps, b + 1), range(branches)))
        wall = time.perf_counter() - t0
        kind = "port"
    attempts = branches * (sched.anneal_sweeps + sched.hold_sweeps) * n
    return attempts / wall, wall, kind


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from qublar_b200 import Schedule, synth
    a = synth.tomography()
    threads = os.cpu_count() or 1
    # each step: the full 306,328-bit problem, min(16, cores) branches of a
    # 25-sweep sample of the schedule (T 50 -> 1 over 20 sweeps, 5 held)
    branches = min(BRANCHES, threads)
    sample = Schedule(50.0, 1.0, 20, 5, 0)
    rates = []
    for k in range(args.warmup + args.steps):
        rate, wall, kind = cpu_baseline(a, sample, threads, branches)
        if k >= args.warmup:
            rates.append(rate)
    value = statistics.mean(rates)
    n = int(a["row_ptr"].size - 1)
    ms = branches * sample.sweeps * n / value * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "attempts/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "bits": n, "rays": int(a["d"].size), "entries": int(a["ray"].size)},
            "cpu_baseline": {"value": value, "unit": "attempts/s", "cores": threads, "kind": kind,
                             "sample": f"{branches} branches x 25-sweep sample of the schedule per step, "
                                       f"full 306,328-bit problem, {threads} threads"},
            "e2e": {"value": value, "unit": "attempts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweeps", type=int, default=250,
                    help="schedule length (default 250 = 200 + 50, the benchmark); shorter runs are for profiling only")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    from qublar_b200 import ResidualProblem, Schedule, synth

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    stream = torch.cuda.current_stream()
    a = synth.tomography()
    n = int(a["row_ptr"].size - 1)
    sched = Schedule()   # 50 -> 1, 200 + 50, refresh 50
    if args.sweeps != 250:
        hold = args.sweeps // 5
        sched = Schedule(50.0, 1.0, args.sweeps - hold, hold, 50)
    P = ResidualProblem.from_arrays(a, device=local, stream=stream)
    pinfo = P.info()
    attempts_step = BRANCHES * sched.sweeps * n
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        r = P.solve(sched, BRANCHES, stream=stream)
        r.info()
        r.close()

    sampler = ClockSampler(local) if rank == 0 else None
    barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    results = []
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        results.append(P.solve(sched, BRANCHES, stream=stream))
        ends[k].record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop() if sampler else None
    total_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    infos = [r.info() for r in results]
    anneal_ms = statistics.mean(i.anneal_ms for i in infos)
    accepted = statistics.mean(i.accepted for i in infos)
    launches = sum(i.launches for i in infos)
    drift = max(i.max_drift for i in infos)
    for r in results:
        r.close()
    total_ms = max_over_ranks(total_ms)
    value = world * attempts_step * args.steps / (total_ms / 1e3)

    # e2e through the C ABI from pinned host memory
    pinned = {}
    for k, v in a.items():
        if isinstance(v, np.ndarray):
            t = torch.empty(v.shape, dtype=getattr(torch, str(v.dtype)), pin_memory=True)
            t.numpy()[...] = v
            pinned[k] = t.numpy()
        else:
            pinned[k] = v
    h2d = sum(v.nbytes for v in pinned.values() if isinstance(v, np.ndarray))
    d2h = n * 4
    e2e_s = [float("nan")]
    if args.e2e_steps > 0:
        e2e_s = []
    barrier()
    for k in range(args.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Q = ResidualProblem.from_arrays(pinned, device=local, stream=stream)
        r = Q.solve(sched, BRANCHES, stream=stream)
        p = r.marginals()
        e2e_s.append(time.perf_counter() - t0)
        r.close()
        Q.close()
        assert p.shape == (n,)
    barrier()
    e2e_mean = max_over_ranks(statistics.mean(e2e_s))
    e2e_value = world * attempts_step / e2e_mean

    hbm, peak_kind = peaks()
    alg = algorithmic_bytes(a, BRANCHES, sched.sweeps, sched.refresh_sweeps, accepted)
    achieved = alg / (anneal_ms / 1e3) / 1e9
    traffic = None
    if NCU_TRAFFIC_PER_SWEEP is not None:
        traffic = NCU_TRAFFIC_PER_SWEEP * sched.sweeps
    line = {
        "metric": METRIC, "value": value, "unit": "attempts/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "bits": n, "rays": int(a["d"].size), "entries": int(a["ray"].size),
                   "branches": BRANCHES, "sweeps": sched.sweeps, "colours": int(pinfo.n_colours),
                   "l2": "flushed (256 MB write) before every timed step; problem footprint "
                         f"{pinfo.device_bytes / 2**20:.0f} MiB", "parallelism": f"{world} independent replicas"},
        "e2e": {"value": e2e_value, "unit": "attempts/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": d2h,
                "s_per_step": e2e_mean},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "traffic": traffic, "kernel": "resid_lockstep_kernel",
                     "kernel_ms": anneal_ms, "algorithmic_bytes": alg, "accepted_flips": accepted},
        "max_residual_drift": drift,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        branches = min(BRANCHES, threads)
        rate, wall, kind = cpu_baseline(a, sched, threads, branches)
        line["cpu_baseline"] = {"value": rate, "unit": "attempts/s", "cores": threads, "kind": kind,
                                "sample": f"{branches} of 16 branches, the full 250-sweep schedule, "
                                          f"{threads} threads, {wall:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
