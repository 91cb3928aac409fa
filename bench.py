"""Benchmark: join output tuples/s of the triangle query on one R-MAT graph.

Workload (the triangle configuration): R(a,b) S(b,c) T(a,c) over one
synthetic R-MAT graph, scale 20 (2^20 vertices), 2^24 generated edges,
quadrant probabilities (0.57, 0.19, 0.19, 0.05), seed 20; self-loops and
duplicates removed, edges oriented u<v, rows shuffled.  One step is one
ALFTJ DFS query over the edge relation resident in HBM: trie (CSR) build by
the radix sort, then the leapfrog intersection, returning count and
checksum.  The unit of work is one output tuple (one triangle).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--algo DFS|BFS|AMHJ]

* value: tuples/s with the input resident on the device (whole job: sum of
  the ranks' tuples / max over ranks of the timed K steps).
* e2e: the same metric through the C ABI with host buffers: every step copies
  the edge relation from pinned host memory to the device, runs the query and
  reads the 16-byte (count, checksum) result back.
* roofline: the intersection kernel, HBM-bound; algorithmic bytes per launch
  = every edge read once (8 B) + two row-pointer pairs per edge (32 B) + the
  shorter child list of every edge read once (4 B x min(d+(a), d+(b))).
* cpu_baseline: the CPU oracle's triangle restatement on all host cores over
  the full workload (the reference has no CPU triangle implementation; its
  MHJ-CPU hard-codes a single-key compare that is wrong for cyclic queries).

With N > 1 (torchrun) every rank runs its own independent instance of the
workload (graph seed 20 + rank): per-GPU work is fixed, no data-path
collective; the ranks' counts are summed once after timing.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

SCALE, NEDGES, RMAT_ABC, SEED = 20, 1 << 24, (0.57, 0.19, 0.19), 20
METRIC = "join output tuples/sec"
L2_FLUSH_BYTES = 256 << 20


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload(rank: int):
    from accmultiwayjoins_b200 import data
    return data.rmat(SCALE, NEDGES, *RMAT_ABC, seed=SEED + rank)


def algorithmic_bytes(src, dst) -> int:
    deg = np.bincount(src, minlength=1 << SCALE).astype(np.int64)
    shorter = np.minimum(deg[src], deg[dst])
    return int(src.shape[0]) * (8 + 32) + 4 * int(shorter.sum())


def run_reference(args, rank, world):
    """CPU arm: the oracle's triangle restatement on all host threads."""
    if rank != 0:
        return
    from oracle import oracle as O
    src, dst = workload(0)
    cores = os.cpu_count() or 1
    times = []
    count = 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        count, chk = O.triangle(src, dst, nthreads=cores)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    sec = sum(times) / len(times)
    value = count / sec
    line = {
        "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded R-MAT)", "impl": "reference",
        "config": {"workload": f"triangle R(a,b)S(b,c)T(a,c), R-MAT scale {SCALE}, {NEDGES} edges "
                               f"(0.57,0.19,0.19,0.05), seed {SEED}", "edges_after_cleaning": int(src.shape[0]),
                   "algo": "CPU merge-intersection restatement", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "tuples/s", "cores": cores, "kind": "port",
                         "sample": "the full workload per step"},
        "e2e": {"value": value, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import ctypes as C
    from accmultiwayjoins_b200 import Context, _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    src, dst = workload(rank)
    E = int(src.shape[0])
    stream = torch.cuda.current_stream(dev)
    ctx = Context(local_rank)
    lib = L.load()
    L.check(lib.amj_ctx_set_stream(ctx.handle, C.c_void_p(stream.cuda_stream)), "set_stream")
    rel = ctx.relation([torch.from_numpy(src).to(dev), torch.from_numpy(dst).to(dev)], [0, 1])
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    algo = args.algo

    def step():
        if algo == "AMHJ":
            return ctx.amhj("TRI", [rel], ws=1)
        return ctx.lftj([rel], algo=algo, ws=1)

    for _ in range(args.warmup):
        r = step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    launches0 = C.c_uint64()
    L.check(lib.amj_ctx_launch_count(ctx.handle, C.byref(launches0)))
    torch.cuda.synchronize()
    evs = []
    probe_ms = []
    build_ms = []
    count = 0
    t_wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()  # L2 flush (256 MB) outside the timed events
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = step()
        b.record(stream)
        evs.append((a, b))
        probe_ms.append(r.probe_ms)
        build_ms.append(r.build_ms)
        count = r.count
        checksum = r.checksum
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    launches1 = C.c_uint64()
    L.check(lib.amj_ctx_launch_count(ctx.handle, C.byref(launches1)))
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ms = sum(step_ms) / len(step_ms)
    # e2e through the C ABI with host buffers
    hs = torch.from_numpy(src).pin_memory()
    hd = torch.from_numpy(dst).pin_memory()
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hr = ctx.relation([hs.numpy(), hd.numpy()], [0, 1])
        if algo == "AMHJ":
            rr = ctx.amhj("TRI", [hr], ws=1)
        else:
            rr = ctx.lftj([hr], algo=algo, ws=1)
        assert (rr.count, rr.checksum) == (count, checksum)
        hr.release()
        dt = (time.perf_counter() - t0) * 1e3
        if i >= args.warmup:
            e2e_ms.append(dt)
    clocks = sampler.stop()
    e2e_mean = sum(e2e_ms) / len(e2e_ms)

    # whole job: max time over ranks, tuples summed over ranks
    tot_count, max_ms, max_e2e = count, ms, e2e_mean
    if world > 1:
        t = torch.tensor([float(count), ms, e2e_mean], dtype=torch.float64, device=dev)
        cnt = torch.tensor([count], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(cnt)
        mx = t.clone()
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        tot_count, max_ms, max_e2e = int(cnt.item()), mx[1].item(), mx[2].item()
    if rank != 0:
        return
    hbm, peak_kind = peaks()
    alg_bytes = algorithmic_bytes(src, dst)
    kern_ms = sum(probe_ms) / len(probe_ms)
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9 if algo == "DFS" else None
    line = {
        "metric": METRIC, "value": tot_count / (max_ms * 1e-3), "unit": "tuples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded R-MAT)",
        "config": {"workload": f"triangle R(a,b)S(b,c)T(a,c), R-MAT scale {SCALE}, {NEDGES} edges "
                               f"(0.57,0.19,0.19,0.05), seed {SEED}+rank; ALFTJ-{algo} count+checksum incl. trie build",
                   "edges_after_cleaning": E, "triangles_per_rank": count,
                   "l2": "flushed between steps (256 MB write)", "parallelism": f"independent instance per GPU x{world}"},
        "e2e": {"value": tot_count / (max_e2e * 1e-3), "unit": "tuples/s", "h2d_bytes_per_step": 8 * E,
                "d2h_bytes_per_step": 16, "ms_per_step": max_e2e},
        "gpu_launches": int(launches1.value - launches0.value),
        "phase_ms": {"build": sum(build_ms) / len(build_ms), "intersect": kern_ms},
        "clocks": clocks,
        "wall_s_timed": t_wall,
    }
    if achieved is not None:
        line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                            "frac": achieved / hbm, "traffic": None, "peak_kind": peak_kind,
                            "kernel": "lftj_tri_dfs_kernel", "alg_bytes_per_launch": alg_bytes}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        c_cnt, c_chk = O.triangle(src, dst, nthreads=cores)
        sec = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": c_cnt / sec, "unit": "tuples/s", "cores": cores, "kind": "port",
                                "sample": "the full workload once (oracle triangle restatement)",
                                "matches_gpu": bool((c_cnt, c_chk) == (count, checksum))}
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--algo", default="DFS", choices=["DFS", "BFS", "AMHJ"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
