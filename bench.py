"""Benchmark: join output tuples/s of the triangle query on one R-MAT graph.

Workload (the triangle configuration): R(a,b) S(b,c) T(a,c) over one
synthetic R-MAT graph, scale 20 (2^20 vertices), 2^24 generated edges,
quadrant probabilities (0.57, 0.19, 0.19, 0.05), seed 20; self-loops and
duplicates removed, edges oriented u<v, rows shuffled.  One step is one
ALFTJ DFS query over the edge relation resident in HBM: trie (CSR) build by
the radix sort, then the leapfrog intersection, returning count and
checksum.  The unit of work is one output tuple (one triangle).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--algo DFS|BFS|AMHJ] [--scale S]
                  [--workload triangle|chain|four|star|batch|serve|ooc] [--no-configs]

--scale S runs the same workload on a smaller R-MAT graph (2^S vertices,
2^(S+4) edges), for profiling.  --workload chain runs the 3-way chain join
R1(a,b) R2(b,c) R3(c,d) (3 x 1M rows, keys uniform in [0, 2^18), seeds 1-3)
through AMHJ (count + checksum, hash builds included).  --workload star
runs the 4-way star (fact 60M rows x 4 Zipf(1.1) keys, dims 1M/200K/100K/10K)
through AMHJ the same way; --workload four the skewed 4-clique (R-MAT
scale 22).  --plan thread_per_row|pairwise runs the chain or star through
the reference's baseline plans instead of the operator; --plan frontier
through the operator's frontier-DFS kernel instead of its flat kernels.  --workload batch
runs 512 heterogeneous queries as one batch (autotuned, CUDA-graph replay)
and reports, beside its tuples/s, the one-query-per-call tuples/s on the
same queries and p50/p99 latencies of both forms.

* value: tuples/s with the input resident on the device (whole job: sum of
  the ranks' tuples / max over ranks of the timed K steps).
* e2e: the same metric through the C ABI with host buffers: every step copies
  the relations from pinned host memory to the device, runs the query and
  reads the 16-byte (count, checksum) result back.
* roofline: the intersection kernels (triangle) or the probe kernel (chain),
  timed with CUDA events inside the library; algorithmic bytes per launch
  as documented below; traffic from the committed ncu capture.
* configs (default triangle run, one GPU): the chain, skewed 4-clique (AMHJ
  FOUR ws=1 fib=1, R-MAT scale 22), star and batched configurations measured
  in the same run, each with its own value, e2e and CPU figure; the batched
  record carries batched vs one-query-per-call tuples/s and p50/p99
  latencies.
* cpu_baseline and --impl reference: the reference's MHJ-CPU
  (MHJ-CPU/MHJ.cpp) compiled from its sources into oracle/_ref, on all host
  cores: as shipped for chains and stars; its multi-key probe branch for the
  triangle and the 4-clique, over the degree-ordered copy of the graph,
  renamed back (see RefTriangle), one bounded probe slice per step.  The
  reference arm generates its inputs with the oracle's generators and never
  loads the product library.

With N > 1 (torchrun) every rank runs its own independent instance of the
workload (seed offset by rank): per-GPU work is fixed, no data-path
collective; the ranks' counts are summed once after timing.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

SCALE, RMAT_ABC, SEED = 20, (0.57, 0.19, 0.19), 20
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


# ------------------------------------------------------------------ workloads

class Triangle:
    def __init__(self, args, rank):
        from accmultiwayjoins_b200 import data
        self.scale = args.scale
        self.nedges = 1 << (self.scale + 4)
        self.algo = args.algo
        self.src, self.dst = data.rmat(self.scale, self.nedges, *RMAT_ABC, seed=SEED + rank)
        self.E = int(self.src.shape[0])
        self.h2d = 8 * self.E

    def describe(self, rank_note):
        return self.describe_static(self.scale, self.algo, rank_note)

    @staticmethod
    def describe_static(scale, algo, rank_note=""):
        return (f"triangle R(a,b)S(b,c)T(a,c), R-MAT scale {scale}, {1 << (scale + 4)} edges "
                f"(0.57,0.19,0.19,0.05), seed {SEED}{rank_note}; "
                f"{'AMHJ TRI' if algo == 'AMHJ' else 'ALFTJ-' + algo} count+checksum incl. index build")

    def device_relations(self, ctx, dev):
        import torch
        return [ctx.relation([torch.from_numpy(self.src).to(dev), torch.from_numpy(self.dst).to(dev)], [0, 1])]

    def host_relations(self, ctx, pinned):
        return [ctx.relation([pinned[0], pinned[1]], [0, 1])]

    def host_columns(self):
        return [self.src, self.dst]

    def run(self, ctx, rels):
        if self.algo == "AMHJ":
            return ctx.amhj("TRI", rels, ws=1)
        return ctx.lftj(rels, algo=self.algo, ws=1)

    def algorithmic_bytes(self):
        """DFS and AMHJ TRI (the wedge kernel over the degree-ranked copy):
        per edge its (b, entry) item (8 B), the level-0 value a (4 B) and the
        end of a's child range (8 B); per tested value 4 B, sum over a of
        C(d+(a), 2) values with d+ the out-degree in (degree, id) order.  BFS:
        every edge once (8 B), two row-pointer pairs (32 B) and the shorter
        child list of the edge once (4 B each), in the relation's order."""
        V = 1 << self.scale
        src, dst = self.src.astype(np.int64), self.dst.astype(np.int64)
        if self.algo in ("DFS", "AMHJ"):
            deg = np.bincount(src, minlength=V) + np.bincount(dst, minlength=V)
            key_s, key_d = deg[src] * V + src, deg[dst] * V + dst
            lo = np.where(key_s < key_d, src, dst)
            dplus = np.bincount(lo, minlength=V).astype(np.int64)
            return self.E * (8 + 4 + 8) + 4 * int((dplus * (dplus - 1) // 2).sum())
        deg = np.bincount(src, minlength=V).astype(np.int64)
        shorter = np.minimum(deg[src], deg[dst])
        return self.E * (8 + 32) + 4 * int(shorter.sum())

    def kernel_name(self):
        return ("lftj_tri_wedge_kernel (intersection)" if self.algo in ("DFS", "AMHJ")
                else "lftj_tri_bfs kernels (intersection)")

    def cpu_baseline(self):
        """The reference's MHJ-CPU multi-key probe on a bounded sample of
        this workload (RefTriangle), about 15 s of CPU time."""
        ref = RefTriangle(self.scale, self.nedges, SEED)
        return ref.sample_until(15.0)


class RefTriangle:
    """The reference's CPU implementation of the triangle workload: MHJ-CPU
    (MHJ-CPU/MHJ.cpp TBJ) with its multi-key probe branch (MHJ.cpp:64-90,
    :205-245), compiled from the reference sources into
    oracle/_ref/libmhjref_mk.so, over the TRI attribute pattern
    (MHJ-GPU/exec_AMHJ.cu:32-49).  It joins the graph's (degree, id)-ranked
    copy and renames the results back (the same triangles; on the relation as
    given its probe does about 24x more work on this graph).  One sample is
    one probe slice: 1/SLICES of the probe relation's rows against the whole
    build relations; TBJ's own partitioning of the build relations is part
    of every timed call.  Inputs come from the oracle's generators, so this
    process never loads the product library."""

    SLICES = 64

    def __init__(self, scale, nedges, seed):
        from oracle import oracle as O
        self.O = O
        s, d = O.gen_rmat(scale, nedges, *RMAT_ABC, seed=seed)
        self.E = int(s.shape[0])
        self.s2, self.d2, self.rank_to_id = O.degree_ordered_copy(s, d)
        self.cores = os.cpu_count() or 1
        self.next = 0
        self.kind = "reference" if O.ref_available(multi_key=True) else "port"

    def step(self):
        """One slice, the next in turn: (tuples, seconds in TBJ)."""
        i = self.next % self.SLICES
        self.next += 1
        lo, hi = i * self.E // self.SLICES, (i + 1) * self.E // self.SLICES
        probe = ([self.s2[lo:hi], self.d2[lo:hi]], [0, 1])
        rels = [probe, ([self.s2, self.d2], [1, 2]), ([self.s2, self.d2], [0, 2])]
        if self.kind == "reference":
            cnt, _, sec = self.O.mhj_reference(rels, nthreads=self.cores, multi_key=True, relabel=self.rank_to_id)
        else:
            t0 = time.perf_counter()
            cnt, _ = self.O.mhj(rels, nthreads=self.cores)
            sec = time.perf_counter() - t0
        return cnt, sec

    def describe(self):
        what = ("reference MHJ-CPU multi-key probe (oracle/_ref/libmhjref_mk.so)" if self.kind == "reference"
                else "the oracle's multi-way join restatement (reference sources absent)")
        return (f"{what} on the TRI pattern over the degree-ordered copy, one 1/{self.SLICES} probe slice per "
                f"sample (slices in turn), whole build relations, TBJ call timed")

    def sample_until(self, budget_s):
        tuples, secs, n = 0, 0.0, 0
        while secs < budget_s and n < self.SLICES:
            c, t = self.step()
            tuples, secs, n = tuples + c, secs + t, n + 1
        return tuples, None, secs, self.cores, self.kind, f"{n} slices: " + self.describe()


class Clique4:
    """The skewed 4-clique over an R-MAT graph of scale S (2^S vertices,
    2^(S+4) edges, quadrant probabilities 0.6/0.15/0.15/0.1), cleaned as the
    triangle graph; the full size is scale 22 (64 Mi edges).  --algo AMHJ
    runs the configured operator, AMHJ FOUR with ws=1 fib=1, whose last three
    levels (the fourth vertex, looked up by pair keys) are answered by the
    triangle matrices of the degree-ranked copy; the default runs the ALFTJ
    4-clique, which gives the same count and checksum."""

    def __init__(self, args, rank):
        from accmultiwayjoins_b200 import data
        self.scale = args.scale
        self.algo = args.algo
        self.src, self.dst = data.rmat(self.scale, 1 << (self.scale + 4), 0.6, 0.15, 0.15, seed=22 + rank)
        self.E = int(self.src.shape[0])
        self.h2d = 8 * self.E

    def describe(self, rank_note):
        return self.describe_static(self.scale, self.algo, rank_note)

    @staticmethod
    def describe_static(scale, algo, rank_note=""):
        op = ("AMHJ FOUR (ws=1 fib=1; pair-key levels by triangle matrices), index build" if algo == "AMHJ"
              else "ALFTJ 4-clique (DFS), trie build")
        return (f"4-clique, R-MAT scale {scale}, {1 << (scale + 4)} edges "
                f"(0.6,0.15,0.15,0.1), seed 22{rank_note}; {op} included, count+checksum")

    def device_relations(self, ctx, dev):
        import torch
        return [ctx.relation([torch.from_numpy(self.src).to(dev), torch.from_numpy(self.dst).to(dev)], [0, 1])]

    def host_relations(self, ctx, pinned):
        return [ctx.relation([pinned[0], pinned[1]], [0, 1])]

    def host_columns(self):
        return [self.src, self.dst]

    def run(self, ctx, rels):
        if self.algo == "AMHJ":
            return ctx.amhj("FOUR", rels, ws=1, fib=1)
        return ctx.lftj(rels, algo="DFS", clique4=True)

    def algorithmic_bytes(self):
        return None

    def kernel_name(self):
        return "lftj_clique4_matrix_kernel"

    def cpu_baseline(self):
        """The reference's MHJ-CPU multi-key probe on the FOUR pattern over a
        scale-14 graph of the same generator (RefClique4)."""
        return RefClique4().sample_until(15.0)


class RefClique4:
    """The reference's CPU implementation of the 4-clique: MHJ-CPU's
    multi-key probe (oracle/_ref/libmhjref_mk.so) on the FOUR attribute
    pattern (MHJ-GPU/exec_AMHJ.cu:50-69) over the degree-ordered copy of an
    R-MAT scale-14 graph of the configured generator (2^18 edges,
    0.6/0.15/0.15/0.1, seed 22; the scale-22 graph's 9.4e10 4-cliques would
    not fit the reference's in-memory result chunks), one 1/SLICES probe
    slice per sample."""

    SLICES = 16

    def __init__(self):
        from oracle import oracle as O
        self.O = O
        s, d = O.gen_rmat(14, 1 << 18, 0.6, 0.15, 0.15, seed=22)
        self.E = int(s.shape[0])
        self.s2, self.d2, self.rank_to_id = O.degree_ordered_copy(s, d)
        self.cores = os.cpu_count() or 1
        self.next = 0
        self.kind = "reference" if O.ref_available(multi_key=True) else "port"

    def step(self):
        i = self.next % self.SLICES
        self.next += 1
        lo, hi = i * self.E // self.SLICES, (i + 1) * self.E // self.SLICES
        rels = self.O.four_relations(self.s2, self.d2)
        rels[0] = ([self.s2[lo:hi], self.d2[lo:hi]], [0, 1])
        if self.kind == "reference":
            cnt, _, sec = self.O.mhj_reference(rels, nthreads=self.cores, multi_key=True, relabel=self.rank_to_id)
        else:
            t0 = time.perf_counter()
            cnt, _ = self.O.mhj(rels, nthreads=self.cores)
            sec = time.perf_counter() - t0
        return cnt, sec

    def describe(self):
        return (f"reference MHJ-CPU multi-key probe, FOUR pattern, R-MAT scale 14 (2^18 edges, seed 22) "
                f"degree-ordered copy, one 1/{self.SLICES} probe slice per sample, TBJ call timed")

    def sample_until(self, budget_s):
        tuples, secs, n = 0, 0.0, 0
        while secs < budget_s and n < self.SLICES:
            c, t = self.step()
            tuples, secs, n = tuples + c, secs + t, n + 1
        return tuples, None, secs, self.cores, self.kind, f"{n} slices: " + self.describe()


def plan_note(plan):
    """The workload text of a baseline plan run in place of the operator."""
    return {"multiway": "", "thread_per_row": " (baseline plan: one thread per probe row, MHJ.cuh)",
            "pairwise": " (baseline plan: 2-relation joins with materialised intermediates, exec_PW.cu)",
            "hash": "", "frontier": " (the operator's frontier-DFS kernel, no flat kernel)"}[plan]


class Chain:
    B = 1 << 19   # buckets = floorPow2(1e6)

    def __init__(self, args, rank, gen=None):
        from accmultiwayjoins_b200 import data
        self.rels = data.chain_relations(1_000_000, 1 << 18, 3, seed=1 + 3 * rank, gen=gen)
        self.h2d = sum(4 * len(c[0]) * len(c) for c, _ in self.rels)
        self.plan = getattr(args, "plan", "multiway")

    def describe(self, rank_note):
        return ("3-way chain R1(a,b)R2(b,c)R3(c,d), 3 x 1M rows, keys U[0,2^18), seeds 1,2,3" + rank_note +
                "; AMHJ NORMAL count+checksum incl. hash builds" + plan_note(self.plan))

    def device_relations(self, ctx, dev):
        import torch
        return [ctx.relation([torch.from_numpy(c).to(dev) for c in cols], a) for cols, a in self.rels]

    def host_relations(self, ctx, pinned):
        out, i = [], 0
        for cols, a in self.rels:
            out.append(ctx.relation(pinned[i:i + len(cols)], a))
            i += len(cols)
        return out

    def host_columns(self):
        return [c for cols, _ in self.rels for c in cols]

    def run(self, ctx, rels):
        return ctx.amhj("NORMAL", rels, plan=self.plan)

    def algorithmic_bytes(self):
        """B_probe of the AMHJ count probe: the probe columns (4 B each a
        row) and, for every lookup, its bucket bounds (8 B), the keys of its
        bucket scanned (4 B each) and per match a row id and the gathered
        payload (8 B); a lookup at level 0 per probe row, at level 1 per
        level-0 match.  Buckets are floorPow2(rows) wide, as built."""
        if self.plan not in ("multiway", "frontier"):
            return None   # a baseline plan: its kernels are not the operator's
        (p0, p1), _ = self.rels[0]
        (b0, b1), _ = self.rels[1]
        (c0, _), _ = self.rels[2]
        m = self.B - 1
        n1 = np.bincount(b0 & m, minlength=self.B).astype(np.int64)
        n2 = np.bincount(c0 & m, minlength=self.B).astype(np.int64)
        k1 = np.bincount(b0, minlength=1 << 18).astype(np.int64)   # level-0 matches of a key
        k2 = np.bincount(c0, minlength=1 << 18).astype(np.int64)   # level-1 matches of a key
        per1 = 8 + 4 * n2[b1 & m] + 8 * k2[b1]                     # the level-1 lookup of each level-0 row
        behind = np.zeros(1 << 18, np.int64)
        np.add.at(behind, b0, per1)                                # level-1 bytes behind a level-0 key
        tot = 8 * len(p0) + int((8 + 4 * n1[p1 & m] + 8 * k1[p1]).sum()) + int(behind[p1].sum())
        return tot

    def lookups_per_launch(self):
        """Bucket lookups: one per probe row and one per level-0 match."""
        (p0, p1), _ = self.rels[0]
        (b0, _), _ = self.rels[1]
        return len(p0) + int(np.bincount(b0, minlength=1 << 18)[p1].sum())

    def kernel_name(self):
        return "amhj_probe_kernel (count pass)" if self.plan == "frontier" else "amhj_chain_canon_kernel"

    def cpu_baseline(self):
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        if O.ref_available():
            cnt, chk, sec = O.mhj_reference(self.rels, nthreads=cores)
            return cnt, chk, sec, cores, "reference", "the full workload once (reference MHJ-CPU, TBJ call timed)"
        t0 = time.perf_counter()
        cnt, chk = O.mhj(self.rels, nthreads=cores)
        return cnt, chk, time.perf_counter() - t0, cores, "port", "the full workload once (oracle restatement)"


class Star:
    """The 4-way star: a fact table of 60M rows of four Zipf(1.1) foreign
    keys into dimensions of 1M, 200K, 100K and 10K rows (unique key, uniform
    payload), seed 3; AMHJ NORMAL count+checksum including the four hash
    builds.  The probe is the flat star path: one thread per fact row, every
    dimension's lookup in flight together."""
    DIMS = (1_000_000, 200_000, 100_000, 10_000)

    def __init__(self, args, rank, gen=None):
        from accmultiwayjoins_b200 import data
        self.rows = args.star_rows
        fact, dims = data.star_relations(self.rows, list(self.DIMS), theta=1.1, seed=3 + rank, gen=gen)
        self.rels = [fact] + dims
        self.h2d = sum(4 * len(c[0]) * len(c) for c, _ in self.rels)
        self.plan = getattr(args, "plan", "multiway")

    def describe(self, rank_note):
        return (f"4-way star, fact {self.rows} rows x 4 Zipf(1.1) foreign keys, dims 1M/200K/100K/10K "
                f"(key, payload), seed 3{rank_note}; AMHJ NORMAL count+checksum incl. hash builds"
                + plan_note(self.plan))

    device_relations = Chain.device_relations
    host_relations = Chain.host_relations
    host_columns = Chain.host_columns
    run = Chain.run

    def algorithmic_bytes(self):
        """B_probe of the AMHJ count probe: the fact row's four keys (16 B)
        and, for each dimension lookup, its bucket bounds (8 B), the keys of
        its bucket scanned (4 B each) and per match a row id and the gathered
        payload (8 B), with floorPow2(rows) buckets as built.  The lookups are
        served by L1 and L2 (the dimensions and their bucket heads are
        L2-resident), so the fraction of HBM can exceed 1."""
        if self.plan not in ("multiway", "frontier"):
            return None   # a baseline plan: its kernels are not the operator's
        fact_cols = self.rels[0][0]
        tot = len(fact_cols[0]) * 16
        for j, (cols, _) in enumerate(self.rels[1:]):
            n = len(cols[0])
            B = 1 << (n.bit_length() - 1)
            per = np.bincount(cols[0] & (B - 1), minlength=B).astype(np.int64)
            f = fact_cols[j]
            hits = np.bincount(cols[0], minlength=int(max(n, f.max() + 1))).astype(np.int64)
            tot += 8 * len(f) + 4 * int(per[f & (B - 1)].sum()) + 8 * int(hits[f].sum())
        return tot

    def lookups_per_launch(self):
        """Random line lookups of the probe: one bucket head per dimension
        and fact row."""
        return len(self.rels[0][0][0]) * (len(self.rels) - 1)

    def kernel_name(self):
        return "amhj_probe_kernel (count pass)" if self.plan == "frontier" else "amhj_star_canon_kernel"

    def cpu_baseline(self, sample_rows=12_000_000):
        """The reference MHJ-CPU over a bounded sample of the fact table (its
        first rows, all dimensions), scaled to tuples/s."""
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        n = min(self.rows, sample_rows)
        (fc, fa) = self.rels[0]
        rels = [([c[:n] for c in fc], fa)] + self.rels[1:]
        if O.ref_available():
            cnt, _, sec = O.mhj_reference(rels, nthreads=cores)
            kind = "reference"
        else:
            t0 = time.perf_counter()
            cnt, _ = O.mhj(rels, nthreads=cores)
            sec, kind = time.perf_counter() - t0, "port"
        return cnt, None, sec, cores, kind, f"the first {n} fact rows with all four dimensions"


class BatchMix:
    """The batched workload: a heterogeneous mix of chain / star / triangle
    queries (sizes log-uniform 10K-4M rows, key domains 2^12-2^24, uniform or
    Zipf theta in [0.5, 1.5]; accmultiwayjoins_b200.data.query_mix, seed 4)
    run as one amj_batch: one build pass and one persistent probe launch,
    captured once into a CUDA graph and replayed every step."""

    def __init__(self, args, rank, gen=None):
        from accmultiwayjoins_b200 import data
        t0 = time.perf_counter()
        self.queries = list(data.query_mix(args.queries, seed=4 + 1000 * rank, min_rows=args.min_rows,
                                           max_rows=args.max_rows, gen=gen))
        self.gen_s = time.perf_counter() - t0
        self.rows = sum(len(cols[0]) for q in self.queries for cols, _ in q["rels"])
        self.h2d = sum(4 * len(c) for q in self.queries for cols, _ in q["rels"] for c in cols)

    def describe(self, rank_note):
        shapes = {}
        for q in self.queries:
            shapes[q["shape"]] = shapes.get(q["shape"], 0) + 1
        return (f"batched: {len(self.queries)} heterogeneous queries {shapes}, {self.rows} relation rows "
                f"(log-uniform sizes in [{self.queries and min(len(c[0]) for q in self.queries for c, _ in q['rels'])}, "
                f"4M], key domains 2^12-2^24, uniform or Zipf theta in [0.5,1.5], seed 4{rank_note}); "
                f"one build pass + one persistent probe launch per step, CUDA graph replay")

    def cpu_sample(self, budget_s=15.0, start=0):
        """The reference MHJ-CPU on the queries from `start` on, one at a
        time, until budget_s of CPU time is spent: chains and stars of 3+
        relations through the shipped single-key probe, triangles through its
        multi-key probe over the degree-ordered copy.  Two-relation joins
        crash the reference's TBJ (one build table), so those run on the
        oracle's restatement."""
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        spent, tuples, n, kinds = 0.0, 0, 0, set()
        for j in range(len(self.queries)):
            q = self.queries[(start + j) % len(self.queries)]
            t0 = time.perf_counter()
            if q["qt"] == "TRI" and O.ref_available(multi_key=True):
                s2, d2, lab = O.degree_ordered_copy(*q["rels"][0][0])
                cnt, _, sec = O.mhj_reference(O.tri_relations(s2, d2), nthreads=cores, multi_key=True, relabel=lab)
                kinds.add("reference")
            elif q["qt"] == "NORMAL" and O.ref_available() and len(q["rels"]) >= 3:
                cnt, _, sec = O.mhj_reference(q["rels"], nthreads=cores)
                kinds.add("reference")
            else:
                rels = O.tri_relations(*q["rels"][0][0]) if q["qt"] == "TRI" else q["rels"]
                cnt, _ = O.mhj(rels, nthreads=cores)
                sec = time.perf_counter() - t0
                kinds.add("port")
            spent += sec
            tuples += cnt
            n += 1
            if spent >= budget_s:
                break
        kind = "reference" if kinds == {"reference"} else ("port" if kinds == {"port"} else "reference+port")
        sample = (f"{n} of {len(self.queries)} queries from query {start}, one query at a time (reference MHJ-CPU: "
                  f"single-key probe for chains and stars of 3+ relations, multi-key probe over the degree-ordered "
                  f"copy for triangles; two-relation joins on the oracle's restatement)")
        return tuples, spent, cores, kind, sample


def pct(xs, p):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(round(p / 100.0 * (len(xs) - 1))))]


def run_batch(args, rank, world, local_rank):
    line = batch_line(args, rank, world, local_rank)
    if line is not None:
        print(json.dumps(line), flush=True)


# the grid point the autotuner chose on the 512-query mix (load factor 0.5,
# block 128, task chunk 128), used where a run skips the tuner
TUNED_BATCH_POINT = (0.5, 128, 128)


def batch_line(args, rank, world, local_rank, fixed_point=None, cpu_budget=15.0):
    """The batched workload measured: returns rank 0's JSON line (None on
    the other ranks).  fixed_point (load factor, block, task chunk) skips the
    autotuner."""
    import ctypes as C
    import torch
    from accmultiwayjoins_b200 import Context, _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = BatchMix(args, rank)
    stream = torch.cuda.current_stream(dev)
    ctx = Context(local_rank, spin_limit_ms=args.spin_limit_ms)
    lib = L.load()
    L.check(lib.amj_ctx_set_stream(ctx.handle, C.c_void_p(stream.cuda_stream)), "set_stream")
    host_cols = [c for q in wl.queries for cols, _ in q["rels"] for c in cols]
    dcols = [torch.from_numpy(c).to(dev) for c in host_cols]
    it = iter(dcols)
    qrels = [[ctx.relation([next(it) for _ in cols], a) for cols, a in q["rels"]] for q in wl.queries]
    b = ctx.batch()
    for q, rels in zip(wl.queries, qrels):
        b.submit(q["qt"], rels)
    torch.cuda.synchronize()

    # plain: one query per call, inputs resident, each call's wall latency; the
    # same plans as the batch (TRI relations joined as given, as a batch joins them)
    plain_lat, plain_tuples, plain_res = [], 0, []
    for q, rels in list(zip(wl.queries, qrels))[:8]:
        ctx.amhj(q["qt"], rels, degree_order=False)
    for q, rels in zip(wl.queries, qrels):
        t0 = time.perf_counter()
        r = ctx.amhj(q["qt"], rels, degree_order=False)
        plain_lat.append((time.perf_counter() - t0) * 1e3)
        plain_tuples += r.count
        plain_res.append((r.count, r.checksum))
    plain_s = sum(plain_lat) / 1e3

    # autotune on every 8th query, then the batched steps (graph replay)
    t0 = time.perf_counter()
    if fixed_point is not None:
        opts, tune_ms = Batch_default_opts(L), None
        opts.load_factor, opts.block_size, opts.task_chunk = fixed_point
    elif args.tune:
        opts, tune_ms = b.tune(sample_every=8, reps=1)
    else:
        opts, tune_ms = Batch_default_opts(L), None
    tune_s = time.perf_counter() - t0
    opts.use_graph = 1
    for _ in range(args.warmup):
        r = b.run(opts=opts)
    assert list(zip(r.counts, r.checksums)) == plain_res, "batched results differ from one query per call"
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    l0 = C.c_uint64()
    L.check(lib.amj_ctx_launch_count(ctx.handle, C.byref(l0)))
    dev_ms, wall_ms = [], []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        r = b.run(opts=opts)
        wall_ms.append((time.perf_counter() - t1) * 1e3)
        dev_ms.append(r.total_ms)
    l1 = C.c_uint64()
    L.check(lib.amj_ctx_launch_count(ctx.handle, C.byref(l1)))
    total = sum(r.counts)

    # end to end: every step copies all relation columns from pinned host
    # memory into the device columns the batch reads, replays, reads results
    pinned = [torch.from_numpy(c).pin_memory() for c in host_cols]
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for d, h in zip(dcols, pinned):
            d.copy_(h, non_blocking=True)
        re_ = b.run(opts=opts)
        if i >= args.warmup:
            e2e_ms.append((time.perf_counter() - t1) * 1e3)
    assert re_.counts == r.counts and re_.checksums == r.checksums
    clocks = sampler.stop()
    ms = sum(dev_ms) / len(dev_ms)
    e2e = sum(e2e_ms) / len(e2e_ms)
    n_queries = len(wl.queries)
    if world > 1:
        # whole job: tuples summed over the ranks, times the slowest rank's
        t = torch.tensor([float(total), float(plain_tuples), float(n_queries)], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t)
        m = torch.tensor([ms, e2e, plain_s], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(m, op=torch.distributed.ReduceOp.MAX)
        total, plain_tuples, n_queries = int(t[0].item()), int(t[1].item()), int(t[2].item())
        ms, e2e, plain_s = m.tolist()
    if rank != 0:
        b.close()
        ctx.close()
        return None
    line = {
        "metric": METRIC, "value": total / (ms * 1e-3), "unit": "tuples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded)",
        "config": {"workload": wl.describe("+rank" if world > 1 else ""), "queries": n_queries, "output_tuples": total,
                   "l2": "inputs far larger than L2 (%.1f GB of relations)" % (wl.h2d / 1e9),
                   "opts": {"layout": int(opts.layout), "load_factor": float(opts.load_factor),
                            "block_size": int(opts.block_size), "task_chunk": int(opts.task_chunk),
                            "use_graph": int(opts.use_graph)},
                   "tuned_on": ("fixed: the point the autotuner chose on this mix" if fixed_point is not None else
                                "every 8th query, full grid" if args.tune else "defaults"),
                   "tune_s": tune_s, "tune_best_sample_ms": tune_ms, "generation_s": wl.gen_s},
        "e2e": {"value": total / (e2e * 1e-3), "unit": "tuples/s", "h2d_bytes_per_step": wl.h2d * world,
                "d2h_bytes_per_step": 16 * n_queries, "ms_per_step": e2e},
        "batched_vs_plain": {
            "plain_value": plain_tuples / plain_s, "plain_ms_total": plain_s * 1e3,
            "batched_over_plain": (total / (ms * 1e-3)) / (plain_tuples / plain_s),
            "latency_ms": {"plain": {"p50": pct(plain_lat, 50), "p99": pct(plain_lat, 99)},
                           "batched": {"p50": pct(wall_ms, 50), "p99": pct(wall_ms, 99),
                                       "note": "every query of a batch completes with the batch"}}},
        "phase_ms": {"build": r.build_ms, "probe": r.probe_ms},
        "gpu_launches": int(l1.value - l0.value),
        "batch_stats": {"launches_per_run": r.launches, "graph": r.graph, "units": r.units,
                        "tasks_pushed": r.tasks_pushed, "build_rows": r.build_rows, "build_jobs": r.build_jobs},
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        tuples, sec, cores, kind, sample = wl.cpu_sample(budget_s=cpu_budget)
        line["cpu_baseline"] = {"value": tuples / sec, "unit": "tuples/s", "cores": cores, "kind": kind,
                                "sample": sample}
    b.close()
    ctx.close()
    return line


class ServeMix:
    """The serving workload: a Poisson request stream (default 200 requests/s)
    of scaled skewed-clique and star queries against relations kept resident
    in HBM, plus out-of-core 4-way chain joins interleaved every few seconds
    whose probe relation stays in pinned host memory.

    Resident templates (each request picks one uniformly, seed 5):
    * FOUR (4-clique) over R-MAT graphs of scale 10, 11, 12 (16 edges per
      vertex, quadrant probabilities 0.6/0.15/0.15/0.1);
    * 4-way star: fact of 50K / 200K / 1M rows of Zipf(1.1) foreign keys into
      dimensions of 1M / 200K / 100K / 10K rows scaled by fact rows / 60M.
    Out-of-core: R1(a,b) R2(b,c) R3(c,d) R4(d,e) of --ooc-rows rows each, keys
    uniform in [0, rows) (about one match per probe row per join)."""

    def __init__(self, args, rank, gen=None, with_ooc=True):
        from accmultiwayjoins_b200 import data
        g = gen or data._Libamj
        self.args = args
        self.templates = []
        for sc in (10, 11, 12):
            s_, d_ = g.rmat(sc, (1 << sc) * 16, 0.6, 0.15, 0.15, seed=5 + sc + 100 * rank)
            self.templates.append(("FOUR", f"4-clique R-MAT scale {sc}", [([s_, d_], [0, 1])]))
        for fr in (50_000, 200_000, 1_000_000):
            dims = [max(100, m * fr // 60_000_000) for m in (1_000_000, 200_000, 100_000, 10_000)]
            fact, dd = data.star_relations(fr, dims, theta=1.1, seed=7 + fr + rank, gen=gen)
            self.templates.append(("NORMAL", f"star fact {fr} dims {dims}", [fact] + dd))
        n = args.ooc_rows if with_ooc else 0
        self.ooc = [([g.uniform(n, 0, n, 31 + i + 10 * rank, 0), g.uniform(n, 0, n, 31 + i + 10 * rank, 1)],
                     [i, i + 1]) for i in range(4)] if n else None

    def describe(self, rank_note):
        return (f"serving: Poisson {self.args.rate:g} requests/s of {len(self.templates)} resident templates "
                f"(FOUR on R-MAT scale 10-12, 4-way star with 50K-1M fact rows) plus an out-of-core 4-way chain "
                f"join of 4 x {self.args.ooc_rows} rows (probe in pinned host memory) every "
                f"{self.args.ooc_every:g} s{rank_note}; continuous batching, {self.args.lanes} lanes")


def run_serve(args, rank, world, local_rank):
    import torch
    from accmultiwayjoins_b200 import Context

    torch.cuda.set_device(local_rank)
    wl = ServeMix(args, rank)
    ctx = Context(local_rank, ooc_slice_rows=args.ooc_slice, spin_limit_ms=args.spin_limit_ms)
    trels = [[ctx.relation(c, a) for c, a in rels] for _, _, rels in wl.templates]
    alone = []
    for (qt, _, _), r in zip(wl.templates, trels):
        x = ctx.amhj(qt, r)
        alone.append((x.count, x.checksum))
    ooc_rels, ooc_want = None, None
    if wl.ooc:
        pinned = [torch.from_numpy(c).pin_memory() for c in wl.ooc[0][0]]
        ooc_rels = [ctx.relation([p.numpy() for p in pinned], wl.ooc[0][1], streamed=True)]
        ooc_rels += [ctx.relation(c, a) for c, a in wl.ooc[1:]]
        x = ctx.amhj("NORMAL", ooc_rels, ooc=1)
        ooc_want = (x.count, x.checksum)
    srv = ctx.server(lanes=args.lanes, max_batch=args.max_batch, ooc_lane=True)
    rng = np.random.Generator(np.random.PCG64(5 + rank))

    def stream(seconds):
        """Submit a Poisson stream for `seconds`; returns [(template or -1, ticket)]."""
        out = []
        t_end = time.perf_counter() + seconds
        t_next = time.perf_counter()
        t_ooc = time.perf_counter() + args.ooc_every / 2
        while True:
            t_next += rng.exponential(1.0 / args.rate)
            if t_next >= t_end:
                break
            while time.perf_counter() < t_next:
                time.sleep(0.0001)
            if ooc_rels is not None and time.perf_counter() >= t_ooc:
                out.append((-1, srv.submit("NORMAL", ooc_rels, ooc=True)))
                t_ooc += args.ooc_every
            i = int(rng.integers(0, len(wl.templates)))
            out.append((i, srv.submit(wl.templates[i][0], trels[i])))
        return out

    warm = stream(args.warmup * 0.5)
    for _, t in warm:
        srv.wait(t)
    st_warm = srv.stats()
    sampler = ClockSampler(local_rank)
    sampler.start()
    t0 = time.perf_counter()
    timed = stream(float(args.steps))
    res = [(i, srv.wait(t)) for i, t in timed]
    clocks = sampler.stop()
    for i, r in res:
        assert (r.count, r.checksum) == (ooc_want if i < 0 else alone[i]), "served result differs from alone"
    st = srv.stats()
    launches_timed = st["launches"] - st_warm["launches"]
    srv.close()
    # the window runs from the first timed submission until every timed request has completed
    total = sum(r.count for _, r in res)
    wall = time.perf_counter() - t0
    n_req = len(res)
    if world > 1:
        dev = torch.device("cuda", local_rank)
        t = torch.tensor([float(total), float(n_req)], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t)
        w = torch.tensor([wall], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(w, op=torch.distributed.ReduceOp.MAX)
        total, n_req, wall = int(t[0].item()), int(t[1].item()), float(w.item())
    if rank != 0:
        ctx.close()
        return
    lat = [r.latency_ms for i, r in res if i >= 0]
    olat = [r.latency_ms for i, r in res if i < 0]
    bsz = [r.batch_size for i, r in res if i >= 0]
    line = {
        "metric": METRIC, "value": total / wall, "unit": "tuples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
        "config": {"workload": wl.describe("+rank" if world > 1 else ""), "step": "one second of the request stream",
                   "requests": n_req, "ooc_requests": len(olat), "output_tuples": total,
                   "l2": "resident relations and ooc inputs larger than L2"},
        "e2e": {"value": total / wall, "unit": "tuples/s",
                "h2d_bytes_per_step": int(len(olat) * 8 * args.ooc_rows / args.steps),
                "d2h_bytes_per_step": int(16 * len(res) / args.steps),
                "note": "requests submitted from the host, results read back; resident relations are not re-copied"},
        "latency_ms": {"resident": {"p50": pct(lat, 50), "p99": pct(lat, 99)},
                       "ooc": {"p50": pct(olat, 50), "p99": pct(olat, 99)} if olat else None},
        "serve_stats": {**st, "mean_batch_size": sum(bsz) / max(1, len(bsz))},
        "gpu_launches": launches_timed,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_ooc(args, rank, world, local_rank):
    """The out-of-core chain of the serving configuration on its own:
    R1(a,b) R2(b,c) R3(c,d) R4(d,e) of --ooc-rows rows each, keys uniform in
    [0, rows) (about one match per probe row per join), every relation kept
    in pinned host memory.  One step is one ooc=1 query through the staged,
    partitioned join (amhj_partitioned.cu) under a memory budget of
    --ooc-budget-gb; the result is checked against the probe-streaming path
    with device-resident builds (when they fit the device) and, with
    --ooc-verify, against the oracle or the reference's MHJ-CPU on the host."""
    import torch
    from accmultiwayjoins_b200 import Context, data
    torch.cuda.set_device(local_rank)
    n = args.ooc_rows
    t0 = time.perf_counter()
    # every column generated straight into pinned host memory (no second copy)
    pinned = []
    for i in range(4):
        cols = []
        for s_ in (0, 1):
            t = torch.empty(n, dtype=torch.int32, pin_memory=True)
            t.numpy()[:] = data.uniform(n, 0, n, 41 + i + 10 * rank, s_)
            cols.append(t)
        pinned.append(cols)
    rels = [([c.numpy() for c in pc], [i, i + 1]) for i, pc in enumerate(pinned)]
    gen_s = time.perf_counter() - t0
    budget = int(args.ooc_budget_gb * (1 << 30))
    ctx = Context(local_rank, mem_budget=budget, spin_limit_ms=args.spin_limit_ms)
    host = [ctx.relation(c, a, streamed=True) for c, a in rels]
    for _ in range(args.warmup):
        r = ctx.amhj("NORMAL", host, ooc=1)
    sampler = ClockSampler(local_rank)
    sampler.start()
    ms, part_ms, join_ms = [], [], []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        r = ctx.amhj("NORMAL", host, ooc=1)
        ms.append((time.perf_counter() - t1) * 1e3)
        part_ms.append(r.kernel_ms[0])
        join_ms.append(r.kernel_ms[1])
    clocks = sampler.stop()
    want = (r.count, r.checksum)
    check = {}
    ctx.trim()   # the staged join's pinned blocks: host memory for the checks
    try:
        dev = [ctx.relation(c, a) for c, a in rels[1:]]
        x = ctx.amhj("NORMAL", [host[0]] + dev, ooc=1)
        check["device_builds_equal"] = (x.count, x.checksum) == want
        for d in dev:
            d.release()
    except Exception as e:   # builds that do not fit the device
        check["device_builds"] = f"not run: {e}"
    if args.ooc_verify != "none":
        # the reference's MHJ-CPU keeps every result tuple and two hash tables
        # of 16-byte entries per build relation in host memory; the oracle's
        # restatement counts and hashes without keeping them
        from oracle import oracle as O
        t1 = time.perf_counter()
        if args.ooc_verify == "reference":
            cnt, chk, _ = O.mhj_reference(rels, nthreads=os.cpu_count() or 1)
        else:
            cnt, chk = O.mhj(rels, nthreads=os.cpu_count() or 1)
        check[f"{args.ooc_verify}_equal"] = (cnt, chk) == want
        check[f"{args.ooc_verify}_seconds"] = time.perf_counter() - t1
    if rank == 0:
        m = sum(ms) / len(ms)
        line = {
            "metric": METRIC, "value": r.count / (m * 1e-3), "unit": "tuples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
            "config": {"workload": f"out-of-core 4-way chain R1(a,b)R2(b,c)R3(c,d)R4(d,e), 4 x {n} rows, keys "
                                   f"U[0,{n}), all relations in pinned host memory; staged hash-partitioned join "
                                   f"under a {args.ooc_budget_gb:g} GB device budget",
                       "output_tuples": r.count, "checksum": f"{r.checksum:016x}", "part_joins": r.stats["slices"],
                       "input_bytes": 32 * n, "generation_s": gen_s},
            "e2e": {"value": r.count / (m * 1e-3), "unit": "tuples/s", "h2d_bytes_per_step": 32 * n,
                    "d2h_bytes_per_step": 16, "note": "inputs start in host memory every step"},
            "check": check, "clocks": clocks,
            "phase_ms": {"host_partitioning": sum(part_ms) / len(part_ms),
                         "part_copies_and_joins": sum(join_ms) / len(join_ms)},
        }
        print(json.dumps(line), flush=True)
    for h in host:
        h.release()
    ctx.close()


def Batch_default_opts(L):
    o = L.amj_batch_opts()
    o.block_size, o.task_chunk = 256, 1024
    return o


def make_workload(args, rank):
    if args.workload == "four":
        return Clique4(args, rank)
    if args.workload == "star":
        return Star(args, rank)
    return Chain(args, rank) if args.workload == "chain" else Triangle(args, rank)


def profiled_traffic(args):
    """DRAM bytes per measured launch from the committed ncu capture of the
    full-size triangle workload, or None."""
    if args.workload != "triangle" or args.scale != SCALE or args.algo != "DFS":
        return None
    p = os.path.join(ROOT, "profiles", "lftj_tri_wedge_kernel_c2.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", open(p).read())
    return int(m.group(1)) if m else None


# ------------------------------------------------------------------ arms

def reference_line(args, value, ms, wl_desc, cpu):
    return {
        "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": wl_desc, "l2": "n/a (CPU)"},
        "cpu_baseline": dict(cpu, value=value),
        "e2e": {"value": value, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference(args, rank, world):
    """CPU arm: the reference's own CPU implementation of the workload on all
    host threads, rank 0 only.  MHJ-CPU (MHJ-CPU/MHJ.cpp) compiled from the
    reference sources into oracle/_ref: as shipped for chains and stars, its
    multi-key probe branch for the cyclic queries.  Each step is a bounded
    sample of the workload (see the classes Ref*).  Inputs are generated by
    the oracle's generators (oracle/orc_gen.cpp, bit-identical to the
    product's), so this process never loads libamj."""
    if rank != 0:
        return
    from oracle import oracle as O
    gen = O.GENERATORS
    cores = os.cpu_count() or 1
    if args.workload == "serve":
        # the reference serves nothing: MHJ-CPU runs the resident templates one
        # request after another, drawn as the stream draws them (stars through
        # the shipped probe, 4-cliques through the multi-key probe over the
        # degree-ordered copy)
        wl = ServeMix(args, 0, gen=gen, with_ooc=False)
        prepared = []
        for qt, _, rels in wl.templates:
            if qt == "FOUR":
                s2, d2, lab = O.degree_ordered_copy(*rels[0][0])
                prepared.append((O.four_relations(s2, d2), True, lab))
            else:
                prepared.append((rels, False, None))
        rng = np.random.Generator(np.random.PCG64(5))
        vals = []
        for i in range(args.warmup + args.steps):
            t_end = time.perf_counter() + 1.0
            tuples, sec, n = 0, 0.0, 0
            while time.perf_counter() < t_end:
                rels, mk, lab = prepared[int(rng.integers(0, len(prepared)))]
                cnt, _, t = O.mhj_reference(rels, nthreads=cores, multi_key=mk, relabel=lab)
                sec += t
                tuples += cnt
                n += 1
            if i >= args.warmup:
                vals.append((tuples, sec, n))
        tuples = sum(v[0] for v in vals)
        sec = sum(v[1] for v in vals)
        sample = (f"{sum(v[2] for v in vals)} requests of the resident templates, one after another, over "
                  f"{args.steps} s (reference MHJ-CPU: shipped probe for the stars, multi-key probe over the "
                  f"degree-ordered copy for the 4-cliques; TBJ calls timed)")
        cpu = {"unit": "tuples/s", "cores": cores, "kind": "reference", "sample": sample}
        print(json.dumps(reference_line(args, tuples / sec, 1e3 * sec / len(vals), wl.describe(""), cpu)),
              flush=True)
        return
    if args.workload == "batch":
        wl = BatchMix(args, 0, gen=gen)
        vals, start = [], 0
        kind = sample = None
        for i in range(args.warmup + args.steps):
            tuples, sec, cores, kind, sample = wl.cpu_sample(budget_s=10.0, start=start)
            start += 1
            if i >= args.warmup:
                vals.append((tuples, sec))
        tuples = sum(t for t, _ in vals)
        sec = sum(t for _, t in vals)
        cpu = {"unit": "tuples/s", "cores": cores, "kind": kind, "sample": sample + "; step i starts at query i"}
        print(json.dumps(reference_line(args, tuples / sec, sec / len(vals) * 1e3, wl.describe(""), cpu)),
              flush=True)
        return
    if args.workload == "ooc":
        # the reference has no out-of-core form for build relations (its
        # ooc=1 keeps them on the GPU): MHJ-CPU joins the same generator's
        # chain at 4 x min(rows, 2^24) rows on the host, one full call per step
        m = min(args.ooc_rows, 1 << 24)
        rels = [([gen.uniform(m, 0, m, 41 + i, 0), gen.uniform(m, 0, m, 41 + i, 1)], [i, i + 1]) for i in range(4)]
        step = lambda: O.mhj_reference(rels, nthreads=cores)[::2]  # noqa: E731  (count, seconds)
        kind = "reference" if O.ref_available() else "port"
        desc = f"out-of-core 4-way chain, keys U[0,rows); sample: 4 x {m} rows"
        sample = "the chain of the same generator at 4 x min(rows, 2^24) rows, MHJ-CPU TBJ call timed"
        times, tuples = [], 0
        for i in range(args.warmup + args.steps):
            cnt, sec = step()
            if i >= args.warmup:
                times.append(sec)
                tuples += cnt
        cpu = {"unit": "tuples/s", "cores": cores, "kind": kind, "sample": sample}
        print(json.dumps(reference_line(args, tuples / sum(times), sum(times) / len(times) * 1e3, desc, cpu)),
              flush=True)
        return
    if args.workload in ("chain", "star"):
        wl = Chain(args, 0, gen=gen) if args.workload == "chain" else Star(args, 0, gen=gen)
        if args.workload == "chain":
            step = lambda: wl.cpu_baseline()[::2][:2]  # noqa: E731  (count, seconds)
        else:
            step = lambda: wl.cpu_baseline(sample_rows=wl.rows)[::2][:2]  # noqa: E731
        desc, sample = wl.describe(""), "the full workload per step (reference MHJ-CPU as shipped, TBJ call timed)"
        kind = "reference" if O.ref_available() else "port"
    else:
        ref = RefClique4() if args.workload == "four" else RefTriangle(args.scale, 1 << (args.scale + 4), SEED)
        step, kind, sample = ref.step, ref.kind, ref.describe()
        desc = (Clique4.describe_static(args.scale, args.algo) if args.workload == "four"
                else Triangle.describe_static(args.scale, args.algo))
    times, tuples = [], 0
    for i in range(args.warmup + args.steps):
        cnt, sec = step()
        if i >= args.warmup:
            times.append(sec)
            tuples += cnt
    sec = sum(times)
    cpu = {"unit": "tuples/s", "cores": cores, "kind": kind, "sample": sample}
    print(json.dumps(reference_line(args, tuples / sec, sec / len(times) * 1e3, desc, cpu)), flush=True)


def chain_record(args, ctx, dev, stream, steps=10, warmup=3):
    """The 3-way chain configuration (3 x 1M rows, keys U[0,2^18)) through
    AMHJ NORMAL: device time per query with the relations resident, the same
    through the C ABI from pinned host buffers, and the reference's MHJ-CPU
    on the full workload."""
    return config_record(args, ctx, dev, stream, Chain(args, 0), steps, warmup)


def config_record(args, ctx, dev, stream, wl, steps=10, warmup=3):
    """One configuration measured beside the headline: device time per query
    with the relations resident, the same through the C ABI from pinned host
    buffers, the main kernel's roofline fraction, and the CPU figure."""
    import torch
    rels = wl.device_relations(ctx, dev)
    for _ in range(warmup):
        r = wl.run(ctx, rels)
    want = (r.count, r.checksum)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    ms, probe = [], []
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = wl.run(ctx, rels)
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
        probe.append(r.kernel_ms[0])
        assert (r.count, r.checksum) == want
    pinned = [torch.from_numpy(c).pin_memory().numpy() for c in wl.host_columns()]
    e2e = []
    for i in range(warmup + steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hr = wl.host_relations(ctx, pinned)
        rr = wl.run(ctx, hr)
        for h in hr:
            h.release()
        if i >= warmup:
            e2e.append((time.perf_counter() - t0) * 1e3)
        assert (rr.count, rr.checksum) == want
    for h in rels:
        h.release()
    m, e = sum(ms) / len(ms), sum(e2e) / len(e2e)
    hbm, _ = peaks()
    kms = sum(probe) / len(probe)
    alg = wl.algorithmic_bytes()
    rec = {"workload": wl.describe(""), "value": want[0] / (m * 1e-3), "unit": "tuples/s", "ms_per_step": m,
           "steps": steps, "output_tuples": want[0], "checksum": f"{want[1]:016x}",
           "e2e": {"value": want[0] / (e * 1e-3), "unit": "tuples/s", "h2d_bytes_per_step": wl.h2d,
                   "d2h_bytes_per_step": 16, "ms_per_step": e},
           "probe_kernel": {"kernel": wl.kernel_name(), "ms": kms}}
    if alg:
        rec["probe_kernel"].update({"alg_bytes": alg, "frac_of_hbm": alg / (kms * 1e-3) / 1e9 / hbm})
    if hasattr(wl, "lookups_per_launch") and kms > 0:
        rec["probe_kernel"]["lookups_per_s"] = wl.lookups_per_launch() / (kms * 1e-3)
    if not args.no_cpu_baseline:
        c_cnt, c_chk, sec, cores, kind, sample = wl.cpu_baseline()
        rec["cpu_baseline"] = {"value": c_cnt / sec, "unit": "tuples/s", "cores": cores, "kind": kind,
                               "sample": sample}
        if c_chk is not None:
            rec["cpu_baseline"]["matches_gpu"] = bool((c_cnt, c_chk) == want)
    return rec


def other_configs(args, ctx, dev, stream, local_rank):
    """Records of the chain (C1), skewed 4-clique (C3a, the configured AMHJ
    FOUR ws=1 fib=1 on R-MAT scale 22), star (C3b) and batched (C4)
    configurations, carried on the default line beside the triangle
    headline."""
    import copy
    out = {"chain": chain_record(args, ctx, dev, stream)}
    fargs = copy.copy(args)
    fargs.scale, fargs.algo = 22, "AMHJ"
    out["four"] = config_record(fargs, ctx, dev, stream, Clique4(fargs, 0), steps=3, warmup=2)
    sargs = copy.copy(args)
    sargs.star_rows = 60_000_000
    out["star"] = config_record(sargs, ctx, dev, stream, Star(sargs, 0), steps=10, warmup=3)
    bargs = copy.copy(args)
    bargs.queries, bargs.steps, bargs.warmup = 512, 5, 3
    bl = batch_line(bargs, 0, 1, local_rank, fixed_point=TUNED_BATCH_POINT, cpu_budget=10.0)
    out["batch"] = {k: bl[k] for k in ("value", "unit", "ms_per_step", "steps", "e2e", "batched_vs_plain",
                                       "phase_ms", "gpu_launches", "cpu_baseline") if k in bl}
    out["batch"]["workload"] = bl["config"]["workload"]
    out["batch"]["opts"] = bl["config"]["opts"]
    out["batch"]["output_tuples"] = bl["config"]["output_tuples"]
    return out


def run_ours(args, rank, world, local_rank):
    import ctypes as C
    import torch
    from accmultiwayjoins_b200 import Context, _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = make_workload(args, rank)
    stream = torch.cuda.current_stream(dev)
    ctx = Context(local_rank, layout=args.layout, spin_limit_ms=args.spin_limit_ms)
    lib = L.load()
    # run the library on torch's stream so torch's CUDA events see its kernels
    L.check(lib.amj_ctx_set_stream(ctx.handle, C.c_void_p(stream.cuda_stream)), "set_stream")
    rels = wl.device_relations(ctx, dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    for _ in range(args.warmup):
        r = wl.run(ctx, rels)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    l0 = C.c_uint64()
    L.check(lib.amj_ctx_launch_count(ctx.handle, C.byref(l0)))
    torch.cuda.synchronize()
    evs, probe_ms, build_ms, kern_ms = [], [], [], []
    t_wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()  # L2 flush (256 MB write) outside the timed events
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = wl.run(ctx, rels)
        b.record(stream)
        evs.append((a, b))
        probe_ms.append(r.probe_ms)
        build_ms.append(r.build_ms)
        kern_ms.append(r.kernel_ms[0] + r.kernel_ms[1])
        count, checksum = r.count, r.checksum
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t_wall = time.perf_counter() - t_wall0
    l1 = C.c_uint64()
    L.check(lib.amj_ctx_launch_count(ctx.handle, C.byref(l1)))
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ms = sum(step_ms) / len(step_ms)

    # end to end through the C ABI from pinned host buffers
    pinned = [torch.from_numpy(c).pin_memory().numpy() for c in wl.host_columns()]
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hr = wl.host_relations(ctx, pinned)
        rr = wl.run(ctx, hr)
        for h in hr:
            h.release()
        dt = (time.perf_counter() - t0) * 1e3
        assert (rr.count, rr.checksum) == (count, checksum)
        if i >= args.warmup:
            e2e_ms.append(dt)
    clocks = sampler.stop()
    e2e_mean = sum(e2e_ms) / len(e2e_ms)

    tot_count, max_ms, max_e2e = count, ms, e2e_mean
    if world > 1:
        cnt = torch.tensor([float(count)], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(cnt)
        mx = torch.tensor([ms, e2e_mean], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        tot_count, max_ms, max_e2e = int(cnt.item()), mx[0].item(), mx[1].item()
    if rank != 0:
        ctx.close()
        return
    hbm, peak_kind = peaks()
    alg = wl.algorithmic_bytes()
    kms = sum(kern_ms) / len(kern_ms)
    achieved = alg / (kms * 1e-3) / 1e9 if (kms > 0 and alg) else None
    rank_note = "+rank" if world > 1 else ""
    line = {
        "metric": METRIC, "value": tot_count / (max_ms * 1e-3), "unit": "tuples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
        "config": {"workload": wl.describe(rank_note) + ("" if args.layout == "bucket" else
                                                          f"; {args.layout} hash tables"),
                   "tuples_per_rank": count,
                   "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"independent instance per GPU x{world}"},
        "e2e": {"value": tot_count / (max_e2e * 1e-3), "unit": "tuples/s", "h2d_bytes_per_step": wl.h2d,
                "d2h_bytes_per_step": 16, "ms_per_step": max_e2e},
        "gpu_launches": int(l1.value - l0.value),
        "latency_ms": {"p50": pct(step_ms, 50), "p99": pct(step_ms, 99),
                       "note": "one query per step; device time of each timed step"},
        "phase_ms": {"build": sum(build_ms) / len(build_ms), "join": sum(probe_ms) / len(probe_ms),
                     "join_kernels": kms},
        "clocks": clocks,
        "wall_s_timed": t_wall,
    }
    if isinstance(wl, Triangle):
        line["config"]["edges_after_cleaning"] = wl.E
    if achieved is not None:
        line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                            "frac": achieved / hbm, "traffic": profiled_traffic(args), "peak_kind": peak_kind,
                            "kernel": wl.kernel_name(), "alg_bytes_per_launch": alg}
        if hasattr(wl, "lookups_per_launch"):
            line["roofline"]["lookups_per_s"] = wl.lookups_per_launch() / (kms * 1e-3)
    if isinstance(wl, Triangle) and world == 1 and not args.no_configs:
        line["configs"] = other_configs(args, ctx, dev, stream, local_rank)
    if not args.no_cpu_baseline:
        c_cnt, c_chk, sec, cores, kind, sample = wl.cpu_baseline()
        line["cpu_baseline"] = {"value": c_cnt / sec, "unit": "tuples/s", "cores": cores, "kind": kind,
                                "sample": sample}
        if c_chk is not None:
            line["cpu_baseline"]["matches_gpu"] = bool((c_cnt, c_chk) == (count, checksum))
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--algo", default="DFS", choices=["DFS", "BFS", "AMHJ"])
    ap.add_argument("--workload", default="triangle", choices=["triangle", "chain", "four", "star", "batch", "serve", "ooc"])
    ap.add_argument("--spin-limit-ms", type=int, default=5000, help="bound on every device-side wait")
    ap.add_argument("--rate", type=float, default=200.0, help="serve workload: requests per second")
    ap.add_argument("--lanes", type=int, default=3, help="serve workload: batches in flight")
    ap.add_argument("--max-batch", type=int, default=128, help="serve workload: requests per batch")
    ap.add_argument("--ooc-rows", type=int, default=64 << 20, help="serve workload: rows per ooc relation")
    ap.add_argument("--ooc-every", type=float, default=2.5, help="serve workload: seconds between ooc joins")
    ap.add_argument("--ooc-slice", type=int, default=8 << 20, help="serve workload: ooc probe slice rows")
    ap.add_argument("--ooc-budget-gb", type=float, default=8.0, help="ooc workload: device memory budget")
    ap.add_argument("--ooc-verify", default="none", choices=["none", "oracle", "reference"],
                    help="ooc workload: also check the result on the host (the oracle, or the reference MHJ-CPU)")
    ap.add_argument("--queries", type=int, default=512, help="batch workload: queries per batch")
    ap.add_argument("--min-rows", type=int, default=10_000, help="batch workload: smallest relation")
    ap.add_argument("--max-rows", type=int, default=4_000_000, help="batch workload: largest relation")
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="batch workload: skip the autotuner")
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--star-rows", type=int, default=60_000_000, help="star workload: fact table rows")
    ap.add_argument("--layout", default="bucket", choices=["bucket", "oa", "cuckoo"],
                    help="chain / star workloads: hash-table layout of the AMHJ builds")
    ap.add_argument("--plan", default="multiway", choices=["multiway", "thread_per_row", "pairwise", "frontier"],
                    help="chain / star workloads: the operator, one of the reference's baseline plans, or the "
                         "operator's frontier-DFS kernel for every plan")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="triangle workload: skip the chain and batched records carried on the line")
    args = ap.parse_args()
    if args.impl == "ours":
        # the out-of-core chain runs a minute or more per step at full size:
        # one warm-up step there, three everywhere else
        args.warmup = max(args.warmup, 1 if args.workload == "ooc" else 3)
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
    if args.workload == "batch":
        run_batch(args, rank, world, local_rank)
    elif args.workload == "serve":
        run_serve(args, rank, world, local_rank)
    elif args.workload == "ooc":
        run_ooc(args, rank, world, local_rank)
    else:
        run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
