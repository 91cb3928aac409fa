"""Writes tests/golden/golden.json: counts and checksums of seeded joins
computed by the reference's MHJ-CPU (MHJ-CPU/MHJ.cpp), compiled from the
reference sources by oracle/Makefile into oracle/_ref/.

* chain / star cases: the reference as shipped (single-key probe,
  _ref/libmhjref.so).
* tri / four cases: the TRI and FOUR attribute patterns of
  MHJ-GPU/exec_AMHJ.cu:32-69 over one cleaned R-MAT edge relation, run by the
  reference's multi-key probe (_ref/libmhjref_mk.so, MHJ.cpp:64-90 and
  :205-245).  "how": "as given" joins the relation as generated (u < v);
  "degree-ordered" joins its (degree, id)-ranked copy and renames every
  result tuple back to vertex ids, sorted (oracle.degree_ordered_copy): the
  same cliques, at a fraction of the reference's work on the skewed graphs.

Every case is also checked against the oracle's restatement before it is
written.  Inputs are regenerated from their seeds by the oracle's own
generators (oracle/orc_gen.cpp), which the CPU tests check bit for bit
against the product's.

Run in a container that has the reference sources:
    make -C oracle && python tests/golden/make_golden.py [--only NAME ...] [--force]
Cases already in golden.json with the same parameters are kept unless
--force is given (the full-size triangle takes about ten minutes on 8 cores).
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from accmultiwayjoins_b200 import data  # noqa: E402  (workload builders; inputs come from gen=O.GENERATORS)
from oracle import oracle as O  # noqa: E402

A, B = (0.57, 0.19, 0.19), (0.6, 0.15, 0.15)

CASES = [
    {"name": "chain3_1k", "kind": "chain", "n": 1000, "key_range": 256, "nrels": 3, "seed": 1},
    {"name": "chain3_64k", "kind": "chain", "n": 65536, "key_range": 1 << 14, "nrels": 3, "seed": 2},
    {"name": "chain4_20k", "kind": "chain", "n": 20000, "key_range": 1 << 12, "nrels": 4, "seed": 3},
    {"name": "chain5_5k_skewfree", "kind": "chain", "n": 5000, "key_range": 1 << 11, "nrels": 5, "seed": 4},
    {"name": "chain3_1M_c1", "kind": "chain", "n": 1000000, "key_range": 1 << 18, "nrels": 3, "seed": 1},
    {"name": "star4_100k", "kind": "star", "fact_rows": 100000, "dims": [10000, 2000, 1000, 100], "theta": 1.1,
     "seed": 3},
    {"name": "star4_1M", "kind": "star", "fact_rows": 1000000, "dims": [100000, 20000, 10000, 1000], "theta": 1.1,
     "seed": 5},
    {"name": "star4_60M_c3b", "kind": "star", "fact_rows": 60000000, "dims": [1000000, 200000, 100000, 10000],
     "theta": 1.1, "seed": 3},
]


def graph_case(kind, scale, abc, seed, how, name=None, nedges=None):
    tag = "a" if abc == A else "b"
    return {"name": name or f"{kind}_rmat{scale}_{tag}", "kind": kind, "scale": scale,
            "nedges": nedges or (1 << (scale + 4)), "abc": list(abc), "seed": seed, "how": how}


CASES += [
    graph_case("tri", 8, A, 8, "as given"),
    graph_case("tri", 10, B, 10, "as given"),
    graph_case("tri", 12, A, 12, "as given"),
    graph_case("tri", 14, B, 14, "as given"),
    graph_case("tri", 16, A, 16, "degree-ordered"),
    graph_case("tri", 16, B, 16, "degree-ordered"),
    graph_case("tri", 20, A, 20, "degree-ordered", name="tri_rmat20_c2"),
    graph_case("four", 8, B, 8, "as given"),
    graph_case("four", 10, A, 10, "as given"),
    graph_case("four", 12, B, 12, "as given"),
    graph_case("four", 14, B, 22, "degree-ordered", name="four_rmat14_b_seed22"),
]


def make(case):
    """The case's relations in query order (TRI / FOUR patterns over one
    relation for the graph cases)."""
    kind = case["kind"]
    if kind == "chain":
        return data.chain_relations(case["n"], case["key_range"], case["nrels"], seed=case["seed"], gen=O.GENERATORS)
    if kind == "star":
        fact, dims = data.star_relations(case["fact_rows"], case["dims"], theta=case["theta"], seed=case["seed"],
                                         gen=O.GENERATORS)
        return [fact] + dims
    return O.gen_rmat(case["scale"], case["nedges"], *case["abc"], seed=case["seed"])


def run(case, cores):
    kind = case["kind"]
    if kind in ("chain", "star"):
        rels = make(case)
        cnt, chk, secs = O.mhj_reference(rels, nthreads=cores)
        assert O.mhj(rels, nthreads=cores) == (cnt, chk), case["name"]
        return {"count": cnt, "checksum": f"{chk:016x}", "seconds": round(secs, 3)}
    src, dst = make(case)
    pattern = O.tri_relations if kind == "tri" else O.four_relations
    if case["how"] == "as given":
        cnt, chk, secs = O.mhj_reference(pattern(src, dst), nthreads=cores, multi_key=True)
    else:
        s2, d2, rank_to_id = O.degree_ordered_copy(src, dst)
        cnt, chk, secs = O.mhj_reference(pattern(s2, d2), nthreads=cores, multi_key=True, relabel=rank_to_id)
    restated = O.triangle(src, dst, nthreads=cores) if kind == "tri" else O.four_clique(src, dst, nthreads=cores)
    assert restated == (cnt, chk), (case["name"], restated, (cnt, chk))
    return {"edges": int(src.shape[0]), "count": cnt, "checksum": f"{chk:016x}", "seconds": round(secs, 3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    if not (O.ref_available() and O.ref_available(multi_key=True)):
        O.build()
    cores = os.cpu_count() or 1
    path = os.path.join(HERE, "golden.json")
    old = {}
    if os.path.exists(path):
        with open(path) as f:
            old = {c["name"]: c for c in json.load(f)["cases"]}
    out = []
    for case in CASES:
        prev = old.get(case["name"])
        keep = prev is not None and all(prev.get(k) == v for k, v in case.items())
        if keep and not args.force and (args.only is None or case["name"] not in args.only):
            out.append(prev)
            continue
        if args.only is not None and case["name"] not in args.only and not keep:
            continue
        t0 = time.perf_counter()
        res = run(case, cores)
        out.append(dict(case, **res))
        print(case["name"], res, f"{time.perf_counter() - t0:.1f}s", flush=True)
    with open(path, "w") as f:
        json.dump({"source": "reference MHJ-CPU (MHJ-CPU/MHJ.cpp TBJ) via oracle/mhj_ref/mhj_ref_harness.cpp; "
                             "tri/four cases with its multi-key probe (_ref/libmhjref_mk.so)",
                   "checksum": "sum of per-tuple splitmix64-chain hashes, include/amj_checksum.h",
                   "cases": out}, f, indent=1)


if __name__ == "__main__":
    main()
