"""Writes tests/golden/golden.json: counts and checksums of seeded chain and
star joins computed by the reference's MHJ-CPU (MHJ-CPU/MHJ.cpp, compiled
from the reference sources by oracle/Makefile into oracle/_ref/).

Run in a container that has the reference sources:
    make -C oracle && python tests/golden/make_golden.py
The inputs are regenerated from their seeds by accmultiwayjoins_b200.data.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from accmultiwayjoins_b200 import data  # noqa: E402
from oracle import oracle as O  # noqa: E402

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
]


def make(case):
    if case["kind"] == "chain":
        return data.chain_relations(case["n"], case["key_range"], case["nrels"], seed=case["seed"])
    fact, dims = data.star_relations(case["fact_rows"], case["dims"], theta=case["theta"], seed=case["seed"])
    return [fact] + dims


def main():
    if not O.ref_available():
        O.build()
    out = []
    for case in CASES:
        rels = make(case)
        cnt, chk, secs = O.mhj_reference(rels)
        assert O.mhj(rels) == (cnt, chk), case["name"]
        out.append(dict(case, count=cnt, checksum=f"{chk:016x}"))
        print(case["name"], cnt, f"{chk:016x}", f"{secs:.3f}s")
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"source": "reference MHJ-CPU (MHJ-CPU/MHJ.cpp TBJ) via oracle/mhj_ref/mhj_ref_harness.cpp",
                   "checksum": "sum of per-tuple splitmix64-chain hashes, include/amj_checksum.h",
                   "cases": out}, f, indent=1)


if __name__ == "__main__":
    main()
