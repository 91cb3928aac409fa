"""Cyclic queries against golden fixtures computed by the reference itself.

tests/golden/golden.json holds triangle (TRI) and 4-clique (FOUR) results of
the reference's MHJ-CPU multi-key probe (MHJ-CPU/MHJ.cpp:64-90, :205-245,
driven through oracle/mhj_ref/mhj_ref_harness.cpp) over seeded R-MAT edge
relations, up to the full triangle configuration (R-MAT scale 20, 2^24
generated edges).  Every CUDA path that answers these queries is compared
with them through the C ABI: AMHJ TRI / FOUR with each work-sharing switch,
on the relation as given and on its degree-ordered copy, through the
bitmap / triangle-matrix levels and with every level a hash lookup; ALFTJ
DFS (wedge
kernel, lane merge), BFS; the ALFTJ 4-clique through the triangle matrices
and through the list-intersection kernel.
"""
import json
import os

import pytest

from accmultiwayjoins_b200 import data

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")
CASES = [c for c in json.load(open(GOLDEN))["cases"] if c["kind"] in ("tri", "four")]


def relation(ctx, case):
    s, d = data.rmat(case["scale"], case["nedges"], *case["abc"], seed=case["seed"])
    assert s.shape[0] == case["edges"]
    return ctx.relation([s, d], [0, 1])


def want(case):
    return case["count"], int(case["checksum"], 16)


@pytest.mark.parametrize("case", [c for c in CASES if c["kind"] == "tri"], ids=lambda c: c["name"])
def test_triangle_paths_match_reference_golden(ctx, case):
    e = relation(ctx, case)
    full = case["edges"] > 4_000_000
    runs = [("ALFTJ DFS ws=1", lambda: ctx.lftj([e], algo="DFS", ws=1)),
            ("ALFTJ BFS", lambda: ctx.lftj([e], algo="BFS")),
            ("AMHJ TRI ws=1", lambda: ctx.amhj("TRI", [e], ws=1)),
            ("AMHJ TRI ws=1, hash plan", lambda: ctx.amhj("TRI", [e], ws=1, plan="hash"))]
    if not full:
        runs += [("ALFTJ DFS ws=0", lambda: ctx.lftj([e], algo="DFS", ws=0)),
                 ("ALFTJ DFS as given", lambda: ctx.lftj([e], algo="DFS", ws=1, degree_order=False)),
                 ("ALFTJ BFS as given", lambda: ctx.lftj([e], algo="BFS", degree_order=False)),
                 ("AMHJ TRI ws=0 as given", lambda: ctx.amhj("TRI", [e], degree_order=False)),
                 ("AMHJ TRI ws=1 dro=1", lambda: ctx.amhj("TRI", [e], ws=1, dro=1)),
                 ("AMHJ TRI ws=0 dro=1, hash plan", lambda: ctx.amhj("TRI", [e], dro=1, plan="hash"))]
    for name, run in runs:
        r = run()
        assert (r.count, r.checksum) == want(case), name


@pytest.mark.parametrize("case", [c for c in CASES if c["kind"] == "four"], ids=lambda c: c["name"])
def test_four_clique_paths_match_reference_golden(ctx, case):
    e = relation(ctx, case)
    runs = [("ALFTJ 4-clique (triangle matrices)", lambda: ctx.lftj([e], clique4=True)),
            ("ALFTJ 4-clique as given (list kernel)", lambda: ctx.lftj([e], clique4=True, degree_order=False)),
            ("AMHJ FOUR ws=1 fib=1", lambda: ctx.amhj("FOUR", [e], ws=1, fib=1)),
            ("AMHJ FOUR ws=1 fib=1, hash plan", lambda: ctx.amhj("FOUR", [e], ws=1, fib=1, plan="hash")),
            ("AMHJ FOUR ws=0 dro=1, hash plan", lambda: ctx.amhj("FOUR", [e], dro=1, plan="hash")),
            ("AMHJ FOUR ws=0 as given", lambda: ctx.amhj("FOUR", [e], degree_order=False))]
    for name, run in runs:
        r = run()
        assert (r.count, r.checksum) == want(case), name
