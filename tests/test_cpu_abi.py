"""The C ABI library without a GPU: it loads, exports every entry point
include/amj.h declares, and its host-side pieces (generators, .db files,
checksum, argument validation, the CLI drivers) behave."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from accmultiwayjoins_b200 import AmjError, _lib as L, data

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in ("amj.h",):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(amj_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(built):
    lib = L.load()
    names = declared_functions()
    assert len(names) > 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(L.SIGNATURES), set(names) - set(L.SIGNATURES)


def test_version_and_stat_names(built):
    lib = L.load()
    assert b"sm_100a" in lib.amj_version()
    assert lib.amj_stat_name(0) == b"tasks_pushed"
    assert lib.amj_stat_name(99) == b""


def test_ctx_create_without_device_reports_status(built):
    lib = L.load()
    h = C.c_void_p()
    st = lib.amj_ctx_create(0, None, C.byref(h))
    if st == L.AMJ_OK:
        lib.amj_ctx_destroy(h)
        pytest.skip("a CUDA device is present")
    assert st == L.AMJ_ECUDA
    assert b"no CUDA device" in lib.amj_last_error()


def test_null_arguments_are_rejected(built):
    lib = L.load()
    res = L.amj_result()
    assert lib.amj_amhj_execute(None, 0, None, 0, 0, 0, 0, 0, 0, C.byref(res)) == L.AMJ_EINVAL
    assert lib.amj_lftj_execute(None, None, 0, 1, 0, 0, 0, C.byref(res)) == L.AMJ_EINVAL
    assert lib.amj_bucket_build(None, None, 0, 3, None, None, None) == L.AMJ_EINVAL


def test_uniform_generator_is_seeded_and_in_range(built):
    a = data.uniform(100000, -7, 13, seed=5)
    b = data.uniform(100000, -7, 13, seed=5)
    c = data.uniform(100000, -7, 13, seed=6)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.min() >= -7 and a.max() < 13
    counts = np.bincount(a + 7)
    assert counts.min() > 4000


def test_permutation_and_zipf(built):
    p = data.permutation(10000, seed=3)
    assert np.array_equal(np.sort(p), np.arange(10000))
    z = data.zipf(200000, 1000, 1.1, seed=2)
    assert z.min() >= 0 and z.max() < 1000
    top = np.bincount(z, minlength=1000)
    assert top[0] > top[1] > top[10] > top[500]
    zk = data.zipf(1000, 100, 1.1, seed=2, rank_to_key=np.arange(100, 200, dtype=np.int32))
    assert zk.min() >= 100 and zk.max() < 200


def test_rmat_relation_is_clean(built):
    s, d = data.rmat(12, 50000, 0.57, 0.19, 0.19, seed=1)
    assert (s < d).all()
    keys = s.astype(np.int64) * (1 << 32) + d
    assert len(np.unique(keys)) == len(keys)
    assert d.max() < 4096
    s2, d2 = data.rmat(12, 50000, 0.57, 0.19, 0.19, seed=1)
    assert np.array_equal(s, s2) and np.array_equal(d, d2)
    assert not np.all(np.diff(s) >= 0), "rows are shuffled"


def test_db_round_trip_and_name(tmp_path, built):
    cols = [data.uniform(1000, -100, 100, seed=1, stream=i) for i in range(3)]
    p = str(tmp_path / data.db_name(1000, [2, 0, 5]))
    data.write_db(p, cols)
    got, attrs = data.read_db(p)
    assert attrs == [2, 0, 5]
    for a, b in zip(cols, got):
        assert np.array_equal(a, b)
    assert os.path.getsize(p) == 1000 * 3 * 4


def test_db_errors(tmp_path, built):
    p = str(tmp_path / "10_0_1.db")
    data.write_db(p, [np.zeros(9, np.int32), np.zeros(9, np.int32)])
    with pytest.raises(AmjError) as e:
        data.read_db(p)
    assert e.value.status == L.AMJ_EIO
    with pytest.raises(AmjError):
        data.read_db(str(tmp_path / "abc_0.db"))
    with pytest.raises(AmjError):
        data.read_db(str(tmp_path / "10_0_99.db"))


def test_cli_drivers_exist_and_print_usage(built):
    for name in ("exec-AMHJ", "exec-LFTJ"):
        exe = os.path.join(ROOT, "accmultiwayjoins_b200", "bin", name)
        assert os.access(exe, os.X_OK), exe
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 2 and "usage" in r.stderr


MIRRORED_STRUCTS = ["amj_opts", "amj_result", "amj_batch_opts", "amj_batch_stats", "amj_batch_tune_grid",
                    "amj_serve_opts", "amj_serve_result", "amj_serve_stats"]


def test_ctypes_mirrors_match_the_header(tmp_path):
    """Every ctypes structure has the size and field offsets the C compiler
    gives the struct of the same name in include/amj.h (a mismatch would pass
    options and read results at the wrong bytes)."""
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "amj.h"', "int main(void) {"]
    for name in MIRRORED_STRUCTS:
        ct = getattr(L, name)
        lines.append(f'printf("{name} sizeof %zu\\n", sizeof({name}));')
        for f in ct._fields_:
            lines.append(f'printf("{name} {f[0]} %zu\\n", offsetof({name}, {f[0]}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for name in MIRRORED_STRUCTS:
        ct = getattr(L, name)
        assert got[(name, "sizeof")] == C.sizeof(ct), name
        for f in ct._fields_:
            assert got[(name, f[0])] == getattr(ct, f[0]).offset, (name, f[0])
