"""Edge-list converters (amj_edgelist_*; the reference's edgelist_2_db,
MHJ-GPU/exec_el_2_db.cu, and switch_el.py) on the CPU: the .db bytes equal
those of the reference's own converter, compiled from its sources into
oracle/_ref, and the parse rules hold."""
import os
import subprocess

import numpy as np
import pytest

from accmultiwayjoins_b200 import AmjError, data
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EL2DB = os.path.join(ROOT, "oracle", "_ref", "exec_el_2_db")
BIN = os.path.join(ROOT, "accmultiwayjoins_b200", "bin")


def write_edgelist(path, src, dst, seps=(" ", "\t", "|", " | ", "  ")):
    with open(path, "w") as f:
        for i, (u, v) in enumerate(zip(src, dst)):
            f.write(f"{u}{seps[i % len(seps)]}{v}\n")


def edges(n, seed):
    s, d = O.gen_rmat(12, n, 0.57, 0.19, 0.19, seed=seed)
    return s, d


@pytest.mark.skipif(not os.path.exists(REF_EL2DB), reason="reference converter not built (reference sources absent)")
def test_db_bytes_equal_reference_converter(tmp_path, built):
    s, d = edges(20000, 3)
    # the reference reads values with stoul and stores int: large and
    # negative values wrap modulo 2^32
    s = np.concatenate([s, np.array([4294967295, 2147483648, 0], np.int64)])
    d = np.concatenate([d, np.array([-5, 7, 2147483647], np.int64)])
    txt = tmp_path / "graph.txt"
    write_edgelist(txt, s, d)
    subprocess.run([REF_EL2DB, str(txt)], check=True, capture_output=True)
    ref = open(str(txt) + ".db", "rb").read()
    ours = tmp_path / "ours.db"
    assert data.edgelist_to_db(str(txt), str(ours)) == len(s)
    assert open(ours, "rb").read() == ref
    a, b = data.read_edgelist(str(txt))
    want = np.frombuffer(ref, np.int32).reshape(2, -1)
    assert np.array_equal(a, want[0]) and np.array_equal(b, want[1])


def test_parse_rules_comments_blank_lines_and_swap(tmp_path, built):
    txt = tmp_path / "g.txt"
    txt.write_text("# SNAP header\n% matrix market comment\n\n1 2\n 3\t4 \r\n5|6\n-1 4294967295\n7  8")
    a, b = data.read_edgelist(str(txt))
    assert a.tolist() == [1, 3, 5, -1, 7] and b.tolist() == [2, 4, 6, -1, 8]
    a2, b2 = data.read_edgelist(str(txt), swap=True)
    assert np.array_equal(a2, b) and np.array_equal(b2, a)
    out = tmp_path / "5_0_1.db"
    assert data.edgelist_to_db(str(txt), str(out), swap=True) == 5
    cols, attrs = data.read_db(str(out))
    assert attrs == [0, 1] and np.array_equal(cols[0], b) and np.array_equal(cols[1], a)


@pytest.mark.parametrize("text", ["1 2 3\n", "1\n", "1 x\n", "1 2\nfoo bar\n", "1 2z\n"])
def test_malformed_lines_are_errors(tmp_path, built, text):
    txt = tmp_path / "bad.txt"
    txt.write_text(text)
    with pytest.raises(AmjError, match="line"):
        data.read_edgelist(str(txt))


def test_empty_and_missing_files(tmp_path, built):
    e = tmp_path / "empty.txt"
    e.write_text("")
    a, b = data.read_edgelist(str(e))
    assert a.size == 0 and b.size == 0
    with pytest.raises(AmjError):
        data.read_edgelist(str(tmp_path / "missing.txt"))


def test_large_file_is_parsed_in_parallel_in_order(tmp_path, built):
    s, d = edges(400000, 9)   # several MB: the parser cuts it into per-thread chunks
    txt = tmp_path / "big.txt"
    write_edgelist(txt, s, d)
    a, b = data.read_edgelist(str(txt))
    assert np.array_equal(a, s) and np.array_equal(b, d)


def test_cli_converter(tmp_path, built):
    txt = tmp_path / "g.txt"
    txt.write_text("4 5\n6 7\n")
    r = subprocess.run([os.path.join(BIN, "exec-el-2-db"), str(txt)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert np.frombuffer(open(str(txt) + ".db", "rb").read(), np.int32).tolist() == [4, 6, 5, 7]
    r = subprocess.run([os.path.join(BIN, "exec-el-2-db"), str(txt), str(tmp_path / "s.db"), "--swap"],
                       capture_output=True, text=True)
    assert r.returncode == 0
    assert np.frombuffer(open(tmp_path / "s.db", "rb").read(), np.int32).tolist() == [5, 7, 4, 6]
    r = subprocess.run([os.path.join(BIN, "edgelist-to-csr")], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


# ---- delimited tables (amj_tbl_to_db; the reference's tbl_2_db, MHJ-GPU/exec_tbl_2_db.cu) ----

REF_TBL2DB = os.path.join(ROOT, "oracle", "_ref", "exec_tbl_2_db")
WORDS = ["quick", "pending", "final", "deposits", "sleep", "ironic", "ideas", "haggle", "blithely"]


def synthetic_table(path, n, seed, nkeys=(1000, 300, 50)):
    """A seeded '|'-delimited table shaped like a TPC-H fact table: three
    integer keys, a decimal, a date, a flag, a free-text comment with spaces,
    and a trailing '|'.  Returns the integer key columns."""
    rng = np.random.default_rng(seed)
    k = [rng.integers(0, m, n) for m in nkeys]
    price = rng.integers(100, 10**7, n)
    with open(path, "w") as f:
        for i in range(n):
            words = " ".join(WORDS[j] for j in rng.integers(0, len(WORDS), 1 + i % 4))
            f.write(f"{k[0][i]}|{k[1][i]}|{k[2][i]}|{price[i] // 100}.{price[i] % 100:02d}|"
                    f"199{i % 8}-0{1 + i % 9}-1{i % 10}|{'NOF'[i % 3]}|{words} |\n")
    return k


@pytest.mark.skipif(not os.path.exists(REF_TBL2DB), reason="reference converter not built (reference sources absent)")
@pytest.mark.parametrize("fields,attrs", [([0, 1], [0, 1]), ([2, 0], [3, 1]), ([1, 2, 0], [2, 0, 1]), ([3], [5])])
def test_tbl_bytes_and_name_equal_reference_converter(tmp_path, built, fields, attrs):
    tbl = tmp_path / "fact.tbl"
    synthetic_table(tbl, 3000, 11)
    refdir = tmp_path / "ref"
    refdir.mkdir()
    subprocess.run([REF_TBL2DB, str(tbl)] + [str(x) for x in fields + attrs], check=True, capture_output=True,
                   cwd=refdir)
    (ref_name,) = os.listdir(refdir)
    ours = data.tbl_to_db(str(tbl), fields, attrs, out_dir=str(tmp_path))
    assert os.path.basename(ours) == ref_name
    assert open(ours, "rb").read() == open(refdir / ref_name, "rb").read()


def test_tbl_columns_in_given_order_and_renamed(tmp_path, built):
    tbl = tmp_path / "t.tbl"
    k = synthetic_table(tbl, 500, 4)
    path = data.tbl_to_db(str(tbl), [2, 0, 3], [7, 1, 4], out_dir=str(tmp_path))
    assert os.path.basename(path) == "500_7_1_4.db"
    cols, attrs = data.read_db(path)
    assert attrs == [7, 1, 4]
    assert np.array_equal(cols[0], k[2]) and np.array_equal(cols[1], k[0])
    # field 3 is a decimal: stoul keeps its integer part
    want = []
    for line in open(tbl):
        want.append(int(line.split("|")[3].split(".")[0]))
    assert cols[2].tolist() == want


def test_tbl_parse_rules(tmp_path, built):
    tbl = tmp_path / "r.tbl"
    # runs of separators collapse (strtok), tabs separate too, spaces stay in
    # a field and lead stoul, negative values and 2^32-1 wrap to int32, blank
    # lines are skipped
    tbl.write_text("1|2|x y|\n\n3\t|4|z|\n -5||4294967295|w\n7|8\n")
    path = data.tbl_to_db(str(tbl), [0, 1], [0, 1], out_dir=str(tmp_path))
    cols, _ = data.read_db(path)
    assert cols[0].tolist() == [1, 3, -5, 7] and cols[1].tolist() == [2, 4, -1, 8]


@pytest.mark.parametrize("text,fields", [("1|2|\n3|\n", [0, 1]), ("1|abc|\n", [1]), ("1|2\n", [0, 5])])
def test_tbl_missing_or_non_integer_fields_are_errors(tmp_path, built, text, fields):
    tbl = tmp_path / "bad.tbl"
    tbl.write_text(text)
    with pytest.raises(AmjError, match="line"):
        data.tbl_to_db(str(tbl), fields, list(range(len(fields))), out_dir=str(tmp_path))


def test_tbl_bad_arguments(tmp_path, built):
    tbl = tmp_path / "t.tbl"
    tbl.write_text("1|2|\n")
    with pytest.raises(AmjError):
        data.tbl_to_db(str(tbl), [0, 0], [0, 1], out_dir=str(tmp_path))
    with pytest.raises(AmjError):
        data.tbl_to_db(str(tmp_path / "missing.tbl"), [0], [0], out_dir=str(tmp_path))
    with pytest.raises(ValueError):
        data.tbl_to_db(str(tbl), [0, 1], [0], out_dir=str(tmp_path))


def test_tbl_large_file_parsed_in_parallel_in_order(tmp_path, built):
    tbl = tmp_path / "big.tbl"
    k = synthetic_table(tbl, 60000, 8)   # a few MB: parsed in per-thread chunks
    path = data.tbl_to_db(str(tbl), [0, 1, 2], [0, 1, 2], out_dir=str(tmp_path))
    cols, _ = data.read_db(path)
    for c in range(3):
        assert np.array_equal(cols[c], k[c])


def test_tbl_cli(tmp_path, built):
    tbl = tmp_path / "c.tbl"
    k = synthetic_table(tbl, 100, 2)
    r = subprocess.run([os.path.join(BIN, "exec-tbl-2-db"), str(tbl), "1", "0", "4", "2"], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    cols, attrs = data.read_db(str(tmp_path / "100_4_2.db"))
    assert attrs == [4, 2] and np.array_equal(cols[0], k[1]) and np.array_equal(cols[1], k[0])
    assert subprocess.run([os.path.join(BIN, "exec-tbl-2-db"), str(tbl), "1"], capture_output=True).returncode == 2
