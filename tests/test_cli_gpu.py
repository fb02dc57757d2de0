"""The drop-in command-line tools on real CSV files: same argv and formats as
the reference tools, final matchings identical to the oracle's."""
import os
import subprocess

import numpy as np
import pytest

import bm
import oracle
from conftest import PKG

pytestmark = pytest.mark.gpu
BIN = os.path.join(PKG, "bin")


@pytest.fixture(scope="module")
def files(tmp_path_factory, cfg0):
    d = tmp_path_factory.mktemp("cli")
    g = cfg0
    for name, (s, t, w) in (("gm.csv", ("src1", "dst1", "w1")), ("gf.csv", ("src2", "dst2", "w2"))):
        with open(d / name, "w") as f:
            f.write("from,to,weight\n")
            for a, b, c in zip(g[s], g[t], g[w]):
                f.write(f"{a},{b},{c}\n")
    bm.write_mapping_csv(str(d / "in.csv"), g["map0"])
    for o in ("ordM.csv", "ordF.csv"):
        (d / o).write_text("node,order\n")
    return d


def _run(args, env=None, cwd=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run(args, capture_output=True, text=True, env=e, cwd=cwd, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def _read(path, n):
    m, _ = bm.read_mapping_csv(str(path), n)
    return m


def test_quick_matches_oracle_hillclimb(files, cfg0):
    g = cfg0
    _run([os.path.join(BIN, "quick"), str(files / "gm.csv"), str(files / "gf.csv"), str(files / "in.csv"),
          str(files / "q.csv")])
    out = files / "q-rank0.csv"
    assert out.exists()
    assert open(out).readline().strip() == "Male Node ID,Female Node ID"
    O = oracle.Oracle.from_pair(g)
    m = g["map0"].copy()
    while O.sweep(m)["committed"]:
        pass
    assert np.array_equal(_read(out, g["n"]), m)


def test_refine_matching_hillclimb_numeric_format(files, cfg0):
    g = cfg0
    out = files / "r.csv"
    stdout = _run([os.path.join(BIN, "refine-matching-hillclimb"), str(files / "gm.csv"), str(files / "gf.csv"),
                   str(files / "in.csv"), str(out)])
    assert "Final matching score:" in stdout
    assert open(out).readline().strip() == "Male ID,Female ID"
    O = oracle.Oracle.from_pair(g)
    m = g["map0"].copy()
    while O.sweep(m)["committed"]:
        pass
    assert np.array_equal(_read(out, g["n"]), m)
    assert f"Final matching score: {O.score(m)}" in stdout


def test_graph_alignment_optimized_reference_order(files, cfg0):
    g = cfg0
    out = files / "gao.csv"
    _run([os.path.join(BIN, "graph-alignment-optimized"), str(files / "gm.csv"), str(files / "gf.csv"),
          str(files / "ordM.csv"), str(files / "ordF.csv"), str(files / "in.csv"), str(out)],
         env={"BM_MAX_PASSES": "1"})
    O = oracle.Oracle.from_pair(g)
    m = g["map0"].copy()
    O.first_improvement(m, 1)
    assert np.array_equal(_read(out, g["n"]), m)


def test_triple_one_round(files, cfg0):
    g = cfg0
    _run([os.path.join(BIN, "triple"), str(files / "gm.csv"), str(files / "gf.csv"), str(files / "in.csv"),
          str(files / "t.csv")], env={"BM_TRIPLE_ROUNDS": "1", "BM_PARTNERS": "64", "BM_SEED": "77"})
    O = oracle.Oracle.from_pair(g)
    m = g["map0"].copy()
    while O.sweep(m)["committed"]:
        pass
    O.triple_round(m, partners=64, seed=77)
    assert np.array_equal(_read(files / "t-rank0.csv", g["n"]), m)


def test_score_matching_prints_score(files, cfg0):
    g = cfg0
    stdout = _run([os.path.join(BIN, "score-matching"), str(files / "gm.csv"), str(files / "gf.csv"),
                   str(files / "in.csv")])
    O = oracle.Oracle.from_pair(g)
    assert stdout.strip().splitlines()[-1] == str(O.score(g["map0"]))


def _oracle_table(O, m):
    n = O.n
    t = np.zeros((n, n), np.int32)
    a, b = np.triu_indices(n, 1)
    d = O.all_deltas(m)
    t[a, b] = d
    t[b, a] = d
    return t


def test_greedy_feature_match_file(files, cfg0):
    g = cfg0
    out = files / "greedy.csv"
    _run([os.path.join(BIN, "greedy-feature-match"), str(files / "gm.csv"), str(files / "gf.csv"), str(out)])
    lines = open(out).read().splitlines()
    assert lines[0] == "Node G1,Node G2"
    got = np.array([[int(x) for x in ln.split(",")] for ln in lines[1:]])
    assert np.array_equal(got[:, 0], np.arange(1, g["n"] + 1))
    assert np.array_equal(got[:, 1], oracle.greedy_match(g)[1:])


def test_create_score_lookup_table(files, cfg0):
    g = cfg0
    out = files / "lookup.csv"
    _run([os.path.join(BIN, "create-score-lookup"), str(files / "gm.csv"), str(files / "gf.csv"),
          str(files / "in.csv"), str(out)])
    t = np.loadtxt(out, delimiter=",", dtype=np.int64)
    O = oracle.Oracle.from_pair(g)
    assert np.array_equal(t, _oracle_table(O, g["map0"]).astype(np.int16).astype(np.int64))


def test_score_lookup_descent_and_files(files, cfg0):
    g = cfg0
    (files / "in_lookup.csv").write_text("0\n")
    _run([os.path.join(BIN, "score-lookup"), str(files / "gm.csv"), str(files / "gf.csv"), str(files / "in.csv"),
          str(files / "in_lookup.csv"), str(files / "sl.csv"), str(files / "sl_lookup.csv")],
         env={"BM_ITERATIONS": "40"})
    lines = open(files / "sl.csv").read().splitlines()
    assert lines[0] == "Male Node ID,Female Node ID" and len(lines) == g["n"] + 1
    O = oracle.Oracle.from_pair(g)
    m = g["map0"].copy()
    O.best_swap_descent(m, 40)
    assert np.array_equal(_read(files / "sl.csv", g["n"]), m)
    t = np.loadtxt(files / "sl_lookup.csv", delimiter=",", dtype=np.int64)
    assert np.array_equal(t, _oracle_table(O, m).astype(np.int16).astype(np.int64))
    r = subprocess.run([os.path.join(BIN, "score-lookup"), str(files / "gm.csv"), str(files / "gf.csv"),
                        str(files / "in.csv"), str(files / "missing.csv"), str(files / "x.csv"),
                        str(files / "y.csv")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
