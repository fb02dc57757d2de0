"""CPU tests of the host side: the C ABI library, file formats, generator and
input validation (no GPU compute)."""
import os
import re

import numpy as np
import pytest

import bm
from conftest import ROOT


def test_library_exports_every_header_symbol():
    hdr = open(os.path.join(ROOT, "include", "bm.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)  # drop comments
    names = sorted(set(re.findall(r"\b(bm_\w+)\s*\(", hdr)))
    assert len(names) >= 20
    L = bm.lib()
    missing = [s for s in names if not hasattr(L, s)]
    assert not missing, missing


def test_generator_properties(cfg0):
    g = cfg0
    n = g["n"]
    assert len(g["src1"]) == 20000
    assert g["src1"].min() >= 1 and g["src1"].max() <= n and g["dst1"].max() <= n
    assert not (g["src1"] == g["dst1"]).any()
    k1 = g["src1"].astype(np.int64) * (n + 1) + g["dst1"]
    assert len(np.unique(k1)) == len(k1) and (np.diff(k1) > 0).all()  # sorted, no duplicates
    assert not (g["src2"] == g["dst2"]).any()
    k2 = g["src2"].astype(np.int64) * (n + 1) + g["dst2"]
    assert len(np.unique(k2)) == len(k2)
    assert len(g["src2"]) == 20000
    assert g["w1"].min() >= 1 and g["w1"].max() <= 5000 and g["w2"].min() >= 1
    assert sorted(g["map0"][1:]) == list(range(1, n + 1))
    assert sorted(g["pi"][1:]) == list(range(1, n + 1))
    # deterministic
    g2 = bm.generate(bm.gen_params())
    for k in ("src1", "dst1", "w1", "src2", "dst2", "w2", "map0"):
        assert np.array_equal(g[k], g2[k])
    g3 = bm.generate(bm.gen_params(seed=7))
    assert not np.array_equal(g["w1"], g3["w1"])


def test_csv_round_trip(tmp_path, cfg0):
    g = cfg0
    p = tmp_path / "g.csv"
    with open(p, "w") as f:
        f.write("from,to,weight\n")
        for s, d, w in zip(g["src1"], g["dst1"], g["w1"]):
            f.write(f"{s},{d},{w}\n")
        f.write("garbage line\n")
    s, d, w, mx = bm.read_graph_csv(str(p))
    assert np.array_equal(s, g["src1"]) and np.array_equal(d, g["dst1"]) and np.array_equal(w, g["w1"])
    assert mx == g["n"]
    mp = tmp_path / "m.csv"
    bm.write_mapping_csv(str(mp), g["map0"])
    txt = open(mp).read().splitlines()
    assert txt[0] == "Male Node ID,Female Node ID" and txt[1] == f"m1,f{g['map0'][1]}"
    m2, cnt = bm.read_mapping_csv(str(mp), g["n"])
    assert cnt == g["n"] and np.array_equal(m2, g["map0"])
    mp2 = tmp_path / "m2.csv"
    bm.write_mapping_csv(str(mp2), g["map0"], numeric=True)
    assert open(mp2).read().splitlines()[0] == "Male ID,Female ID"
    m3, _ = bm.read_mapping_csv(str(mp2), g["n"])
    assert np.array_equal(m3, g["map0"])


def test_mapping_reader_rejects_out_of_range(tmp_path):
    p = tmp_path / "m.csv"
    p.write_text("h\nm1,f2\nm9,f1\n")
    with pytest.raises(bm.BMError) as e:
        bm.read_mapping_csv(str(p), 5)
    assert e.value.status == bm.BM_E_INPUT


def test_missing_files_are_io_errors(tmp_path):
    with pytest.raises(bm.BMError) as e:
        bm.read_graph_csv(str(tmp_path / "nope.csv"))
    assert e.value.status == bm.BM_E_IO


@pytest.mark.parametrize("bad", ["id0", "id_big", "neg_w", "n_small", "overflow"])
def test_create_rejects_bad_input_before_touching_the_device(bad):
    s1, d1, w1 = [1, 2], [2, 3], [5, 6]
    n = 3
    if bad == "id0":
        s1 = [0, 2]
    elif bad == "id_big":
        d1 = [2, 4]
    elif bad == "neg_w":
        w1 = [5, -1]
    elif bad == "n_small":
        n = 1
    elif bad == "overflow":
        w1 = [2**30, 2**30]
    w2 = [2**30] if bad == "overflow" else [1]  # min(w1,w2) must be able to reach 2^30
    with pytest.raises(bm.BMError) as e:
        bm.Engine(n, s1, d1, w1, [1], [2], w2)
    want = bm.BM_E_OVERFLOW if bad == "overflow" else bm.BM_E_INPUT
    assert e.value.status == want


def test_cli_argument_errors_like_the_reference(tmp_path):
    """Usage and missing-file errors are reported before any device work."""
    import subprocess
    from conftest import PKG
    binq = os.path.join(PKG, "bin", "quick")
    bing = os.path.join(PKG, "bin", "graph-alignment-optimized")
    r = subprocess.run([binq, "only-one-arg"], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
    (tmp_path / "o.csv").write_text("node,order\n")
    r = subprocess.run([bing, "gm.csv", "gf.csv", str(tmp_path / "missing.csv"), str(tmp_path / "o.csv"),
                        "in.csv", "out.csv"], capture_output=True, text=True)
    assert r.returncode == 1 and "Error opening file" in r.stderr


def test_new_cli_argument_errors(tmp_path):
    """The greedy matcher and the lookup tools check their arguments and files
    before any device work, with the reference's exit codes."""
    import subprocess
    from conftest import PKG
    b = lambda name: os.path.join(PKG, "bin", name)
    r = subprocess.run([b("greedy-feature-match"), "a.csv"], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
    r = subprocess.run([b("greedy-feature-match"), str(tmp_path / "no1.csv"), str(tmp_path / "no2.csv"),
                        str(tmp_path / "out.csv")], capture_output=True, text=True)
    assert r.returncode == 1 and "Failed to load first graph" in r.stderr
    r = subprocess.run([b("create-score-lookup"), "a", "b"], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
    r = subprocess.run([b("score-lookup"), "a", "b", "c"], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
    r = subprocess.run([b("score-lookup"), "gm", "gf", "in", str(tmp_path / "missing_lookup.csv"), "o", "l"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "Failed to load lookup file" in r.stderr


def test_greedy_rejects_bad_edges_before_touching_the_device():
    g = dict(n=3, src1=[1, 4], dst1=[2, 3], w1=[1, 1], src2=[1], dst2=[2], w2=[1])
    with pytest.raises(bm.BMError) as e:
        bm.greedy_match(g)
    assert e.value.status == bm.BM_E_INPUT and "outside 1..3" in str(e.value)
    g = dict(n=3, src1=[1], dst1=[2], w1=[1], src2=[1], dst2=[2], w2=[-4])
    with pytest.raises(bm.BMError) as e:
        bm.greedy_match(g)
    assert e.value.status == bm.BM_E_INPUT and "negative weight" in str(e.value)
