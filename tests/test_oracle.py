"""The oracle (C restatement of the reference's CPU query path) pinned against the
reference's own outputs captured in tests/golden, plus known-answer tests written
independently of both."""

import math

import numpy as np
import pytest

import pyoracle
from conftest import CASES, case_index, case_queries, load_case, oracle_params


@pytest.mark.parametrize("case", CASES)
def test_oracle_bit_exact_vs_reference(golden, case):
    c = golden(case)
    res, hist = pyoracle.search(c["index"].lengths, c["queries"], oracle_params(c), hist=True)
    rep = (res["status"] & 2) != 0
    assert np.array_equal(rep, c["cap_reported"] == 1)
    m = rep
    assert m.sum() > 0
    top = res["top"][m]
    assert np.array_equal(top["psid"], c["cap_psid"][m])
    assert np.array_equal(top["idxoffset"], c["cap_idxoffset"][m])
    assert np.array_equal(top["sharedions"], c["cap_sharedions"][m])
    assert np.array_equal(top["totalions"], c["cap_totalions"][m])
    assert np.array_equal(top["hyperscore"].view(np.uint32), c["cap_hyperscore"][m].view(np.uint32))
    assert np.array_equal(res["cpsms"][m], c["cap_npsms"][m].astype(np.int32))
    assert np.array_equal(res["e_x"][m].view(np.uint64), c["cap_e_x"][m].view(np.uint64))
    # histogram mass equals the candidate count
    assert np.array_equal(hist.sum(axis=1), res["cpsms"].astype(np.uint64))


def test_lgfact_table():
    t = pyoracle.lgfact()
    acc = 0.0
    for i in range(2, 81):
        acc = math.log10(i) + acc
        assert t[i] == acc
    assert t[0] == 0.0 and t[1] == 0.0


def test_heap_capacity():
    assert pyoracle.heap_capacity(5) == 7
    assert pyoracle.heap_capacity(10) == 15
    assert pyoracle.heap_capacity(1) == 0
    assert pyoracle.heap_capacity(0) == 0


def _tiny_index():
    """3 peptides of length 4, maxz 1 (speclen 6), hand-placed ion bins."""
    nb = 500001
    speclen = 6
    # ions per peptide: b1 b2 b3 y1 y2 y3 (positions 0..5)
    bins = {
        0: [10000, 20000, 30000, 11000, 21000, 31000],
        1: [10000, 20002, 30100, 11000, 22000, 31000],
        2: [10003, 20000, 30000, 11500, 21000, 32000],
    }
    ids = []
    for p, bl in bins.items():
        for pos, b in enumerate(bl):
            ids.append((b, p * speclen + pos))
    ids.sort()
    iA = np.array([i for _, i in ids], np.uint32)
    cnt = np.zeros(nb, np.int64)
    for b, _ in ids:
        cnt[b] += 1
    bA = np.zeros(nb, np.uint32)
    bA[1:] = np.cumsum(cnt)[:-1]
    mass = np.array([500.0, 500.5, 501.0], np.float32)
    return [dict(L=4, N=3, speclen=speclen, mass=mass, bA=bA, iA=iA)], bins


def test_known_answer_scorecard():
    """bc/yc/ibc/iyc written out by hand for a 3-peptide index."""
    lens, bins = _tiny_index()
    moz = np.array([10001, 20000, 30000, 11000, 31002, 21000], np.int32)
    intn = np.array([100, 200, 300, 400, 500, 600], np.int32)
    cands = pyoracle.candidates(lens, moz, intn, 500.5, 10.0, pyoracle.Params(dM=10.0, dF=5))
    got = {int(c["psid"]): (int(c["bc"]), int(c["yc"]), int(c["ibc"]), int(c["iyc"])) for c in cands}
    # expected, peak by peak (window +-5 bins):
    # p0: b 10000 (10001), 20000 (20000), 30000 (30000); y 11000, 21000 (21000), 31000 (31002)
    # p1: b 10000 (10001), 20002 (20000);                 y 11000, 31000 (31002)
    # p2: b 10003 (10001), 20000, 30000;                  y 21000 (21000) only
    exp = {
        0: (3, 3, 100 + 200 + 300, 400 + 600 + 500),
        1: (2, 2, 100 + 200, 400 + 500),
        2: (3, 1, 100 + 200 + 300, 600),
    }
    assert got == exp
    # hyperscore of peptide 0 from its definition
    lg = pyoracle.lgfact()
    h0 = np.float32(lg[3] + lg[3] + math.log10(1 + 600) + math.log10(1 + 1500) - 4)
    h = {int(c["psid"]): c["h"] for c in cands}
    assert h[0] == h0
    assert h[1] == np.float32(lg[2] + lg[2] + math.log10(301) + math.log10(901) - 4)


def test_window_edges():
    lens, _ = _tiny_index()
    x = lens[0]
    assert pyoracle.window(x, 500.5, 0.5) == (0, 2)
    assert pyoracle.window(x, 500.5, 0.25) == (1, 1)
    assert pyoracle.window(x, 499.0, 0.5) == (1, 0)       # below every mass: skipped
    assert pyoracle.window(x, 502.0, 0.5) == (1, 0)       # above every mass: skipped
    assert pyoracle.window(x, 500.5, -1.0) == (1, 0)      # negative tolerance: skipped
    assert pyoracle.window(x, float("nan"), 1.0) == (1, 0)


def test_tailfit_short_branches():
    """Tail-fit branches by histogram length (sizes 0..4) against a direct restatement."""
    h = np.zeros(802)
    # one populated bin below the top -> stt1 == end1, region widened by one
    h[100] = 3
    r = pyoracle.tailfit(h, 4, 150)
    assert (r["stt1"], r["end1"]) == (100, 101)
    # two points, n=2 fit: slope through both survival values
    s0 = math.log10(1 - 3 / 4)
    s1 = s0  # bin 101 is empty: cumulative unchanged
    assert r["slope"] == 0.0 and r["icpt"] == (s0 + s1) / 2
    # a three-point region uses the 22% mark only
    h = np.zeros(802)
    h[[10, 11, 12]] = [5, 3, 1]
    r = pyoracle.tailfit(h, 10, 30)
    assert (r["stt1"], r["end1"]) == (10, 12)
    assert r["mu"] == int(r["slope"] * 1e6)
    e = 10 * 10 ** ((r["mu"] / 1e6) * 30 + r["beta"] / 1e6)
    assert r["e_x"] == pytest.approx(e, rel=1e-12)


def test_oracle_min_cpsm_zero_acts_as_one():
    """A spectrum without candidate PSMs has no top score, so no e-value even at min_cpsm 0."""
    c = load_case("open_mox")
    H, q = case_index(c), case_queries(c)
    a, ha = pyoracle.search(H.lengths, q, pyoracle.Params(dM=500.0, min_shp=16, min_cpsm=0), hist=True)
    b, hb = pyoracle.search(H.lengths, q, pyoracle.Params(dM=500.0, min_shp=16, min_cpsm=1), hist=True)
    assert a.tobytes() == b.tobytes() and np.array_equal(ha, hb)
    none = a["cpsms"] == 0
    assert none.sum() > 10 and np.all(a["status"][none] == 0) and np.all((a["status"][~none] & 1) != 0)
