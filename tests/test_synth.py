"""Synthetic workload generator: determinism, the .pbin layout, and the peak
normalisation rules of the reference's preprocessing."""

import numpy as np

from gicops_b200 import synth


def test_database_is_deterministic_and_sorted():
    a = synth.make_database(30, seed=5)
    b = synth.make_database(30, seed=5)
    assert a.lengths == b.lengths
    for L in a.lengths:
        assert np.array_equal(a.peps[L], b.peps[L])
        rows = [bytes(r).replace(b"K", b"*").replace(b"L", b"K").replace(b"*", b"L") for r in a.peps[L]]
        assert rows == sorted(set(rows))
        assert min(a.peps) >= 6 and max(a.peps) <= 46


def test_tryptic_rules():
    res = np.frombuffer(b"AAAKPAAARAAAAAAKAAAAAAR", np.uint8).copy()
    db = synth.tryptic_digest(res, np.array([0]), np.array([len(res)]), missed=0, minlen=1, maxlen=46)
    got = sorted(bytes(r).decode() for L in db.lengths for r in db.peps[L])
    # no cleavage before P
    assert got == sorted(["AAAKPAAAR", "AAAAAAK", "AAAAAAR"])


def test_normalise_peaks():
    mz = np.arange(1, 8, dtype=np.int64) * 1000
    it = np.array([50, 400, 1000, 30, 2000, 999, 10], np.int64)
    m, i = synth.normalise_peaks(mz, it)
    # ascending intensity, top = base intensity, others scaled by truncation and cut at 1000
    assert i[-1] == synth.BASE_INT and m[-1] == 5000
    f = synth.BASE_INT / 2000.0
    # 10 * f = 500 < 1000 ends the scan; everything above it is kept
    assert list(i[:-1]) == [int(30 * f), int(50 * f), int(400 * f), int(999 * f), int(1000 * f)]
    assert list(m) == [4000, 1000, 2000, 6000, 3000, 5000]


def test_pbin_roundtrip(tmp_path):
    H = {7: (np.frombuffer(b"PEPTIDEKPEPTIDR", np.uint8)[:14].reshape(2, 7).copy(), np.array([0, 1], np.uint32),
             np.zeros(2, np.uint64), np.array([800.0, 810.0], np.float32))}
    q = synth.make_queries(H, 5, seed=1)
    p = tmp_path / "q.pbin"
    q.write_pbin(str(p))
    r = synth.QueryBatch.read_pbin(str(p))
    assert np.array_equal(r.idx, q.idx) and np.array_equal(r.moz, q.moz) and np.array_equal(r.intn, q.intn)
    assert np.array_equal(r.prec, q.prec) and np.array_equal(r.charge, q.charge)
    s = q.subset([3, 1])
    assert s.n == 2 and np.array_equal(s.moz[: s.idx[1]], q.moz[q.idx[3]:q.idx[4]])


def test_concat_keeps_spectra_and_offsets():
    import gicops_b200 as gx
    db = gx.synth.make_database(60, seed=3)
    H = gx.HostIndex.build(db, maxz=1, ions=False)
    a = gx.synth.make_queries(H.entries_by_len(), 7, seed=1, window="mixed")
    b = gx.synth.make_queries(H.entries_by_len(), 5, seed=2)
    c = gx.synth.QueryBatch.concat([a, b])
    assert c.n == 12 and c.idx[0] == 0 and c.idx[-1] == len(a.moz) + len(b.moz)
    for i in range(a.n):
        assert np.array_equal(c.moz[c.idx[i]:c.idx[i + 1]], a.moz[a.idx[i]:a.idx[i + 1]])
    for i in range(b.n):
        j = a.n + i
        assert np.array_equal(c.intn[c.idx[j]:c.idx[j + 1]], b.intn[b.idx[i]:b.idx[i + 1]])
    assert np.array_equal(c.prec, np.concatenate([a.prec, b.prec]))
    assert np.array_equal(np.isnan(c.dM[a.n:]), np.ones(b.n, bool))   # b had no per-spectrum tolerances
