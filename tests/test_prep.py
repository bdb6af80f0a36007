"""Query preprocessing (MS2 text -> peak-picked query batch -> .pbin) on the CPU.

The golden ``prep.ms2.pbin`` was written by the reference's own conversion
(MSQuery::convertAndprepMS2bin, compiled from its sources: tests/golden/
make_ms2_golden.py).  The library's MS2 reader followed by the oracle's peak picking
(the reference's pickpeaks and key-value quicksort, restated in C) must reproduce it
byte for byte; the reader's line rules are checked on small files."""

import os

import numpy as np
import pytest

import pyoracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _oracle_batch(raw):
    from gicops_b200.synth import QueryBatch
    idx, mz, it = pyoracle.pickpeaks(raw.seg, raw.size, raw.mz, raw.intn)
    return QueryBatch(idx, mz, it, raw.prec.copy(), raw.charge.copy(), raw.rtime.copy())


def test_reader_and_oracle_reproduce_reference_pbin(tmp_path):
    import gicops_b200 as gx
    raw = gx.prep.read_ms2(os.path.join(GOLDEN, "prep.ms2"))
    assert raw.nspec == 160
    q = _oracle_batch(raw)
    out = tmp_path / "o.pbin"
    q.write_pbin(str(out))
    ref = open(os.path.join(GOLDEN, "prep.ms2.pbin"), "rb").read()
    got = out.read_bytes()
    assert len(got) == len(ref)
    assert got == ref
    # the fixture reaches the cases it is meant to: the 100-peak cut, empty spectra,
    # an all-zero spectrum, values before the first S line
    lens = np.diff(q.idx.astype(np.int64))
    assert lens.max() == 100 and (lens == 0).sum() >= 1
    assert raw.seg[1] - raw.seg[0] == raw.size[0] + 2


def _read_text(tmp_path, text):
    import gicops_b200 as gx
    p = tmp_path / "t.ms2"
    p.write_bytes(text.encode())
    return gx.prep.read_ms2(str(p))


def test_reader_line_rules(tmp_path):
    raw = _read_text(tmp_path, "H\tx\n100.5 7\nS\t1\t1\t500\nZ\t0\t1001.25\nI\tRTime\t-3\n"
                               "200.256 10.5\n300.1\t99\nD\tq\n400 1e3\r\nS\t2\nZ\nI\tRTime\t12.5\n150 2\n")
    assert raw.nspec == 2
    assert list(raw.seg) == [0, 4, 5] and list(raw.size) == [3, 1]   # the line before S joins spectrum 0
    assert list(raw.mz) == [int(x * 100.0) for x in (100.5, 200.256, 300.1, 400.0, 150.0)]
    # tab-separated line: one field, intensity "0.01" -> 1; "1e3" -> 100000
    assert list(raw.intn) == [700, 1050, 1, 100000, 200]
    assert list(raw.charge) == [1, 1]                      # max(1, 0); empty Z line -> "1"
    assert raw.prec[0] == np.float32(1001.25) and raw.prec[1] == np.float32(0.01)
    assert list(raw.rtime) == [0.0, 12.5]                  # max(0, -3)


def test_reader_empty_file_and_errors(tmp_path):
    import gicops_b200 as gx
    raw = _read_text(tmp_path, "")
    assert raw.nspec == 1 and raw.nvalues == 0 and list(raw.size) == [0]
    with pytest.raises(gx.GxError) as e:
        gx.prep.read_ms2(str(tmp_path / "missing.ms2"))
    assert e.value.code == -3006


def test_oracle_pickpeaks_rules():
    # ties: the reference's quicksort order decides which tied peaks pass the cut
    rng = np.random.default_rng(3)
    it = rng.choice([5, 9, 9, 9, 12], size=240).astype(np.int32) * 1000
    mz = np.arange(240, dtype=np.int32) + 1000
    idx, m, i = pyoracle.pickpeaks(np.array([0, 240], np.uint32), np.array([240], np.uint32), mz, it)
    assert idx[1] == 100 and i[-1] == 100000 and np.all(np.diff(i) >= 0)
    # all intensities 0: x86 conversion of 0 * inf gives INT32_MIN, below min_int
    idx, m, i = pyoracle.pickpeaks(np.array([0, 5], np.uint32), np.array([5], np.uint32),
                                   np.arange(5, dtype=np.int32), np.zeros(5, np.int32))
    assert idx[1] == 1 and i[0] == 100000
