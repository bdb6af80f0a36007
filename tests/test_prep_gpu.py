"""GPU peak picking (gx_pickpeaks_device) against the reference's own MS2 conversion
(golden .pbin) and against the oracle's restatement on seeded raw spectra with many
intensity ties, sizes from 0 to several hundred, and values outside the counted size."""

import os

import numpy as np
import pytest

import pyoracle
from conftest import has_gpu

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200
    return gicops_b200


def test_gpu_conversion_reproduces_reference_pbin(gx, tmp_path):
    out = tmp_path / "prep.pbin"
    q = gx.prep.convert_ms2(os.path.join(GOLDEN, "prep.ms2"), str(out))
    assert q.n == 160
    assert out.read_bytes() == open(os.path.join(GOLDEN, "prep.ms2.pbin"), "rb").read()


class _Raw:
    pass


def _random_raw(seed, nspec):
    rng = np.random.default_rng(seed)
    r = _Raw()
    sizes = rng.choice([0, 1, 2, 3, 50, 99, 100, 101, 150, 400, 600], size=nspec)
    extra = np.where(rng.random(nspec) < 0.05, rng.integers(1, 4, nspec), 0)   # values outside the size
    seg = np.zeros(nspec + 1, np.uint32)
    seg[1:] = np.cumsum(sizes + extra)
    n = int(seg[-1])
    r.seg, r.size, r.nspec, r.nvalues = seg, sizes.astype(np.uint32), nspec, n
    r.mz = rng.integers(10000, 200000, n).astype(np.int32)
    levels = rng.integers(0, 4, n)
    r.intn = np.where(levels == 0, rng.integers(0, 50, n),                    # coarse: many ties
                      np.where(levels == 1, rng.integers(0, 3, n) * 777,
                               rng.lognormal(6, 2, n).astype(np.int64))).astype(np.int32)
    r.prec = rng.uniform(500, 4000, nspec).astype(np.float32)
    r.charge = rng.integers(1, 5, nspec).astype(np.int32)
    r.rtime = rng.uniform(0, 100, nspec).astype(np.float32)
    return r


@pytest.mark.parametrize("seed", [1, 2])
def test_gpu_pickpeaks_matches_oracle(gx, seed):
    raw = _random_raw(seed, 3000)
    q = gx.prep.pickpeaks(raw)
    idx, mz, it = pyoracle.pickpeaks(raw.seg, raw.size, raw.mz, raw.intn)
    assert np.array_equal(q.idx, idx)
    assert np.array_equal(q.moz, mz) and np.array_equal(q.intn, it)


def test_gpu_pickpeaks_empty_and_errors(gx):
    raw = _random_raw(5, 1)
    raw.seg = np.zeros(1, np.uint32)
    raw.size = np.zeros(0, np.uint32)
    raw.nspec, raw.nvalues = 0, 0
    raw.mz = raw.intn = np.zeros(0, np.int32)
    raw.prec = raw.rtime = np.zeros(0, np.float32)
    raw.charge = np.zeros(0, np.int32)
    q = gx.prep.pickpeaks(raw)
    assert q.n == 0 and list(q.idx) == [0]
    import gicops_b200._native as N
    assert N.lib().gx_pickpeaks_device(1, 0, 0, 0, 0, 100000, 1000, 100, 0, 0, 0, None) == -3008
    assert N.lib().gx_pickpeaks_device(0, 0, 0, 0, 0, 100000, 1000, 0, 1, 0, 0, None) == -3002
