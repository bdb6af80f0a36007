"""GPU query path vs the oracle on an index whose peptide lengths span several entry
blocks (conftest.MULTIBLOCK: up to 35,522 entries per length).  These are the code paths
that an open search of a large database runs on nearly every spectrum and that the
golden cases (one block, one tile per length) never reach:

* windows over two or more 11,264-entry blocks in the batched kernel, with the next
  block's bin offsets loaded one tile ahead and its span table built while the current
  tile is scored;
* the 12-byte scorecard's second sub-tile of a block (the same span table, restreamed), and
  narrower tiles (several sub-tiles per block in either scorecard), with more than 256
  intervals too (the span table rebuilt per 256-interval chunk for every sub-tile);
* spectra with more than 256 merged bin intervals (span tables built per 256-interval
  chunk, offsets not carried), in the 8-byte and in the 12-byte scorecard;
* the plain path's candidate tiles after the first 8,192 entries of a window;
* the pipelined kernel (two scorecard tiles per CTA) over the same windows;
* per-spectrum precursor tolerances (half the spectra at +-10 ppm).

The comparison is the same as for the golden cases (conftest.assert_same): counts,
histograms and heap arrays bit-exact, e-values within 1e-9 relative.  A CPU test checks
that the workload does reach those paths.
"""

import numpy as np
import pytest

import pyoracle
from conftest import (MULTIBLOCK, PLAIN_TILE, assert_same, concat_queries, has_gpu, many_interval_spectra,
                      merged_intervals, multiblock_index, multiblock_queries, window_spans)

DM = MULTIBLOCK["dM"]


def workload(maxz: int):
    H = multiblock_index(maxz)
    q_open = multiblock_queries(H, 160, seed=41)
    q_mixed = multiblock_queries(H, 48, seed=42, window="mixed")
    q_many = many_interval_spectra(H, 6, pairs=150 if maxz >= 2 else 95, seed=43)
    return H, concat_queries(q_open, q_mixed, q_many), q_many.n


def test_multiblock_workload_reaches_the_paths():
    """CPU check of the workload itself: windows over >= 3 blocks and > 4 plain tiles,
    and spectra with more than 256 intervals that fit the 8-byte scorecard at maxz 1."""
    for maxz in (1, 2):
        H, q, nmany = workload(maxz)
        n, blocks = window_spans(H, q, DM)
        assert max(x["N"] for x in H.lengths) > 3 * 11264
        assert (blocks >= 3).any(axis=1).sum() > 0.3 * q.n
        assert (n > 4 * PLAIN_TILE).any(axis=1).sum() > 0.3 * q.n
        iv = merged_intervals(q)
        assert np.all(iv[-nmany:] > 256), iv[-nmany:]
        npk = np.diff(q.idx.astype(np.int64))[-nmany:]
        if maxz == 1:
            assert np.all(npk <= 255)                  # packed-scorecard guard: maxz * peaks <= 255
        else:
            assert np.all(npk * maxz > 255)            # these take the 12-byte scorecard
        assert q.dM is not None and np.isfinite(q.dM).sum() > 10


@pytest.fixture(scope="module")
def gx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200
    return gicops_b200


@pytest.fixture(scope="module")
def searched():
    """Oracle results per maxz (cached for the parametrised tests)."""
    cache = {}

    def get(maxz):
        if maxz not in cache:
            H, q, nmany = workload(maxz)
            o, oh = pyoracle.search(H.lengths, q, pyoracle.Params(dM=DM), hist=True)
            cache[maxz] = (H, q, nmany, o, oh)
        return cache[maxz]
    return get


@pytest.mark.gpu
@pytest.mark.parametrize("maxz", [1, 2])
@pytest.mark.parametrize("flags", [0, 1, 2, "piped", "narrow"], ids=["default", "wide", "plain", "piped", "narrow"])
def test_gpu_multiblock(gx, searched, maxz, flags):
    H, q, nmany, o, oh = searched(maxz)
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    if flags == "piped":   # the pipelined kernel for the 8-byte spectra, the batched one for the rest
        s.tiles = dict(s.tiles, pipeline=1)
        flags = 0
    elif flags == "narrow":   # tiles of 4,096 candidates: several sub-tiles per block in both scorecards
        s.tiles = dict(s.tiles, tile=4096)
        flags = 0
    r = s.search(q, gx.SearchParams(dM=DM, expect_max=1e300, flags=flags), heap=True, hist=True)
    assert_same(r.result, r.heap, r.hist, o, oh, None)
    assert not np.any(r.result["status"] & 4)
    wide = (r.result["status"] & 8) != 0
    if flags == 1:
        assert wide.all()
    elif flags == 0:
        # the many-interval spectra: 8-byte scorecard at maxz 1, 12-byte at maxz 2
        assert np.all(wide[-nmany:] == (maxz >= 2))
    assert (o["status"] & 1).sum() > 0.7 * q.n   # +-10 ppm spectra at maxz 1 often have < 4 candidate PSMs


@pytest.mark.gpu
def test_gpu_multiblock_other_heaps(gx, searched):
    """Other heap capacities and shared-peak thresholds over the multi-block windows."""
    H, q, nmany, _, _ = searched(2)
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    for tm, shp in [(10, 4), (31, 6)]:
        r = s.search(q, gx.SearchParams(dM=DM, topmatches=tm, min_shp=shp, expect_max=1e300), heap=True, hist=True)
        o, oh = pyoracle.search(H.lengths, q, pyoracle.Params(dM=DM, topmatches=tm, min_shp=shp), hist=True)
        assert_same(r.result, r.heap, r.hist, o, oh, None)
