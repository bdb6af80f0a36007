"""GPU query path vs the oracle where every candidate of a window is a PSM.

A database of 3,000 length-20 peptides that share their first 15 residues: a spectrum made
of the shared b ions matches every one of them with at least 15 ions, so in the first tile
of each spectrum (the heap not yet full) every candidate enters the heap.  Each warp of the
batched kernel then keeps one entrant per candidate of its range, the longest entrant lists
the kernel can produce, at the default tile and at two narrower ones (several sub-tiles per
block).  Counts, histograms and heap arrays must be bit-exact against the oracle, as in the
golden cases.
"""

import numpy as np
import pytest

import pyoracle
from conftest import assert_same, has_gpu
from gicops_b200 import synth

PREFIX = b"GASPVTLNDQEFYWH"   # 15 residues, no K/R
RESIDUES = b"ACDEFGHILNPQSTVWY"
NPEP = 3000
DM = 500.0
# the spectra's own entries (the best PSM of each): some at the positions 128-383 of the first
# tile (the far end of the first warps' ranges) and of a second sub-tile
DENSE_PICKS = [0, 150, 200, 300, 700, 1500, 2150, NPEP - 1]


def dense_database():
    rng = np.random.Generator(np.random.PCG64(5))
    seen = set()
    while len(seen) < NPEP:
        seen.add(bytes(rng.choice(np.frombuffer(RESIDUES, np.uint8), 4)) + b"K")
    rows = sorted(PREFIX + s for s in seen)
    return synth.Database(peps={20: np.frombuffer(b"".join(rows), np.uint8).reshape(NPEP, 20).copy()})


def dense_queries(H, picks):
    """Spectra of the given entries: the 15 shared b ions and the first four y ions (charge
    1), intensities of the preprocessed range."""
    x = H.lengths[0]
    mtab = synth.residue_mass_table()
    moz, intn, idx = [], [], [0]
    for k, e in enumerate(picks):
        seq = bytes(x["seqs"][int(x["entries"]["seqid"][e])])
        ions = synth.fragment_mz(seq, 0, None, (1,), mtab)
        mz = np.concatenate([ions[:15], ions[19:23]])
        m = np.floor(mz * synth.SCALE).astype(np.int32)
        it = (np.arange(len(m), dtype=np.int32) * 3000 + 10000 + 500 * k).astype(np.int32)
        moz.append(m)
        intn.append(it)
        idx.append(idx[-1] + len(m))
    n = len(picks)
    return synth.QueryBatch(np.array(idx, np.uint32), np.concatenate(moz), np.concatenate(intn),
                            x["mass"][np.asarray(picks)].astype(np.float32), np.full(n, 2, np.int32),
                            np.zeros(n, np.float32))


@pytest.fixture(scope="module")
def dense():
    H = synth_index()
    q = dense_queries(H, DENSE_PICKS)
    o, oh = pyoracle.search(H.lengths, q, pyoracle.Params(dM=DM), hist=True)
    return H, q, o, oh


def synth_index():
    import gicops_b200 as gx
    return gx.HostIndex.build(dense_database(), maxz=1)


def test_dense_workload_makes_every_candidate_a_psm(dense):
    """CPU check of the workload: the window of each spectrum holds all 3,000 entries and the
    oracle counts every one of them as a candidate PSM."""
    H, q, o, oh = dense
    assert H.lengths[0]["N"] == NPEP
    assert np.all(o["cpsms"] == NPEP), o["cpsms"]


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [11264, 4096, 1952])
def test_gpu_dense_entrants(dense, tile):
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200 as gx
    H, q, o, oh = dense
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    s.tiles = dict(s.tiles, tile=tile)
    for topmatches in (5, 31):
        r = s.search(q, gx.SearchParams(dM=DM, topmatches=topmatches, expect_max=1e300), heap=True, hist=True)
        if topmatches == 5:
            assert_same(r.result, r.heap, r.hist, o, oh, None)
        else:
            o2, oh2 = pyoracle.search(H.lengths, q, pyoracle.Params(dM=DM, topmatches=topmatches), hist=True)
            assert_same(r.result, r.heap, r.hist, o2, oh2, None)
