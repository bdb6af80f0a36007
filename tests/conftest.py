import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN = os.path.join(ROOT, "tests", "golden")
# e-values (device log10/pow against the host C library): relative tolerance
E_RTOL = 1e-9
CASES = ["closed_small", "closed_1k", "open_mox", "mixed_window"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_case(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    peps = {int(k.split("_")[1]): z[k] for k in z.files if k.startswith("peps_")}
    d = {k: z[k] for k in z.files if not k.startswith("peps_")}
    d["meta"] = meta
    d["peps"] = peps
    return d


def case_queries(c: dict):
    from gicops_b200.synth import QueryBatch
    dM = c["q_dM"] if len(c["q_dM"]) else None
    return QueryBatch(c["q_idx"], c["q_moz"], c["q_intn"], c["q_prec"], c["q_charge"],
                      np.zeros(len(c["q_prec"]), np.float32), dM)


def case_index(c: dict, ions: bool = True):
    """Index of a golden case built by the library's host builder (entries only when
    ions is False)."""
    import gicops_b200 as gx
    from gicops_b200.synth import Database
    m = c["meta"]
    db = Database(peps=c["peps"], nproteins=m["nproteins"])
    mods = [tuple(x) for x in m["mods"]]
    return gx.HostIndex.build(db, maxz=m["maxz"], mods=mods, nmods=m["nmods"], min_mass=m["min_mass"],
                              max_mass=m["max_mass"], ions=ions)


def oracle_params(c: dict):
    import pyoracle
    m = c["meta"]
    return pyoracle.Params(dM=m["dM"], dF=m["dF"], topmatches=m["topmatches"], min_cpsm=m["min_cpsm"],
                           min_shp=m["min_shp"], expect_max=1e300)


def search_params(c: dict, **kw):
    import gicops_b200 as gx
    m = c["meta"]
    return gx.SearchParams(dM=m["dM"], dF=m["dF"], topmatches=m["topmatches"], min_cpsm=m["min_cpsm"],
                           min_shp=m["min_shp"], expect_max=1e300, **kw)


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(name):
        if name not in cache:
            c = load_case(name)
            c["index"] = case_index(c)
            c["queries"] = case_queries(c)
            cache[name] = c
        return cache[name]
    return get


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _heap_cells(arr):
    return [(float(c["hyperscore"]), int(c["psid"]), int(c["idxoffset"]), int(c["sharedions"]), int(c["totalions"]))
            for c in arr]


def assert_same(res, heap, hist, ores, ohist, cap):
    """GPU results against the oracle: bit-exact counts, status bits 1/2/4, histograms, heap
    arrays, top PSM and fit region; slope and e-values within tolerance; and, when `cap`
    holds the compiled reference's capture, the PSMs the reference reported."""
    assert np.array_equal(res["cpsms"], ores["cpsms"])
    assert np.array_equal(res["status"] & 7, ores["status"] & 7)
    assert np.array_equal(hist, ohist)
    for i in range(len(res)):
        n = int(ores["heap_size"][i])
        assert _heap_cells(heap[i][:n]) == _heap_cells(ores["heap"][i][:n]), i
        assert np.all(heap[i][n:]["psid"] == 0)
    m = (ores["status"] & 1) != 0
    for f in ("psid", "idxoffset", "sharedions", "totalions"):
        assert np.array_equal(res["top"][f][m], ores["top"][f][m]), f
    assert np.array_equal(res["top"]["hyperscore"][m].view(np.uint32), ores["top"]["hyperscore"][m].view(np.uint32))
    for f in ("maxhyp", "mu", "beta", "stt1", "end1"):
        assert np.array_equal(res[f][m], ores[f][m]), f
    ok = m & np.isfinite(ores["e_x"])
    np.testing.assert_allclose(res["e_x"][ok], ores["e_x"][ok], rtol=E_RTOL)
    np.testing.assert_allclose(res["slope"][ok], ores["slope"][ok], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(res["e_fp64"][ok], ores["e_fp64"][ok], rtol=E_RTOL)
    if cap is not None:
        rep = (res["status"] & 2) != 0
        assert np.array_equal(rep, cap["cap_reported"] == 1)
        assert np.array_equal(res["top"]["psid"][rep], cap["cap_psid"][rep])
        assert np.array_equal(res["top"]["idxoffset"][rep], cap["cap_idxoffset"][rep])
        assert np.array_equal(res["top"]["hyperscore"][rep].view(np.uint32), cap["cap_hyperscore"][rep].view(np.uint32))
        np.testing.assert_allclose(res["e_x"][rep], cap["cap_e_x"][rep], rtol=E_RTOL)


# ---- a database whose peptide lengths span several entry blocks ------------------------
# 5,000 proteins with Met oxidation <= 2 give up to 35,522 entries per length: precursor
# windows over three or more 11,264-entry blocks of the batched kernel's block layout and
# over more than four 8,192-candidate tiles of the plain path.  (The golden cases hold at
# most 5,886 entries per length: one block, one tile.)
MULTIBLOCK = dict(nproteins=5000, seed=31, mods=[("M", 15.9949, 2)], nmods=2, dM=500.0)
BLOCK_ENTRIES = 11264
PLAIN_TILE = 8192
_multiblock = {}


def multiblock_index(maxz: int):
    """Host index of the multi-block database with fragment charges 1..maxz (cached)."""
    if maxz not in _multiblock:
        import gicops_b200 as gx
        w = MULTIBLOCK
        db = gx.synth.make_database(w["nproteins"], seed=w["seed"])
        _multiblock[maxz] = gx.HostIndex.build(db, maxz=maxz, mods=w["mods"], nmods=w["nmods"])
    return _multiblock[maxz]


def multiblock_queries(H, n: int, seed: int, **kw):
    """Open-search spectra of the multi-block database (30-150 peaks, 20-80% ion retention)."""
    import gicops_b200 as gx
    args = dict(charges=(2, 4), frag_charge2=H.maxz >= 2, keep_p=(0.2, 0.8), noise_mode="fill",
                npeaks_range=(30, 150))
    args.update(kw)
    return gx.synth.make_queries(H.entries_by_len(), n, seed=seed, **args)


def many_interval_spectra(H, n: int, pairs: int, seed: int):
    """Spectra of database peptides (their b/y ions only) plus `pairs` pairs of noise peaks
    6 bins apart, the pairs at least 40 bins from each other: with the +-5-bin fragment
    window each pair makes three merged bin intervals, so 86 pairs or more give a spectrum
    more than 256 intervals."""
    from gicops_b200.synth import QueryBatch
    base = multiblock_queries(H, n, seed, keep_p=(0.6, 0.6), npeaks_range=(1, 1))
    rng = np.random.default_rng(seed)
    idx, moz, intn = [0], [], []
    for s in range(n):
        a, b = int(base.idx[s]), int(base.idx[s + 1])
        anchors = 10000 + 40 * rng.choice(4700, size=pairs, replace=False)
        noise = np.concatenate([anchors, anchors + 6]).astype(np.int32)
        m = np.concatenate([base.moz[a:b], noise])
        it = np.concatenate([base.intn[a:b], rng.integers(1000, 50000, size=len(noise)).astype(np.int32)])
        perm = rng.permutation(len(m))
        moz.append(m[perm])
        intn.append(it[perm])
        idx.append(idx[-1] + len(m))
    return QueryBatch(np.array(idx, np.uint32), np.concatenate(moz).astype(np.int32),
                      np.concatenate(intn).astype(np.int32), base.prec.copy(), base.charge.copy(),
                      np.zeros(n, np.float32))


def concat_queries(*qs):
    from gicops_b200.synth import QueryBatch
    idx = [np.zeros(1, np.int64)]
    off = 0
    for q in qs:
        idx.append(q.idx[1:].astype(np.int64) + off)
        off += int(q.idx[-1])
    dm = None
    if any(q.dM is not None for q in qs):
        dm = np.concatenate([q.dM if q.dM is not None else np.full(q.n, np.nan) for q in qs])
    return QueryBatch(np.concatenate(idx).astype(np.uint32), np.concatenate([q.moz for q in qs]),
                      np.concatenate([q.intn for q in qs]), np.concatenate([q.prec for q in qs]),
                      np.concatenate([q.charge for q in qs]), np.concatenate([q.rtime for q in qs]), dm)


def window_spans(H, q, dM: float):
    """Per (spectrum, length): the candidate window's entry count and the number of
    BLOCK_ENTRIES blocks it touches (float bounds as the reference computes them)."""
    n = np.zeros((q.n, H.nlen), np.int64)
    blocks = np.zeros((q.n, H.nlen), np.int64)
    for s in range(q.n):
        d = dM if q.dM is None or np.isnan(q.dM[s]) else float(q.dM[s])
        p1, p2 = np.float32(float(q.prec[s]) - d), np.float32(float(q.prec[s]) + d)
        for i, x in enumerate(H.lengths):
            lo = int(np.searchsorted(x["mass"], p1, side="left"))
            hi = int(np.searchsorted(x["mass"], p2, side="right")) - 1
            if hi >= lo:
                n[s, i] = hi - lo + 1
                blocks[s, i] = hi // BLOCK_ENTRIES - lo // BLOCK_ENTRIES + 1
    return n, blocks


def merged_intervals(q, dF: int = 5, upper: float = 5000 * 100 - 1 - 5):
    """Per spectrum: the number of disjoint bin intervals its probed peaks' windows
    [mz - dF, mz + dF] merge into (runs of bins with a constant set of covering peaks)."""
    out = np.zeros(q.n, np.int64)
    for s in range(q.n):
        m = q.moz[int(q.idx[s]):int(q.idx[s + 1])].astype(np.int64)
        m = np.sort(m[(m > dF) & (m < upper)])
        # runs between consecutive window starts/ends that some window covers
        pos = np.unique(np.concatenate([m - dF, m + dF + 1]))
        cov = np.searchsorted(m - dF, pos[:-1], side="right") - np.searchsorted(m + dF + 1, pos[:-1], side="right")
        out[s] = int(np.count_nonzero(cov > 0))
    return out
