"""Search API: the counterpart of the reference's query-path boundary.

``Searcher`` mirrors ``hcp::gpu::cuda::s3::{initialize, search, deinitialize}``
(source/core/include/cuda/superstep3/kernel.hpp:88-100) followed by
``s4::processResults`` (source/core/cuda/superstep4/kernel.cu:491-596): a batch of
spectra in the ``Queries<int>`` layout goes in, per-spectrum results (top PSM,
candidate count, tail-fit parameters, e-value) come out.  Errors raise
``GxError`` carrying the reference's status code (source/core/include/slmerr.h).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .index import DeviceIndex
from .synth import QueryBatch


@dataclass
class SearchParams:
    """The ``gParams`` fields the query path reads (source/core/include/slm_dsts.h:349-516)."""

    dM: float = 10.0          # precursor tolerance, Da
    dF: int = 5               # fragment tolerance, bins of 1/scale Da
    scale: int = 100
    max_mass: float = 5000.0
    min_shp: int = 4
    min_cpsm: int = 4
    topmatches: int = 5
    expect_max: float = 20.0
    flags: int = 0

    def c(self) -> N.Params:
        return N.Params(self.dM, self.dF, self.scale, self.max_mass, self.min_shp, self.min_cpsm, self.topmatches,
                        self.flags, self.expect_max)

    @property
    def heap_cap(self) -> int:
        return int(N.lib().gx_heap_capacity(self.topmatches))


@dataclass
class SearchResults:
    result: np.ndarray                 # RESULT_DTYPE [nspec]
    heap: np.ndarray | None = None     # CELL_DTYPE [nspec, heap_cap] final top-K heap arrays
    hist: np.ndarray | None = None     # uint32 [nspec, 802] score histograms

    @property
    def reported(self) -> np.ndarray:
        """Spectra whose PSM the reference prints (e-value below expect_max)."""
        return (self.result["status"] & 2) != 0


class Searcher:
    """Workspace + entry points for one host thread on one device index."""

    def __init__(self, index: DeviceIndex, max_spec: int, max_peaks: int):
        self.index = index
        self.max_spec = max_spec
        self.max_peaks = max_peaks
        self.handle = C.c_void_p()
        N.check(N.lib().gx_workspace_create(index.handle, max_spec, max_peaks, C.byref(self.handle)))

    def close(self) -> None:
        if self.handle:
            N.lib().gx_workspace_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tail(self, model, sparse_below: int = 500) -> None:
        """Apply a trained gicops_b200.tail.TailModel to queries with fewer than
        ``sparse_below`` candidate PSMs in every batched search (None detaches)."""
        N.check(N.lib().gx_workspace_set_tail(self.handle, model.handle if model else None, sparse_below))
        self._tail = model   # keep the model alive while attached

    def set_graph(self, on: bool = True) -> None:
        """Capture the batched launch sequence in CUDA graphs and replay them
        (gx_workspace_set_graph); off releases them."""
        N.check(N.lib().gx_workspace_set_graph(self.handle, int(on)))

    @property
    def tiles(self) -> dict:
        """Launch shape of the batched path (gx_tiles)."""
        t = N.Tiles()
        N.check(N.lib().gx_workspace_get_tiles(self.handle, C.byref(t)))
        return t.as_dict()

    @tiles.setter
    def tiles(self, t: dict) -> None:
        c = N.Tiles(t["chunks_per_lane"], t["ctas_per_sm"], t["tile"], t["sorted"], t.get("pipeline", 0))
        N.check(N.lib().gx_workspace_set_tiles(self.handle, C.byref(c)))

    def autotune(self, q_dev: dict, params: SearchParams, reps: int = 3, use_cache: bool = True,
                 stream: int = 0) -> dict:
        """Time every launch shape on a device-resident sample of the workload (gx_autotune),
        keep the fastest on this workspace; returns the choice and every candidate's time."""
        cq = N.Queries(q_dev["nspec"], q_dev["npeaks"], q_dev["idx"], q_dev["moz"], q_dev["intn"], q_dev["prec"],
                       q_dev.get("charge"), q_dev.get("dM"))
        p = params.c()
        r = N.TuneResult()
        N.check(N.lib().gx_autotune(self.index.handle, self.handle, C.byref(cq), C.byref(p), reps, int(use_cache),
                                    C.byref(r), stream))
        return {"best": r.best.as_dict(), "cached": bool(r.cached),
                "candidates": [dict(r.cand[i].as_dict(), ms=float(r.ms[i])) for i in range(r.ncand)]}

    def search(self, q: QueryBatch, params: SearchParams, heap: bool = False, hist: bool = False) -> SearchResults:
        """Host buffers in, host results out (H2D, kernels, D2H, synchronise)."""
        n = q.n
        cq, keep = make_c_queries(q, params)
        out = np.zeros(n, N.RESULT_DTYPE)
        cap = params.heap_cap
        hp = np.zeros((n, cap), N.CELL_DTYPE) if heap else None
        hs = np.zeros((n, N.HIST_BINS), np.uint32) if hist else None
        p = params.c()
        N.check(N.lib().gx_search_host(self.index.handle, self.handle, C.byref(cq), C.byref(p), out.ctypes.data,
                                       N.ptr(hp), N.ptr(hs)))
        return SearchResults(out, hp, hs)

    def search_device(self, q_dev: dict, params: SearchParams, out_dev, heap_dev=None, hist_dev=None,
                      stream: int = 0) -> None:
        """Device buffers (integers: device pointers) already in HBM; stream-ordered, no sync.

        ``q_dev`` holds ``nspec, npeaks, idx, moz, intn, prec`` and optionally ``charge``, ``dM``.
        """
        cq = N.Queries(q_dev["nspec"], q_dev["npeaks"], q_dev["idx"], q_dev["moz"], q_dev["intn"], q_dev["prec"],
                       q_dev.get("charge"), q_dev.get("dM"))
        p = params.c()
        N.check(N.lib().gx_search_device(self.index.handle, self.handle, C.byref(cq), C.byref(p), out_dev, heap_dev,
                                         hist_dev, stream))


class Streamer:
    """Chunked search of a host batch (gx_streamer): chunk i+1's upload and chunk i-1's
    result download overlap chunk i's search.  Results equal one search of the whole
    batch.  The batch's arrays should be pinned for the copies to overlap."""

    def __init__(self, index: DeviceIndex, chunk: int = 65536, max_peaks: int = 0):
        self.index = index
        self.chunk = chunk
        self.handle = C.c_void_p()
        N.check(N.lib().gx_streamer_create(index.handle, chunk, max_peaks, C.byref(self.handle)))

    def close(self) -> None:
        if self.handle:
            N.lib().gx_streamer_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tail(self, model, sparse_below: int = 500) -> None:
        """As Searcher.set_tail, for every chunk's search."""
        ws = N.lib().gx_streamer_workspace(self.handle)
        N.check(N.lib().gx_workspace_set_tail(ws, model.handle if model else None, sparse_below))
        self._tail = model

    def search(self, q: QueryBatch, params: SearchParams, out=None, stats: bool = False):
        """Results (gx_result records, host) of the batch; with stats also the timing
        dict (chunks, total/upload/search/download ms).  `out` may be a preallocated
        (pinned) record array."""
        cq, keep = make_c_queries(q, params)
        res = np.zeros(q.n, N.RESULT_DTYPE) if out is None else out
        p = params.c()
        st = N.StreamStats()
        N.check(N.lib().gx_search_stream(self.handle, C.byref(cq), C.byref(p), res.ctypes.data,
                                         C.byref(st) if stats else None))
        if not stats:
            return res
        return res, {f: getattr(st, f) for f in ("chunks", "total_ms", "upload_ms", "search_ms", "download_ms")}


def make_c_queries(q: QueryBatch, params: SearchParams):
    """C view of a QueryBatch (host arrays); returns (struct, keep-alive list)."""
    idx = np.ascontiguousarray(q.idx, np.uint32)
    moz = np.ascontiguousarray(q.moz, np.int32)
    it = np.ascontiguousarray(q.intn, np.int32)
    pr = np.ascontiguousarray(q.prec, np.float32)
    ch = np.ascontiguousarray(q.charge, np.int32)
    dm = None
    if q.dM is not None:
        dm = np.ascontiguousarray(np.where(np.isnan(q.dM), params.dM, q.dM), np.float64)
    cq = N.Queries(q.n, int(idx[-1]) if q.n else 0, idx.ctypes.data, moz.ctypes.data, it.ctypes.data,
                   pr.ctypes.data, ch.ctypes.data, N.ptr(dm))
    return cq, [idx, moz, it, pr, ch, dm]


def algorithmic_traffic(host_index, q: QueryBatch, params: SearchParams, threads: int = 0):
    """Per-spectrum (in-window ion ids of distinct probed bins, distinct probed bins)."""
    cq, keep = make_c_queries(q, params)
    ids = np.zeros(q.n, np.int64)
    bins = np.zeros(q.n, np.int64)
    p = params.c()
    N.check(N.lib().gx_traffic_host(host_index.descs(), host_index.nlen, C.byref(cq), C.byref(p), ids.ctypes.data,
                                    bins.ctypes.data, threads))
    return ids, bins


def algorithmic_bytes(host_index, q: QueryBatch, params: SearchParams, threads: int = 0) -> np.ndarray:
    """Bytes per spectrum the path must move at least (the roofline numerator)."""
    ids, bins = algorithmic_traffic(host_index, q, params, threads)
    npk = np.diff(q.idx.astype(np.int64))
    return 8 * npk + 8 * bins + 4 * ids + 8 * host_index.nlen + N.RESULT_DTYPE.itemsize
