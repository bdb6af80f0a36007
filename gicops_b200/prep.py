"""Query preprocessing: MS2 text -> peak-picked query batch (-> .pbin), the reference's
MS2 conversion (MSQuery::convertAndprepMS2bin, source/core/msquery.cpp:137-336).

``read_ms2`` parses the file on the host with the reference's rules (``gx_ms2_read``);
``pickpeaks`` sorts, normalises and picks the peaks of every spectrum on the GPU
(``gx_pickpeaks_device``: the reference's MSQuery::pickpeaks, msquery.cpp:338-423,
with its key-value quicksort, so ties end in the same order); ``convert_ms2`` does both
and writes the ``.pbin`` the reference would write (``QueryBatch.write_pbin``).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .synth import BASE_INT, MIN_INT, QALEN, QueryBatch


class RawSpectra:
    """Spectra of an MS2 file before peak picking (host arrays owned by the library).

    Spectrum s owns the values ``seg[s]:seg[s+1]`` of ``mz`` / ``intn`` and counts
    ``size[s]`` of them (they differ only for values before the file's first S line)."""

    def __init__(self, path: str, scale: int = 100):
        self.handle = C.c_void_p()
        N.check(N.lib().gx_ms2_read(path.encode(), scale, C.byref(self.handle)))
        d = N.Ms2Raw()
        N.check(N.lib().gx_ms2_desc(self.handle, C.byref(d)))
        self.nspec, self.nvalues = int(d.nspec), int(d.nvalues)

        def arr(ptr, n, ct, dt):
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), (n,)).view(dt) if n else np.zeros(0, dt)
        self.seg = arr(d.seg, self.nspec + 1, C.c_uint32, np.uint32)
        self.size = arr(d.size, self.nspec, C.c_uint32, np.uint32)
        self.mz = arr(d.mz, self.nvalues, C.c_int32, np.int32)
        self.intn = arr(d.intn, self.nvalues, C.c_int32, np.int32)
        self.prec = arr(d.prec, self.nspec, C.c_float, np.float32)
        self.charge = arr(d.charge, self.nspec, C.c_int32, np.int32)
        self.rtime = arr(d.rtime, self.nspec, C.c_float, np.float32)

    def close(self) -> None:
        if self.handle:
            N.lib().gx_ms2_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_ms2(path: str, scale: int = 100) -> RawSpectra:
    return RawSpectra(path, scale)


def pickpeaks(raw: RawSpectra, device: int = 0, base_int: int = BASE_INT, min_int: int = MIN_INT,
              qalen: int = QALEN) -> QueryBatch:
    """Peak picking and normalisation of every spectrum on the GPU; a host QueryBatch."""
    import torch
    d = torch.device("cuda", device)
    with torch.cuda.device(d):
        seg = torch.from_numpy(raw.seg.astype(np.int32)).to(d)
        size = torch.from_numpy(raw.size.astype(np.int32)).to(d)
        mz = torch.from_numpy(raw.mz.copy()).to(d)
        it = torch.from_numpy(raw.intn.copy()).to(d)
        idx = torch.empty(raw.nspec + 1, dtype=torch.int32, device=d)
        omz = torch.empty(max(raw.nvalues, 1), dtype=torch.int32, device=d)
        oit = torch.empty(max(raw.nvalues, 1), dtype=torch.int32, device=d)
        st = torch.cuda.current_stream(d)
        N.check(N.lib().gx_pickpeaks_device(raw.nspec, seg.data_ptr(), size.data_ptr(), mz.data_ptr(), it.data_ptr(),
                                            base_int, min_int, qalen, idx.data_ptr(), omz.data_ptr(), oit.data_ptr(),
                                            C.c_void_p(st.cuda_stream)))
        st.synchronize()
        hidx = idx.cpu().numpy().view(np.uint32)
        n = int(hidx[-1])
        return QueryBatch(hidx.copy(), omz[:n].cpu().numpy().copy(), oit[:n].cpu().numpy().copy(),
                          raw.prec.copy(), raw.charge.copy(), raw.rtime.copy())


def convert_ms2(path: str, out: str | None = None, device: int = 0, scale: int = 100) -> QueryBatch:
    """MS2 file -> query batch, written to ``out`` (default ``path + '.pbin'``) as the
    reference's conversion writes it."""
    raw = read_ms2(path, scale)
    try:
        q = pickpeaks(raw, device)
    finally:
        raw.close()
    q.write_pbin(out if out is not None else path + ".pbin")
    return q
