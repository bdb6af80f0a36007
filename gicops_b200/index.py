"""Host and device fragment-ion indexes.

``HostIndex`` is the query-path view of the reference's ``Index[]`` array (one entry
per peptide length, source/core/include/slm_dsts.h:313-346): mass-sorted entries,
CSR ``bA`` row offsets per 0.01 Da bin and ``iA`` ion ids.  It is built by the
library's host builder (``gx_build_length``) from per-length peptide lists, or
wrapped around arrays built elsewhere (e.g. dumped from the reference).

``DeviceIndex`` keeps one index resident in HBM (``gx_index_upload``), the
counterpart of the reference's ``hcp::gpu::cuda::s1::getdIndex``
(source/core/cuda/superstep1/kernel.cu:310-358).  With ``on_device`` it computes the
fragment ions, the CSR and the block layout on the GPU from the host entries
(``gx_index_build``); a HostIndex built with ``ions=False`` holds only those entries.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _native as N
from .synth import Database


def _build_params(maxz, mods, nmods, min_mass, max_mass, scale, threads):
    """gx_build_params (and the Mod array it points to, which the caller keeps alive)."""
    marr = (N.Mod * max(1, len(mods)))()
    for i, (res, mass, mx) in enumerate(mods):
        marr[i] = N.Mod(res.encode()[:4], float(mass), int(mx))
    bp = N.BuildParams(maxz, scale, min_mass, max_mass, len(mods), nmods if mods else 0, marr, threads)
    return bp, marr


class HostIndex:
    def __init__(self, lengths: list[dict], maxz: int, scale: int = 100, max_mass: int = 5000,
                 handles: list | None = None, build_args: tuple | None = None):
        self.lengths = lengths          # [{L, N, speclen, mass, bA, iA, seqs?, entries?, handle?}]
        self.maxz = maxz
        self.scale = scale
        self.max_mass = max_mass
        self.nbins = max_mass * scale + 1
        self._handles = handles or []
        self._build_args = build_args   # (maxz, scale, min_mass, max_mass, mods, nmods) of build()

    # ------------------------------------------------------------------ construction
    @classmethod
    def build(cls, db: Database, maxz: int, mods=(), nmods: int = 0, min_mass: int = 500, max_mass: int = 5000,
              scale: int = 100, minlen: int = 6, maxlen: int = 46, threads: int = 0, ions: bool = True) -> "HostIndex":
        """Index every length of ``db`` with the reference's construction rules.

        ``mods`` is a sequence of (residues, mass_Da, max_per_peptide); ``nmods`` the
        total modified residues per peptide (the reference's ``vmods_per_pep``).  With
        ``ions=False`` only the entries are built (bA and iA are None): the fragment ions
        are then computed on the GPU by ``DeviceIndex(..., on_device=True)``.
        """
        L_ = N.lib()
        bp, marr = _build_params(maxz, mods, nmods, min_mass, max_mass, scale, threads)
        lengths, handles = [], []
        for L in range(minlen, maxlen + 1):
            seqs = db.peps.get(L)
            if seqs is None or not len(seqs):
                continue
            h = C.c_void_p()
            fn = L_.gx_build_length if ions else L_.gx_build_length_entries
            N.check(fn(np.ascontiguousarray(seqs).ctypes.data_as(C.c_char_p), len(seqs), L, C.byref(bp), C.byref(h)))
            handles.append(h)
            d = N.LengthDesc()
            N.check(L_.gx_host_length_desc(h, C.byref(d)))
            if d.npep == 0:
                continue
            nb = max_mass * scale + 1
            mass = np.ctypeslib.as_array(C.cast(d.mass, C.POINTER(C.c_float)), (d.npep,))
            bA = np.ctypeslib.as_array(C.cast(d.bA, C.POINTER(C.c_uint32)), (nb,)) if ions else None
            iA = np.ctypeslib.as_array(C.cast(d.iA, C.POINTER(C.c_uint32)), (d.npep * d.speclen,)) if ions else None
            ent_p = L_.gx_host_length_entries(h)
            ent = np.ctypeslib.as_array(C.cast(ent_p, C.POINTER(C.c_uint8)),
                                        (d.npep * N.PEP_ENTRY_DTYPE.itemsize,)).view(N.PEP_ENTRY_DTYPE)
            nk = C.c_uint32()
            sp = L_.gx_host_length_seqs(h, C.byref(nk))
            kept = np.ctypeslib.as_array(C.cast(sp, C.POINTER(C.c_uint8)), (nk.value * L,)).reshape(nk.value, L) \
                if nk.value else np.zeros((0, L), np.uint8)
            lengths.append(dict(L=L, N=int(d.npep), speclen=int(d.speclen), mass=mass, bA=bA, iA=iA,
                                entries=ent, seqs=kept, handle=h))
        return cls(lengths, maxz, scale, max_mass, handles, (maxz, scale, min_mass, max_mass, tuple(mods), nmods))

    def close(self) -> None:
        L_ = N.lib()
        for h in self._handles:
            L_.gx_host_length_free(h)
        self._handles = []
        self.lengths = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ views
    @property
    def nlen(self) -> int:
        return len(self.lengths)

    def total_entries(self) -> int:
        return sum(x["N"] for x in self.lengths)

    def total_ions(self) -> int:
        return sum(x["N"] * x["speclen"] for x in self.lengths)

    def entries_by_len(self) -> dict:
        """{L: (seqs, seqid, sites, mass)} for the query generator."""
        return {x["L"]: (x["seqs"], x["entries"]["seqid"], x["entries"]["sites"], x["mass"]) for x in self.lengths}

    def descs(self):
        arr = (N.LengthDesc * self.nlen)()
        for i, x in enumerate(self.lengths):
            arr[i] = N.LengthDesc(x["L"], x["N"], x["speclen"], 0, x["mass"].ctypes.data, x["bA"].ctypes.data,
                                  x["iA"].ctypes.data)
        return arr

    def peptide(self, ixx: int, psid: int) -> str:
        """Sequence of entry ``psid`` of length index ``ixx`` (lower case at modified sites)."""
        x = self.lengths[ixx]
        e = x["entries"][psid]
        s = bytearray(bytes(x["seqs"][int(e["seqid"])]))
        for i in range(len(s)):
            if (int(e["sites"]) >> i) & 1:
                s[i] += 32
        return s.decode()


class DeviceIndex:
    """An index resident in HBM on one device.

    ``on_device``: compute the fragment ions, CSR and block layout on the GPU from the
    host entries (``gx_index_build``) instead of uploading the host CSR
    (``gx_index_upload``); the default is to do so when the host index has no CSR."""

    def __init__(self, host: HostIndex, device: int = 0, on_device: bool | None = None):
        self.host = host
        self.device = device
        self.handle = C.c_void_p()
        has_csr = all(x["bA"] is not None for x in host.lengths)
        if on_device is None:
            on_device = not has_csr
        if on_device:
            if host._build_args is None or any("handle" not in x for x in host.lengths):
                raise ValueError("on_device needs a HostIndex made by HostIndex.build")
            maxz, scale, min_mass, max_mass, mods, nmods = host._build_args
            bp, marr = _build_params(maxz, mods, nmods, min_mass, max_mass, scale, 0)
            hs = (C.c_void_p * host.nlen)(*[x["handle"] for x in host.lengths])
            N.check(N.lib().gx_index_build(hs, host.nlen, C.byref(bp), device, C.byref(self.handle)))
        else:
            if not has_csr:
                raise ValueError("the host index has no CSR (built with ions=False): use on_device")
            N.check(N.lib().gx_index_upload(host.descs(), host.nlen, host.nbins, device, C.byref(self.handle)))

    def save(self, path: str) -> None:
        """Write the device arrays to a file (gx_index_save)."""
        N.check(N.lib().gx_index_save(self.handle, os.fsencode(path)))

    @classmethod
    def load(cls, path: str, device: int = 0, host: "HostIndex | None" = None) -> "DeviceIndex":
        """An index written by save(), put back on `device` without building (gx_index_load).
        `host` (optional) is the HostIndex it was built from, for read_length and the
        peptide strings of results."""
        obj = cls.__new__(cls)
        obj.host, obj.device, obj.handle = host, device, C.c_void_p()
        N.check(N.lib().gx_index_load(os.fsencode(path), device, C.byref(obj.handle)))
        return obj

    def read_length(self, i: int) -> dict:
        """Device arrays of length i: bA, iA (ids 2*entry + (y ion)), iAb (block-local), mass."""
        x = self.host.lengths[i]
        n = x["N"] * x["speclen"]
        out = dict(bA=np.zeros(self.host.nbins, np.uint32), iA=np.zeros(n, np.uint32), iAb=np.zeros(n, np.uint16),
                   mass=np.zeros(x["N"], np.float32))
        N.check(N.lib().gx_index_read_length(self.handle, i, out["bA"].ctypes.data, out["iA"].ctypes.data,
                                             out["iAb"].ctypes.data, out["mass"].ctypes.data))
        return out

    @property
    def nbytes(self) -> int:
        return int(N.lib().gx_index_bytes(self.handle))

    def close(self) -> None:
        if self.handle:
            N.lib().gx_index_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
