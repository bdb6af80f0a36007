"""Test infrastructure only: readers for the files the compiled reference harness
(oracle/ref_harness.cpp) writes.

* index dump (``--dump-index``): per length L the peptide sequences, the index
  entries in the reference's final (mass-sorted) order, and the CSR arrays bA/iA
  built by source/core/dslim.cpp:46-153 (left out with ``--entries-only``);
* PSM capture (``--out``): one 32-byte record per spectrum with the fields that
  source/core/dslim_query.cpp:1017-1061 hands to DFile_PrintScore.
"""

from __future__ import annotations

import numpy as np

CAPTURE_DTYPE = np.dtype([
    ("reported", "<i4"), ("psid", "<i4"), ("idxoffset", "<u2"), ("sharedions", "<u2"),
    ("totalions", "<u2"), ("pad0", "<u2"), ("hyperscore", "<f4"), ("npsms", "<u4"), ("e_x", "<f8"),
])


def read_capture(path: str) -> np.ndarray:
    return np.fromfile(path, dtype=CAPTURE_DTYPE)


def read_index_dump(path: str):
    """Returns (header dict, list of per-length dicts).  An entries-only dump
    (``--entries-only``, magic GXREFEN1) has no bA / iA arrays."""
    raw = np.fromfile(path, dtype=np.uint8)
    magic = raw[:8].tobytes()
    assert magic in (b"GXREFIX1", b"GXREFEN1"), "not a reference index dump"
    full = magic == b"GXREFIX1"
    off = 8
    nlen, minlen, maxz, nb = np.frombuffer(raw, dtype="<i4", count=4, offset=off)
    off += 16
    out = []
    for _ in range(int(nlen)):
        L, N, npep, speclen = (int(x) for x in np.frombuffer(raw, dtype="<u4", count=4, offset=off))
        off += 16
        seqs = raw[off:off + npep * L].reshape(npep, L).copy()
        off += npep * L
        mass = np.frombuffer(raw, dtype="<f4", count=N, offset=off).copy(); off += 4 * N
        seqid = np.frombuffer(raw, dtype="<u4", count=N, offset=off).copy(); off += 4 * N
        sites = np.frombuffer(raw, dtype="<u8", count=N, offset=off).copy(); off += 8 * N
        modnum = np.frombuffer(raw, dtype="<u4", count=N, offset=off).copy(); off += 4 * N
        bA = iA = None
        if full:
            bA = np.frombuffer(raw, dtype="<u4", count=int(nb), offset=off).copy(); off += 4 * int(nb)
            iA = np.frombuffer(raw, dtype="<u4", count=N * speclen, offset=off).copy(); off += 4 * N * speclen
        out.append(dict(L=L, N=N, npep=npep, speclen=speclen, seqs=seqs, mass=mass, seqid=seqid,
                        sites=sites, modnum=modnum, bA=bA, iA=iA))
    return dict(nlen=int(nlen), minlen=int(minlen), maxz=int(maxz), nbins=int(nb)), out
