"""Host index builder vs the reference's own index (SHA-256 digests captured from the
compiled reference in tests/golden): entry order, float masses, modification sites,
bA and iA must be identical, length by length."""

import hashlib

import numpy as np
import pytest

from conftest import CASES


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("case", CASES)
def test_builder_matches_reference_index(golden, case):
    c = golden(case)
    H = c["index"]
    assert [x["L"] for x in H.lengths] == list(c["lengths"])
    for i, x in enumerate(H.lengths):
        e = x["entries"]
        assert x["N"] == c["ref_N"][i]
        assert _sha(x["mass"].view(np.uint32), e["seqid"], e["sites"], e["modnum"]) == c["ref_entries_sha"][i], x["L"]
        assert _sha(x["bA"]) == c["ref_bA_sha"][i], x["L"]
        assert _sha(x["iA"]) == c["ref_iA_sha"][i], x["L"]


def test_builder_csr_invariants(golden):
    H = golden("open_mox")["index"]
    for x in H.lengths:
        bA, iA, sl = x["bA"], x["iA"], x["speclen"]
        assert bA[0] == 0 and bA[-1] == x["N"] * sl
        assert np.all(np.diff(bA.astype(np.int64)) >= 0)
        # ids ascending inside every bucket, every id exactly once
        d = np.diff(iA.astype(np.int64))
        inside = np.ones(len(iA) - 1, bool)
        cut = bA[1:-1].astype(np.int64) - 1          # last slot before a bucket boundary
        cut = cut[(cut >= 0) & (cut < len(inside))]
        inside[cut] = False
        assert np.all(d[inside] > 0)
        assert np.array_equal(np.sort(iA), np.arange(x["N"] * sl, dtype=np.uint32))
        assert np.all(np.diff(x["mass"]) >= 0)


def test_builder_rejects_bad_input():
    import ctypes as C
    import gicops_b200._native as N
    L = N.lib()
    h = C.c_void_p()
    bp = N.BuildParams(1, 100, 500, 5000, 0, 0, None, 1)
    seq = np.frombuffer(b"PEPT1DE", np.uint8).copy()
    assert L.gx_build_length(seq.ctypes.data_as(C.c_char_p), 1, 7, C.byref(bp), C.byref(h)) == -3002
    bp0 = N.BuildParams(0, 100, 500, 5000, 0, 0, None, 1)
    seq = np.frombuffer(b"PEPTIDE", np.uint8).copy()
    assert L.gx_build_length(seq.ctypes.data_as(C.c_char_p), 1, 7, C.byref(bp0), C.byref(h)) == -3002
    assert L.gx_build_length(seq.ctypes.data_as(C.c_char_p), 1, 7, None, C.byref(h)) == -3008


def test_entries_only_build_matches_full_build():
    """ions=False stops after the entries: same entries, masses and sequences, no CSR."""
    import gicops_b200 as gx
    db = gx.synth.make_database(120, seed=5)
    a = gx.HostIndex.build(db, maxz=2, mods=[("M", 15.9949, 2)], nmods=2)
    b = gx.HostIndex.build(db, maxz=2, mods=[("M", 15.9949, 2)], nmods=2, ions=False)
    assert [x["L"] for x in a.lengths] == [x["L"] for x in b.lengths]
    for x, y in zip(a.lengths, b.lengths):
        assert x["N"] == y["N"] and x["speclen"] == y["speclen"]
        assert x["entries"].tobytes() == y["entries"].tobytes()
        assert x["mass"].tobytes() == y["mass"].tobytes()
        assert x["seqs"].tobytes() == y["seqs"].tobytes()
        assert y["bA"] is None and y["iA"] is None
    with pytest.raises(ValueError):
        gx.DeviceIndex(b, 0, on_device=False)   # no CSR to upload (raised before any device call)


def test_device_build_rejects_mismatched_lengths():
    """gx_index_build checks its lengths on the host before any device call."""
    import gicops_b200 as gx
    import ctypes as C
    import gicops_b200._native as N
    from gicops_b200.index import _build_params
    db = gx.synth.make_database(50, seed=3)
    H = gx.HostIndex.build(db, maxz=2, ions=False)
    bp, marr = _build_params(1, (), 0, 500, 5000, 100, 0)       # maxz 1 vs lengths built at 2
    hs = (C.c_void_p * H.nlen)(*[x["handle"] for x in H.lengths])
    out = C.c_void_p()
    assert N.lib().gx_index_build(hs, H.nlen, C.byref(bp), 0, C.byref(out)) == -3003 and not out
    bp2, marr2 = _build_params(2, (), 0, 500, 5000, 100, 0)
    assert N.lib().gx_index_build(hs, 0, C.byref(bp2), 0, C.byref(out)) == -3002 and not out
