"""Seeded synthetic workloads for the peptide-search query path.

No public dataset is involved: proteins, peptides and spectra are drawn here from
a seeded ``numpy.random.Generator(PCG64(seed))``.

* Database: random proteins (length U[200, 800], residues i.i.d. from standard
  amino-acid background frequencies), digested with trypsin (cleave after K/R,
  not before P, up to 2 missed cleavages), lengths 6..46, one sorted unique list
  per length -- the ``L.peps`` layout that tools/dbtools/db_prep.sh writes in the
  reference (plain sequences, lexicographic order with K and L swapped).
* Queries: spectra sampled from database entries (peptides and their Met-ox
  variants), written in the reference's preprocessed form: integer m/z bins
  (``int(mz * 100)``), integer intensities normalised as
  source/core/msquery.cpp:339-423 does (ascending-intensity order, top peak set
  to the base intensity, others scaled by truncation, cut at the minimum
  intensity, at most QALEN peaks).  The ``.pbin`` byte layout follows
  source/core/msquery.cpp:425-462.
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

# Standard amino-acid background frequencies (percent).
AA_FREQ = {
    "A": 8.25, "R": 5.53, "N": 4.06, "D": 5.45, "C": 1.37, "Q": 3.93, "E": 6.75,
    "G": 7.07, "H": 2.27, "I": 5.96, "L": 9.66, "K": 5.84, "M": 2.42, "F": 3.86,
    "P": 4.70, "S": 6.56, "T": 5.34, "W": 1.08, "Y": 2.92, "V": 6.87,
}

# Residue masses used by the reference (cmake/Templates/aamasses.hpp.in:25-80),
# as float32, plus its fixed carbamidomethyl C.
_AA_MASS = {
    "A": 71.03712, "C": 103.00919, "D": 115.030, "E": 129.0426, "F": 147.068,
    "G": 57.02146, "H": 137.060, "I": 113.084, "K": 128.094, "L": 113.084,
    "M": 131.0405, "N": 114.043, "P": 97.0527, "Q": 128.05858, "R": 156.1012,
    "S": 87.032, "T": 101.0476, "V": 99.06841, "W": 186.0793, "Y": 163.0633,
}
_STAT_MODS = {"C": 57.021464}
H2O = np.float32(18.015)
PROTON = np.float32(1.00727647)

QALEN = 100
BASE_INT = 1000 * 100
MIN_INT = int(BASE_INT * 0.01 + 0.5)
SCALE = 100


def residue_mass_table() -> np.ndarray:
    """float64 residue + static mod mass indexed by ASCII code (0 for non-residues)."""
    t = np.zeros(256, dtype=np.float64)
    for a, m in _AA_MASS.items():
        t[ord(a)] = float(np.float32(m)) + float(np.float32(_STAT_MODS.get(a, 0.0)))
    return t


@dataclass
class Database:
    """Per-length sorted unique peptide sequences: ``peps[L]`` is an (n_L, L) uint8 array."""

    peps: dict = field(default_factory=dict)
    nproteins: int = 0

    @property
    def lengths(self):
        return sorted(self.peps)

    def total(self) -> int:
        return int(sum(len(v) for v in self.peps.values()))

    def write_peps(self, outdir: str, minlen: int = 6, maxlen: int = 46) -> None:
        os.makedirs(outdir, exist_ok=True)
        for L in range(minlen, maxlen + 1):
            arr = self.peps.get(L)
            with open(os.path.join(outdir, f"{L}.peps"), "wb") as f:
                if arr is not None and len(arr):
                    rows = np.concatenate([arr, np.full((len(arr), 1), ord("\n"), np.uint8)], axis=1)
                    f.write(rows.tobytes())


def make_proteome(nproteins: int, seed: int, minlen: int = 200, maxlen: int = 800):
    """Random proteins: returns (residues uint8, starts int64, ends int64)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    letters = np.frombuffer("".join(AA_FREQ).encode(), dtype=np.uint8)
    p = np.array(list(AA_FREQ.values()), dtype=np.float64)
    p /= p.sum()
    lens = rng.integers(minlen, maxlen + 1, size=nproteins)
    ends = np.cumsum(lens)
    starts = ends - lens
    res = letters[rng.choice(len(letters), size=int(ends[-1]) if nproteins else 0, p=p)]
    return res, starts.astype(np.int64), ends.astype(np.int64)


def _swap_kl(a: np.ndarray) -> np.ndarray:
    out = a.copy()
    out[a == ord("K")] = ord("L")
    out[a == ord("L")] = ord("K")
    return out


def tryptic_digest(res, starts, ends, missed: int = 2, minlen: int = 6, maxlen: int = 46) -> Database:
    """Trypsin rules: cleave after K or R unless the next residue is P."""
    n = len(res)
    P = len(starts)
    pid = np.repeat(np.arange(P), ends - starts)
    nxt = np.empty(n, dtype=np.uint8)
    nxt[:-1] = res[1:]
    nxt[-1] = 0
    last = np.zeros(n, dtype=bool)
    last[ends - 1] = True
    cut = ((res == ord("K")) | (res == ord("R"))) & ~last & (nxt != ord("P"))
    cpos = np.nonzero(cut)[0] + 1
    bpos = np.concatenate([starts, cpos, ends])
    bpid = np.concatenate([np.arange(P), pid[cpos - 1], np.arange(P)])
    bord = np.concatenate([np.zeros(P), np.ones(len(cpos)), np.full(P, 2)])
    o = np.lexsort((bord, bpos, bpid))
    bpos, bpid = bpos[o], bpid[o]
    pep_s, pep_l = [], []
    for k in range(1, missed + 2):
        same = bpid[:-k] == bpid[k:]
        s = bpos[:-k][same]
        l = bpos[k:][same] - s
        keep = (l >= minlen) & (l <= maxlen)
        pep_s.append(s[keep])
        pep_l.append(l[keep])
    pep_s = np.concatenate(pep_s)
    pep_l = np.concatenate(pep_l)
    db = Database(nproteins=P)
    for L in range(minlen, maxlen + 1):
        s = pep_s[pep_l == L]
        if not len(s):
            continue
        rows = res[s[:, None] + np.arange(L)[None, :]]
        # db_prep.sh: swap K<->L, lexicographic sort, uniq, swap back
        sw = np.ascontiguousarray(_swap_kl(rows)).view(f"S{L}").ravel()
        u = np.unique(sw)
        rows = _swap_kl(np.frombuffer(u.tobytes(), dtype=np.uint8).reshape(-1, L))
        db.peps[L] = np.ascontiguousarray(rows)
    return db


def make_database(nproteins: int, seed: int, minlen: int = 6, maxlen: int = 46) -> Database:
    res, s, e = make_proteome(nproteins, seed)
    return tryptic_digest(res, s, e, minlen=minlen, maxlen=maxlen)


# --------------------------------------------------------------------------------------
# Queries
# --------------------------------------------------------------------------------------

@dataclass
class QueryBatch:
    """Preprocessed query spectra in the reference's ``Queries<int>`` shape (CSR)."""

    idx: np.ndarray        # uint32 [n+1] row offsets
    moz: np.ndarray        # int32 [npeaks] m/z bins (0.01 Da)
    intn: np.ndarray       # int32 [npeaks] normalised intensity
    prec: np.ndarray       # float32 [n] precursor mass
    charge: np.ndarray     # int32 [n]
    rtime: np.ndarray      # float32 [n]
    dM: np.ndarray | None = None   # float64 [n] per-query precursor tolerance (Da), optional
    truth: np.ndarray | None = None  # int64 [n, 2] (length index, entry) the spectrum came from

    @property
    def n(self) -> int:
        return len(self.prec)

    def subset(self, sel) -> "QueryBatch":
        sel = np.asarray(sel)
        lens = np.diff(self.idx.astype(np.int64))[sel]
        starts = self.idx[:-1].astype(np.int64)[sel]
        gather = np.concatenate([np.arange(a, a + l) for a, l in zip(starts, lens)]) if len(sel) else np.zeros(0, np.int64)
        idx = np.zeros(len(sel) + 1, dtype=np.uint32)
        idx[1:] = np.cumsum(lens)
        return QueryBatch(idx, self.moz[gather], self.intn[gather], self.prec[sel], self.charge[sel],
                          self.rtime[sel], None if self.dM is None else self.dM[sel],
                          None if self.truth is None else self.truth[sel])

    @staticmethod
    def concat(batches) -> "QueryBatch":
        """One batch of the spectra of several, in order."""
        idx = [np.zeros(1, np.int64)]
        off = 0
        for b in batches:
            idx.append(b.idx[1:].astype(np.int64) + off)
            off += int(b.idx[-1])
        dm = None
        if any(b.dM is not None for b in batches):
            dm = np.concatenate([b.dM if b.dM is not None else np.full(b.n, np.nan) for b in batches])
        truth = None
        if all(b.truth is not None for b in batches):
            truth = np.concatenate([b.truth for b in batches])
        return QueryBatch(np.concatenate(idx).astype(np.uint32), np.concatenate([b.moz for b in batches]),
                          np.concatenate([b.intn for b in batches]), np.concatenate([b.prec for b in batches]),
                          np.concatenate([b.charge for b in batches]), np.concatenate([b.rtime for b in batches]),
                          dm, truth)

    def write_pbin(self, path: str) -> None:
        with open(path, "wb") as f:
            for i in range(self.n):
                a, b = int(self.idx[i]), int(self.idx[i + 1])
                f.write(np.float32(self.prec[i]).tobytes())
                f.write(np.int32(self.charge[i]).tobytes())
                f.write(np.float32(self.rtime[i]).tobytes())
                f.write(np.int32(b - a).tobytes())
                f.write(self.moz[a:b].astype(np.int32).tobytes())
                f.write(self.intn[a:b].astype(np.int32).tobytes())

    @staticmethod
    def read_pbin(path: str) -> "QueryBatch":
        raw = open(path, "rb").read()
        off = 0
        prec, z, rt, mz, it, lens = [], [], [], [], [], []
        while off < len(raw):
            p, c, r, l = np.frombuffer(raw, dtype=np.float32, count=1, offset=off)[0], \
                np.frombuffer(raw, dtype=np.int32, count=1, offset=off + 4)[0], \
                np.frombuffer(raw, dtype=np.float32, count=1, offset=off + 8)[0], \
                int(np.frombuffer(raw, dtype=np.int32, count=1, offset=off + 12)[0])
            off += 16
            mz.append(np.frombuffer(raw, dtype=np.int32, count=l, offset=off)); off += 4 * l
            it.append(np.frombuffer(raw, dtype=np.int32, count=l, offset=off)); off += 4 * l
            prec.append(p); z.append(c); rt.append(r); lens.append(l)
        idx = np.zeros(len(lens) + 1, dtype=np.uint32)
        idx[1:] = np.cumsum(lens)
        return QueryBatch(idx, np.concatenate(mz) if mz else np.zeros(0, np.int32),
                          np.concatenate(it) if it else np.zeros(0, np.int32),
                          np.array(prec, np.float32), np.array(z, np.int32), np.array(rt, np.float32))


def normalise_peaks(mz_int: np.ndarray, intn_int: np.ndarray):
    """Intensity normalisation and peak picking of source/core/msquery.cpp:339-423.

    Peaks are ordered by ascending intensity (ties by position: this generator
    writes the preprocessed form directly, so its order *is* the input), the top
    peak gets BASE_INT, every other peak ``int(intn * factor)``, peaks are kept
    from the top down while ``>= MIN_INT``, at most QALEN of them.
    """
    n = len(mz_int)
    if n == 0:
        return mz_int, intn_int
    o = np.argsort(intn_int, kind="stable")
    mz_s = mz_int[o].astype(np.int64)
    in_s = intn_int[o].astype(np.int64)
    factor = float(BASE_INT) / float(in_s[-1])
    in_s[-1] = BASE_INT
    keep = 1
    j = n - 2
    while j >= n - QALEN and j >= 0:
        in_s[j] = int(float(in_s[j]) * factor)
        if in_s[j] >= MIN_INT:
            keep += 1
        else:
            break
        j -= 1
    keep = min(keep, QALEN)
    return mz_s[n - keep:].astype(np.int32), in_s[n - keep:].astype(np.int32)


def fragment_mz(seq: bytes, site_mask: int, mod_of_site, frag_charges, mtab) -> np.ndarray:
    """b and y fragment m/z (float64) of a (modified) peptide at the given charges."""
    L = len(seq)
    m = np.array([mtab[c] for c in seq], dtype=np.float64)
    for i in range(L):
        if (site_mask >> i) & 1:
            m[i] += mod_of_site(i)
    b = np.cumsum(m[:-1])
    y = np.cumsum(m[::-1][:-1]) + float(H2O)
    out = []
    for z in frag_charges:
        out.append((b + z * float(PROTON)) / z)
        out.append((y + z * float(PROTON)) / z)
    return np.concatenate(out)


def make_queries(entries_by_len: dict, nspec: int, seed: int, *, charges=(2, 3), frag_charge2: bool = False,
                 keep_p=(0.6, 0.6), noise_mode: str = "fixed40", npeaks_range=(30, 150),
                 mz_sigma: float = 0.01, mod_mass: float = 15.99, window: str = "fixed") -> QueryBatch:
    """Spectra sampled from database entries.

    ``entries_by_len[L] = (seqs (n_pep x L uint8), seqID u32[N], sites u64[N], mass f32[N])``
    lists every index entry (peptide or variant) of length L in index order.
    ``keep_p`` is (lo, hi) of the per-spectrum ion retention probability.
    ``noise_mode``: "fixed40" adds 40 U[100, 2000] noise peaks; "fill" adds noise up
    to a U[npeaks_range] total.  ``frag_charge2`` emits charge-2 fragments for
    precursor charge >= 3.  ``window`` = "mixed" gives half the spectra a
    +-10 ppm precursor tolerance (``dM`` set per spectrum, the rest NaN).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    mtab = residue_mass_table()
    lens = sorted(entries_by_len)
    counts = np.array([len(entries_by_len[L][1]) for L in lens], dtype=np.int64)
    cum = np.cumsum(counts)
    picks = rng.integers(0, int(cum[-1]), size=nspec)
    moz, intn, idx = [], [], [0]
    prec = np.zeros(nspec, np.float32)
    chg = np.zeros(nspec, np.int32)
    truth = np.zeros((nspec, 2), np.int64)
    dM = np.full(nspec, np.nan)
    for q in range(nspec):
        li = int(np.searchsorted(cum, picks[q], side="right"))
        e = int(picks[q] - (cum[li - 1] if li else 0))
        L = lens[li]
        seqs, seqid, sites, mass = entries_by_len[L]
        seq = bytes(seqs[int(seqid[e])])
        z = int(rng.integers(charges[0], charges[1] + 1))
        fz = (1, 2) if (frag_charge2 and z >= 3) else (1,)
        ions = fragment_mz(seq, int(sites[e]), lambda i: mod_mass, fz, mtab)
        p = rng.uniform(keep_p[0], keep_p[1]) if keep_p[0] != keep_p[1] else keep_p[0]
        ions = ions[rng.random(len(ions)) < p]
        ions = ions + rng.normal(0.0, mz_sigma, size=len(ions))
        if noise_mode == "fixed40":
            nn = 40
        else:
            tot = int(rng.integers(npeaks_range[0], npeaks_range[1] + 1))
            nn = max(0, tot - len(ions))
        noise = rng.uniform(100.0, 2000.0, size=nn)
        mzs = np.concatenate([ions, noise])
        inten = rng.lognormal(0.0, 1.0, size=len(mzs)).astype(np.float32)
        mz_i = np.floor(mzs * SCALE).astype(np.int64)            # int(atof(mz) * scale)
        in_i = np.floor(inten.astype(np.float64) * 100).astype(np.int64)  # int(atof(intn) * 100)
        in_i = np.maximum(in_i, 1)
        m_i, n_i = normalise_peaks(mz_i, in_i)
        moz.append(m_i)
        intn.append(n_i)
        idx.append(idx[-1] + len(m_i))
        prec[q] = mass[e]
        chg[q] = z
        truth[q] = (li, e)
        if window == "mixed" and rng.random() < 0.5:
            dM[q] = float(prec[q]) * 10e-6
    return QueryBatch(np.array(idx, np.uint32), np.concatenate(moz).astype(np.int32),
                      np.concatenate(intn).astype(np.int32), prec, chg, np.zeros(nspec, np.float32),
                      dM if window == "mixed" else None, truth)


# --------------------------------------------------------------------------------------
# Named workloads (shapes of the five benchmark configurations)
# --------------------------------------------------------------------------------------

WORKLOADS = {
    # closed search, small
    "closed-1k": dict(nproteins=1000, maxz=1, mods=(), nmods=0, nspec=2000, dM=10.0,
                      q=dict(charges=(2, 3), frag_charge2=False, keep_p=(0.6, 0.6), noise_mode="fixed40")),
    # open search, medium
    "open-20k": dict(nproteins=20000, maxz=2, mods=(("M", 15.9949, 2),), nmods=2, nspec=50000, dM=500.0,
                     q=dict(charges=(2, 4), frag_charge2=True, keep_p=(0.6, 0.6), noise_mode="fill")),
    # large mixed search
    "mixed-200k": dict(nproteins=200000, maxz=2, mods=(("M", 15.9949, 3),), nmods=3, nspec=200000, dM=500.0,
                       q=dict(charges=(2, 4), frag_charge2=True, keep_p=(0.2, 0.8), noise_mode="fill",
                              window="mixed")),
}
