"""Generates the golden fixtures of this folder from the reference's own CPU code.

Needs the compiled reference harness (oracle/_ref/ref_harness, built by
``make -C oracle`` where the reference source tree is present).  For each case it

1. draws a seeded synthetic peptide database (gicops_b200.synth) and writes the
   per-length ``L.peps`` files;
2. lets the reference build its index (LBE + DSLIM_Construct) and dumps it;
3. draws query spectra from the reference's index entries and runs the reference's
   DSLIM_QuerySpectrum on them, capturing every PSM it reports;
4. stores the peptide lists, SHA-256 digests of the reference's index arrays per
   length, the queries and the captured PSMs in ``<case>.npz``.

The fixtures pin the oracle (tests/test_oracle.py) and the host index builder
(tests/test_index_build.py) on machines without the reference, and the GPU path
(tests/test_gpu_parity.py) on the GPU box.

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from gicops_b200 import synth  # noqa: E402
import refdump  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")

CASES = {
    # closed search: charge-1 fragments, no variable modifications, +-10 Da; min_cpsm 1
    # so that e-values of spectra with 1..3 candidates (the short tail-fit branches) are
    # captured too
    "closed_small": dict(nproteins=200, seed=11, maxz=1, mods=[], nmods=0, dM=10.0, nspec=300, min_cpsm=1,
                         q=dict(charges=(2, 3), frag_charge2=False, keep_p=(0.6, 0.6), noise_mode="fixed40")),
    # the closed-search workload's database size (1,000 proteins)
    "closed_1k": dict(nproteins=1000, seed=14, maxz=1, mods=[], nmods=0, dM=10.0, nspec=150,
                      q=dict(charges=(2, 3), frag_charge2=False, keep_p=(0.6, 0.6), noise_mode="fixed40")),
    # open search: charge 1-2 fragments, Met oxidation (<= 2), +-500 Da, 30-150 peaks
    "open_mox": dict(nproteins=150, seed=12, maxz=2, mods=[("M", 15.9949, 2)], nmods=2, dM=500.0, nspec=200,
                     q=dict(charges=(2, 4), frag_charge2=True, keep_p=(0.6, 0.6), noise_mode="fill")),
    # mixed windows: half the spectra at +-10 ppm, the rest +-500 Da; Met-ox <= 3
    "mixed_window": dict(nproteins=150, seed=13, maxz=2, mods=[("M", 15.9949, 3)], nmods=3, dM=500.0, nspec=200,
                         q=dict(charges=(2, 4), frag_charge2=True, keep_p=(0.2, 0.8), noise_mode="fill",
                                window="mixed")),
}


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def entry_digest(x) -> str:
    return sha(x["mass"].view(np.uint32), x["seqid"], x["sites"], x["modnum"])


def make_case(name: str, cfg: dict, tmp: str) -> None:
    db = synth.make_database(cfg["nproteins"], seed=cfg["seed"])
    dbdir = os.path.join(tmp, name)
    db.write_peps(dbdir)
    base = [HARNESS, "--db", dbdir, "--maxz", str(cfg["maxz"]), "--dM", str(cfg["dM"]), "--dF", "5",
            "--threads", "4", "--topmatches", "5", "--expect-max", "1e300",
            "--min-cpsm", str(cfg.get("min_cpsm", 4))]
    for r, m, n in cfg["mods"]:
        base += ["--mods", f"{r}:{m}:{n}"]
    if cfg["mods"]:
        base += ["--nmods", str(cfg["nmods"])]
    dump = os.path.join(tmp, name + ".idx")
    subprocess.run(base + ["--dump-index", dump], check=True, capture_output=True)
    hdr, R = refdump.read_index_dump(dump)
    R = [x for x in R if x["N"]]
    ent = {x["L"]: (x["seqs"], x["seqid"], x["sites"], x["mass"]) for x in R}
    q = synth.make_queries(ent, cfg["nspec"], seed=cfg["seed"] + 1000, **cfg["q"])
    qf = os.path.join(tmp, name + ".pbin")
    q.write_pbin(qf)
    cap = os.path.join(tmp, name + ".cap")
    cmd = base + ["--queries", qf, "--out", cap]
    if q.dM is not None:
        dm = np.where(np.isnan(q.dM), cfg["dM"], q.dM).astype(np.float64)
        dmf = os.path.join(tmp, name + ".qdm")
        dm.tofile(dmf)
        cmd += ["--qdm", dmf]
    subprocess.run(cmd, check=True, capture_output=True)
    c = refdump.read_capture(cap)
    out = dict(
        meta=json.dumps(dict(name=name, nproteins=cfg["nproteins"], seed=cfg["seed"], maxz=cfg["maxz"],
                             mods=cfg["mods"], nmods=cfg["nmods"], dM=cfg["dM"], dF=5, topmatches=5,
                             min_cpsm=cfg.get("min_cpsm", 4), min_shp=4,
                             min_mass=500, max_mass=5000, minlen=6, maxlen=46)),
        lengths=np.array([x["L"] for x in R], np.int32),
        ref_N=np.array([x["N"] for x in R], np.int64),
        ref_entries_sha=np.array([entry_digest(x) for x in R]),
        ref_bA_sha=np.array([sha(x["bA"]) for x in R]),
        ref_iA_sha=np.array([sha(x["iA"]) for x in R]),
        q_idx=q.idx, q_moz=q.moz, q_intn=q.intn, q_prec=q.prec, q_charge=q.charge,
        q_dM=q.dM if q.dM is not None else np.zeros(0),
        cap_reported=c["reported"], cap_psid=c["psid"], cap_idxoffset=c["idxoffset"],
        cap_sharedions=c["sharedions"], cap_totalions=c["totalions"], cap_hyperscore=c["hyperscore"],
        cap_npsms=c["npsms"], cap_e_x=c["e_x"],
    )
    for L, seqs in db.peps.items():
        out[f"peps_{L}"] = seqs
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "entries", int(sum(x["N"] for x in R)), "spectra", q.n, "reported", int(c["reported"].sum()))


def main() -> None:
    if not os.path.exists(HARNESS):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True)
    with tempfile.TemporaryDirectory() as tmp:
        for name, cfg in CASES.items():
            make_case(name, cfg, tmp)


if __name__ == "__main__":
    main()
