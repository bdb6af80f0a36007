"""Benchmark of the peptide-search query path (spectra/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload large-200k] [--impl ours|reference]

A step is one search of the whole synthetic batch.  The default workload is the large
open-search configuration: 200,000 proteins with Met oxidation <= 3 (39.7M index entries,
3.3G fragment-ion ids, b/y ions of charge 1-2, a 27 GB index in HBM), 200,000 spectra of
30-150 peaks with 20-80% ion retention, half at a +-10 ppm and half at a +-500 Da precursor
window, +-0.05 Da fragment tolerance, top-K 5.  Its index is larger than L2, so steps run
back to back; an index smaller than twice L2 (the closed-1k workload's) is flushed from L2
before each timed step instead, and the step timed alone.

Printed (rank 0, one JSON line): value = spectra/s with queries resident in HBM (CUDA
events on the launching stream, max over ranks); e2e = spectra/s through the host-buffer
API (pinned host queries in, results out, per step); roofline of the dominant kernel
against the measured HBM copy bandwidth; parity = the benchmarked batch's own outputs
against the oracle on a seeded sample, with the accuracy figures; plain_path = the plain
one-spectrum-per-CTA path on a seeded sample, beside the batched path on the same sample;
cpu_baseline = the reference's own OpenMP CPU query path timed on a bounded sample on
this host.

Under torchrun each rank searches its own batch against a replica of the index
(spectra are independent: weak scaling, no collective on the data path).
``--impl reference`` times the reference's CPU implementation alone (rank 0); that arm
runs the compiled reference and numpy only (its queries come from the reference's own
index entries), and loads nothing of this package's native library.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "open-20k": dict(nproteins=20000, db_seed=1, maxz=2, mods=[("M", 15.9949, 2)], nmods=2, nspec=50000, dM=500.0,
                     q=dict(charges=(2, 4), frag_charge2=True, keep_p=(0.6, 0.6), noise_mode="fill",
                            npeaks_range=(30, 150))),
    # the large config's window mix (half +-10 ppm, half +-500 Da; 20-80% ion retention) on the
    # 20,000-protein database
    "mixed-20k": dict(nproteins=20000, db_seed=1, maxz=2, mods=[("M", 15.9949, 2)], nmods=2, nspec=50000, dM=500.0,
                      q=dict(charges=(2, 4), frag_charge2=True, keep_p=(0.2, 0.8), noise_mode="fill",
                             npeaks_range=(30, 150), window="mixed")),
    "closed-1k": dict(nproteins=1000, db_seed=1, maxz=1, mods=[], nmods=0, nspec=2000, dM=10.0,
                      q=dict(charges=(2, 3), frag_charge2=False, keep_p=(0.6, 0.6), noise_mode="fixed40")),
    # the large config at its stated size: 200,000 proteins, Met oxidation <= 3 (39.7M entries,
    # 3.3G ion ids), 200,000 spectra, half +-10 ppm and half +-500 Da, 20-80% ion retention
    # (the N-terminal acetylation of that config cannot be expressed in the reference: left out)
    "large-200k": dict(nproteins=200000, db_seed=1, maxz=2, mods=[("M", 15.9949, 3)], nmods=3, nspec=200000,
                       dM=500.0, q=dict(charges=(2, 4), frag_charge2=True, keep_p=(0.2, 0.8), noise_mode="fill",
                                        npeaks_range=(30, 150), window="mixed")),
}


# The stress configuration: 1M proteins with Met oxidation <= 3 (about 200M index entries and
# 16G fragment-ion ids, built on the GPU), 1M spectra at +-500 Da streamed from pinned host
# memory in 64k-spectrum chunks (--stream-run; a measurement beside the bench, not its step)
STRESS = dict(nproteins=1000000, db_seed=1, maxz=2, mods=[("M", 15.9949, 3)], nmods=3, nspec=1000000, dM=500.0,
              chunk=65536, q=dict(charges=(2, 4), frag_charge2=True, keep_p=(0.2, 0.8), noise_mode="fill",
                                  npeaks_range=(30, 150)))

# spectra per step of the reference's CPU path: a seeded random subset of the workload's
# batch (the whole batch where it takes seconds), sized for a few seconds per step
REF_SAMPLE = {"large-200k": 1024, "mixed-20k": 4096, "open-20k": 2048, "closed-1k": 2000}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def ref_sample(name: str, n: int) -> np.ndarray:
    """The seeded subset of the batch that the reference's CPU path is timed on (both arms)."""
    m = min(n, REF_SAMPLE.get(name, 2048))
    sel = np.random.Generator(np.random.PCG64(7)).choice(n, size=m, replace=False)
    sel.sort()
    return sel


def make_reference_workload(name: str):
    """The workload for the reference arm, with no call into this package's native library:
    the database from the seeded generator (numpy), the index entries (peptides and Met-ox
    variants in index order) from the compiled reference itself (ref_harness
    --entries-only), and the spectra drawn from those entries by the same generator and
    seed as rank 0 of the GPU arm (the two sets of entries are identical: the library's
    builder is pinned to the reference's arrays)."""
    from gicops_b200 import synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refdump
    w = WORKLOADS[name]
    t = time.time()
    db = synth.make_database(w["nproteins"], seed=w["db_seed"])
    with tempfile.TemporaryDirectory() as tmp:
        dbdir = os.path.join(tmp, "db")
        db.write_peps(dbdir)
        dump = os.path.join(tmp, "entries.bin")
        cmd = [os.path.join(ROOT, "oracle", "_ref", "ref_harness"), "--db", dbdir, "--maxz", str(w["maxz"]),
               "--entries-only", "--dump-index", dump]
        for r, m, n in w["mods"]:
            cmd += ["--mods", f"{r}:{m}:{n}"]
        if w["mods"]:
            cmd += ["--nmods", str(w["nmods"])]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed: {r.stderr[-400:]}")
        _, R = refdump.read_index_dump(dump)
    ent = {x["L"]: (x["seqs"], x["seqid"], x["sites"], x["mass"]) for x in R if x["N"]}
    q = synth.make_queries(ent, w["nspec"], seed=1000, **w["q"])
    log(f"[bench] reference workload {name}: {sum(x['N'] for x in R)} entries (reference build), {q.n} spectra "
        f"({time.time() - t:.1f}s)")
    return w, db, q


def make_workload(name: str, rank: int):
    import gicops_b200 as gx
    w = WORKLOADS[name]
    t = time.time()
    db = gx.synth.make_database(w["nproteins"], seed=w["db_seed"])
    t1 = time.perf_counter()
    H = gx.HostIndex.build(db, maxz=w["maxz"], mods=w["mods"], nmods=w["nmods"])
    w = dict(w, host_build_s=time.perf_counter() - t1)
    q = gx.synth.make_queries(H.entries_by_len(), w["nspec"], seed=1000 + rank, **w["q"])
    log(f"[bench] workload {name}: {H.total_entries()} entries, {H.total_ions()} ion ids, {q.n} spectra, "
        f"{len(q.moz)} peaks ({time.time() - t:.1f}s)")
    return w, db, H, q


def prep_measure(gx, q, local: int, rank: int) -> dict:
    """Peak picking of the workload's spectra as raw input (each spectrum's peaks shuffled,
    intensities unnormalised, plus as many low noise peaks again), on the GPU
    (gx_pickpeaks_device, CUDA events on its stream) and, on rank 0, the CPU baseline of
    this step: the oracle's restatement on one host thread over a 2,000-spectrum sample.
    Untimed set-up of the bench."""
    import ctypes as C
    import torch
    import gicops_b200._native as N
    rng = np.random.default_rng(77 + rank)
    lens = np.diff(q.idx.astype(np.int64))
    seg = np.zeros(q.n + 1, np.int64)
    seg[1:] = np.cumsum(2 * lens)
    n = int(seg[-1])
    mz = np.empty(n, np.int32)
    it = np.empty(n, np.int32)
    for s in range(q.n):
        a, b, k = int(q.idx[s]), int(q.idx[s + 1]), int(lens[s])
        o = int(seg[s])
        mz[o:o + k] = q.moz[a:b]
        it[o:o + k] = (q.intn[a:b].astype(np.float64) * rng.uniform(0.5, 3.0)).astype(np.int32)
        mz[o + k:o + 2 * k] = rng.integers(10000, 200000, k)
        it[o + k:o + 2 * k] = rng.integers(0, 600, k)
        perm = o + rng.permutation(2 * k)
        mz[o:o + 2 * k], it[o:o + 2 * k] = mz[perm], it[perm]
    d = torch.device("cuda", local)
    t_seg = torch.from_numpy(seg.astype(np.int32)).to(d)
    t_size = torch.from_numpy((2 * lens).astype(np.int32)).to(d)
    t_mz0, t_it0 = torch.from_numpy(mz).to(d), torch.from_numpy(it).to(d)
    t_mz, t_it = t_mz0.clone(), t_it0.clone()
    o_idx = torch.empty(q.n + 1, dtype=torch.int32, device=d)
    o_mz = torch.empty(max(n, 1), dtype=torch.int32, device=d)
    o_it = torch.empty(max(n, 1), dtype=torch.int32, device=d)
    st = torch.cuda.current_stream()
    times = []
    for rep in range(4):
        t_mz.copy_(t_mz0)
        t_it.copy_(t_it0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        N.check(N.lib().gx_pickpeaks_device(q.n, t_seg.data_ptr(), t_size.data_ptr(), t_mz.data_ptr(),
                                            t_it.data_ptr(), 100000, 1000, 100, o_idx.data_ptr(), o_mz.data_ptr(),
                                            o_it.data_ptr(), C.c_void_p(st.cuda_stream)))
        e1.record(st)
        st.synchronize()
        if rep:
            times.append(e0.elapsed_time(e1))
    gpu_ms = float(np.median(times))
    out = {"spectra": int(q.n), "raw_peaks": n, "gpu_ms": round(gpu_ms, 3),
           "gpu_spectra_per_s": round(q.n / (gpu_ms / 1e3), 1)}
    if rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        m = min(2000, q.n)
        t1 = time.perf_counter()
        idx, _, _ = pyoracle.pickpeaks(seg[:m + 1], 2 * lens[:m], mz, it)
        cpu_s = time.perf_counter() - t1
        out["cpu_baseline"] = {"value": round(m / cpu_s, 1), "unit": "spectra/s", "cores": 1, "kind": "port",
                               "sample": f"first {m} spectra"}
        out["kept_counts_equal_on_sample"] = bool(np.array_equal(
            idx.astype(np.int64), o_idx[:m + 1].cpu().numpy().astype(np.int64)))
    log(f"[bench] peak picking: {out['gpu_spectra_per_s']:.0f} spectra/s on the GPU")
    return out


def smi_id(local: int) -> str:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local < len(ids):
            return ids[local]
    return str(local)


def sample_clocks(stop: threading.Event, out: list, gpu: int):
    cmd = ["nvidia-smi", f"--id={smi_id(gpu)}", "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits",
           "-lms", "200"]
    try:
        p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return
    try:
        while not stop.is_set():
            line = p.stdout.readline()
            if not line:
                break
            out.append([x.strip() for x in line.split(",")])
    finally:
        p.terminate()
        p.wait()


def summarize_clocks(rows: list) -> dict:
    if not rows:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
    mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 4 + i and r[4 + i].lower() == "active"})
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": reasons, "samples": len(rows)}


def _harness_run(w: dict, db, parts, steps: int, warmup: int, cores: int) -> list:
    """Per-step query seconds of the reference harness: one index build, then per step every
    (QueryBatch, tolerance in Da) part of `parts` searched in turn (their times summed)."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    with tempfile.TemporaryDirectory() as tmp:
        dbdir = os.path.join(tmp, "db")
        db.write_peps(dbdir)
        cmd = [harness, "--db", dbdir, "--maxz", str(w["maxz"]), "--dF", "5", "--threads", str(cores),
               "--topmatches", "5", "--repeat", str(warmup + steps)]
        for i, (sq, dM) in enumerate(parts):
            qf = os.path.join(tmp, f"q{i}.pbin")
            sq.write_pbin(qf)
            cmd += ["--batch", f"{qf}:{float(dM)!r}"]
        for r, m, n in w["mods"]:
            cmd += ["--mods", f"{r}:{m}:{n}"]
        if w["mods"]:
            cmd += ["--nmods", str(w["nmods"])]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed: {r.stderr[-400:]}")
        rec = json.loads(r.stdout.strip().splitlines()[-1])
    log(f"[bench] reference CPU: {sum(p[0].n for p in parts)} spectra in {len(parts)} batch(es) at dM "
        f"{', '.join('%g' % p[1] for p in parts)} Da x {len(rec['query_s_each'])} repeats, "
        f"index build {rec['index_s']:.1f}s")
    return rec["query_s_each"][warmup:]


def reference_cpu(w: dict, db, q, sel, steps: int, warmup: int):
    """The reference's OpenMP CPU query path (oracle/_ref/ref_harness) on the spectra sel of q.

    The reference reads one global precursor tolerance, so a batch with per-spectrum
    tolerances is timed in two batches: the spectra at the workload's window, and the
    narrow-window spectra at the median of their tolerances (timing only)."""
    cores = os.cpu_count() or 1
    sample = len(sel)
    sq = q.subset(sel)
    if sq.dM is None or np.all(np.isnan(sq.dM)):
        parts = [(sq, w["dM"])]
    else:
        narrow = ~np.isnan(sq.dM)
        parts = []
        for idx, dm in ((np.nonzero(~narrow)[0], w["dM"]), (np.nonzero(narrow)[0], float(np.median(sq.dM[narrow])))):
            if len(idx):
                sub = sq.subset(idx)
                sub.dM = None
                parts.append((sub, dm))
    each = np.asarray(_harness_run(w, db, parts, steps, warmup, cores))
    per = float(np.mean(each))
    log(f"[bench] reference CPU: {sample} spectra, {per:.3f} s per step")
    return dict(value=sample / per, cores=cores, sample=sample, seconds=per, steps=len(each))


def train_tail(ws, qd, params, t_out, t_hist, t_pre, t_chg, device: int, n_train: int, sparse_below: int):
    """The learned tail, trained (untimed) on the batch's own well-populated queries (+-500 Da,
    at least 10^4 candidates): 64 subsamples of each one's histogram against the plain fit of
    all its candidates, with Huber's loss.  The candidate threshold below which the model
    replaces the plain fit is calibrated on 300 other such queries (unless given), and the
    gain reported on 300 held-out ones.  Returns (model or None, info dict)."""
    import torch
    import gicops_b200._native as N
    import gicops_b200.tail as T
    t0 = time.perf_counter()
    stream = torch.cuda.current_stream()
    ws.search_device(qd, params, t_out.data_ptr(), hist_dev=t_hist.data_ptr(), stream=stream.cuda_stream)
    torch.cuda.synchronize()
    res0 = t_out.cpu().numpy().view(N.RESULT_DTYPE)
    pop = np.nonzero(((res0["status"] & 1) != 0) & (res0["cpsms"] >= 10000) & np.isfinite(res0["slope"]) &
                     (res0["slope"] < 0))[0]
    pop = np.random.default_rng(7).permutation(pop)
    held, calib, train = pop[:300], pop[300:600], pop[600:600 + n_train]
    if len(train) < 64:
        return None, {"skipped": f"{len(pop)} well-populated queries"}
    tail = T.TailModel(device, max_batch=8192, seed=11)
    tail.set_loss(0.5)
    dv = dict(hist=t_hist, res=t_out, prec=t_pre, charge=t_chg)
    smp = T.plan(train, per_query=64, keep_range=(8, 512), seed=1)
    xs, ts = T.training_set(tail, dv, res0, smp)
    tail.set_norm_from(ts.cpu().numpy())
    losses = tail.train(xs, ts, epochs=6, batch=512, opt=T.Adam(lr=1e-3, w_slope=0.2), seed=2, lr_decay=0.8)
    del xs, ts
    cal = T.evaluate(tail, dv, res0, T.plan(calib, per_query=8, keep_range=(20, 500), seed=4))
    below = sparse_below or T.choose_sparse_below(cal["err_plain"], cal["err_learned"], cal["cpsms_sub"])
    ev = T.evaluate(tail, dv, res0, T.plan(held, per_query=8, keep_range=(20, 500), seed=3))
    m = ev["cpsms_sub"] < below
    qf = lambda e, f: round(float(np.quantile(e, f)), 3) if len(e) else None  # noqa: E731
    ep, el = ev["err_plain"][m], ev["err_learned"][m]
    info = {"sparse_below": int(below), "sparse_below_from": "argument" if sparse_below else
            "calibration (300 held-out well-populated queries subsampled to 20-500 candidates)",
            "loss": "huber 0.5", "train_queries": int(len(train)), "train_samples": int(len(smp)),
            "train_loss": [round(x, 4) for x in losses], "train_s": round(time.perf_counter() - t0, 2),
            "held_out": {"queries": int(len(held)), "subsamples_below_threshold": int(m.sum()),
                         "abs_log10_e_error_vs_full_fit": {
                             "plain": {"median": qf(ep, .5), "p90": qf(ep, .9), "p99": qf(ep, .99)},
                             "learned": {"median": qf(el, .5), "p90": qf(el, .9), "p99": qf(el, .99)}},
                         "share_within_0.1_log10": {"plain": float(np.mean(ep <= .1)) if len(ep) else None,
                                                    "learned": float(np.mean(el <= .1)) if len(el) else None}}}
    log(f"[bench] learned tail: {info}")
    return (tail if below > 0 else None), info


_STRESS_ENTRIES = None


def _stress_part(n: int, seed: int, qargs: dict):
    from gicops_b200 import synth
    return synth.make_queries(_STRESS_ENTRIES, n, seed=seed, **qargs)


def stream_run(args) -> None:
    """The stress configuration through the streamed entry point: index entries on the host,
    fragment ions, CSR and block layout on the GPU (gx_index_build); 1M spectra, drawn in
    64k-spectrum parts by forked workers before CUDA starts, searched from pinned host memory
    by gx_search_stream with the learned tail attached (trained on the first chunk).  Prints
    one JSON line: spectra/s over the whole streamed batch (GPU clock, first upload to last
    download) and the share of the copies hidden behind the search."""
    global _STRESS_ENTRIES
    import multiprocessing as mp
    import gicops_b200 as gx
    w = STRESS
    t0 = time.time()
    db = gx.synth.make_database(w["nproteins"], seed=w["db_seed"])
    t1 = time.perf_counter()
    E = gx.HostIndex.build(db, maxz=w["maxz"], mods=w["mods"], nmods=w["nmods"], ions=False)
    entries_s = time.perf_counter() - t1
    del db
    _STRESS_ENTRIES = E.entries_by_len()
    nspec = args.stream_spectra or w["nspec"]
    parts = [(min(w["chunk"], nspec - i), 5000 + k) for k, i in enumerate(range(0, nspec, w["chunk"]))]
    with mp.get_context("fork").Pool(min(len(parts), os.cpu_count() or 1)) as pool:   # before any CUDA call
        q = gx.synth.QueryBatch.concat(pool.starmap(_stress_part, [(n, sd, w["q"]) for n, sd in parts]))
    log(f"[stress] {E.total_entries()} entries, {q.n} spectra, {len(q.moz)} peaks ({time.time() - t0:.1f}s)")

    import torch
    import gicops_b200._native as N
    torch.cuda.set_device(0)
    d = torch.device("cuda", 0)
    t1 = time.perf_counter()
    dev = gx.DeviceIndex(E, 0)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t1
    log(f"[stress] device index {dev.nbytes / 1e9:.1f} GB built in {build_s:.1f}s")
    params = gx.SearchParams(dM=w["dM"], dF=5, topmatches=5, expect_max=20.0)
    tail = tail_info = None
    if not args.no_tail:
        q0 = q.subset(np.arange(min(w["chunk"], q.n)))
        ws0 = gx.Searcher(dev, q0.n, len(q0.moz))
        t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(d) for k, v in
             dict(idx=q0.idx.view(np.int32), moz=q0.moz, intn=q0.intn, prec=q0.prec,
                  charge=q0.charge.astype(np.int32)).items()}
        qd0 = dict(nspec=q0.n, npeaks=len(q0.moz), **{k: v.data_ptr() for k, v in t.items()})
        out0 = torch.empty(q0.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=d)
        hist0 = torch.empty((q0.n, N.HIST_BINS), dtype=torch.int32, device=d)
        tail, tail_info = train_tail(ws0, qd0, params, out0, hist0, t["prec"], t["charge"], 0, args.tail_queries,
                                     args.sparse_below)
        del ws0, out0, hist0, t
    st = gx.Streamer(dev, chunk=w["chunk"])
    if tail is not None:
        st.set_tail(tail, tail_info["sparse_below"])
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    qp = gx.synth.QueryBatch(pin(q.idx), pin(q.moz), pin(q.intn), pin(q.prec), pin(q.charge.astype(np.int32)),
                             q.rtime)
    out = torch.empty(q.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory().numpy().view(N.RESULT_DTYPE)
    st.search(qp.subset(np.arange(min(2 * w["chunk"], q.n))), params)          # warm-up: two chunks
    clocks, stop = [], threading.Event()
    th = threading.Thread(target=sample_clocks, args=(stop, clocks, 0), daemon=True)
    th.start()
    time.sleep(0.5)
    t1 = time.perf_counter()
    res, stats = st.search(qp, params, out=out, stats=True)
    wall = time.perf_counter() - t1
    stop.set()
    th.join(timeout=5)
    copies = stats["upload_ms"] + stats["download_ms"]
    hidden = stats["upload_ms"] + stats["search_ms"] + stats["download_ms"] - stats["total_ms"]
    line = {"metric": "streamed query spectra/s (stress configuration)", "value": q.n / (stats["total_ms"] / 1e3),
            "unit": "spectra/s", "n_gpus": 1, "wall_s": round(wall, 2), "host_wall_spectra_per_s": q.n / wall,
            "stream": {k: (round(v, 2) if isinstance(v, float) else v) for k, v in stats.items()},
            "copies_hidden_share": round(max(0.0, min(1.0, hidden / copies)), 3) if copies > 0 else None,
            "search_share_of_total": round(stats["search_ms"] / stats["total_ms"], 3),
            "config": {"proteins": w["nproteins"], "index_entries": E.total_entries(), "spectra": q.n,
                       "chunk": w["chunk"], "window_da": w["dM"], "index_gb": round(dev.nbytes / 1e9, 1),
                       "entries_s": round(entries_s, 1), "device_build_s": round(build_s, 1)},
            "learned_tail": dict(tail_info or {}, queries_replaced=int(
                ((res["status"] & N.STATUS_LEARNED_TAIL) != 0).sum())) if tail is not None else tail_info,
            "reported_psms": int(((res["status"] & 2) != 0).sum()),
            "clocks": summarize_clocks(clocks)}
    print(json.dumps(line), flush=True)


def parity_block(gx, N, H, q, params, w, run_full, tail_on: bool, n_sample: int = 256, n_hyp: int = 32) -> dict:
    """Untimed check of the benchmarked batch's own outputs: one more search of the whole
    batch (the timed step's launch sequence, with heap and histogram outputs) against the
    oracle on a seeded sample of its spectra.  Exact: candidate counts, histograms, heap
    arrays, top PSMs, and the tail fit of every query that kept the plain fit; FP64 slope
    and e-value to 1e-12 / 1e-9 relative.  Accuracy: the top PSMs' FP32 hyperscores
    against FP64 (n_hyp spectra), the reference's quantized e-value against the
    unquantized FP64 fit, and the learned tail's e-values against the plain FP64 fit of
    the same histograms (every query of the batch that took it)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    rng = np.random.Generator(np.random.PCG64(3))
    sel = np.sort(rng.choice(q.n, size=min(q.n, n_sample), replace=False))
    res_all, heap, hist = run_full(sel)
    res = res_all[sel]
    sq = q.subset(sel)
    t0 = time.perf_counter()
    o, oh = pyoracle.search(H.lengths, sq, pyoracle.Params(dM=w["dM"], topmatches=params.topmatches,
                                                           expect_max=params.expect_max), hist=True)
    oracle_s = time.perf_counter() - t0
    learned = (res["status"] & N.STATUS_LEARNED_TAIL) != 0
    fitted = (o["status"] & 1) != 0
    heaps_ok = True
    for i in range(len(sel)):
        k = int(o["heap_size"][i])
        a_, b_ = heap[i][:k], o["heap"][i][:k]
        heaps_ok &= bool(np.array_equal(a_["psid"], b_["psid"]) and np.array_equal(a_["idxoffset"], b_["idxoffset"])
                         and np.array_equal(a_["sharedions"], b_["sharedions"])
                         and np.array_equal(a_["hyperscore"].view(np.uint32), b_["hyperscore"].view(np.uint32)))
    top_ok = all(np.array_equal(res["top"][f][fitted], o["top"][f][fitted])
                 for f in ("psid", "idxoffset", "sharedions", "totalions")) and \
        np.array_equal(res["top"]["hyperscore"][fitted].view(np.uint32), o["top"]["hyperscore"][fitted].view(np.uint32))
    plain = fitted & ~learned
    fit_ok = all(np.array_equal(res[f][plain], o[f][plain]) for f in ("maxhyp", "mu", "beta", "stt1", "end1")) and \
        np.array_equal(res["status"][plain] & 7, o["status"][plain] & 7) and \
        np.array_equal(res["status"][learned] & 5, o["status"][learned] & 5)
    fin = fitted & np.isfinite(o["e_fp64"]) & (o["e_fp64"] > 0)
    rel = lambda x, y: float(np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300))) if len(y) else 0.0  # noqa: E731
    e_rel = rel(res["e_x"][plain & fin], o["e_x"][plain & fin])
    fp64_rel = rel(res["e_fp64"][fin], o["e_fp64"][fin])
    slope_rel = rel(res["slope"][fin], o["slope"][fin])
    # hyperscore of the top PSM in FP32 against its FP64 value, from that candidate's matched
    # ions counted in the index's own buckets (dslim_query.cpp:853-914 for one candidate)
    lg = pyoracle.lgfact()
    hyp_err = 0.0
    dF = params.dF
    for i in np.nonzero(fitted)[0][:n_hyp]:
        t = res["top"][i]
        ln = H.lengths[int(t["idxoffset"])]
        speclen = int(ln["speclen"])
        bA, iA = ln["bA"], ln["iA"]
        a0, a1 = int(sq.idx[i]), int(sq.idx[i + 1])
        bc = yc = ibc = iyc = 0
        for mz, it in zip(sq.moz[a0:a1].astype(np.int64), sq.intn[a0:a1].astype(np.int64)):
            if not (mz > dF and mz < params.max_mass * params.scale - 1 - dF):
                continue
            ids = iA[int(bA[mz - dF]):int(bA[mz + dF + 1])].astype(np.int64)
            hit = ids[ids // speclen == int(t["psid"])]
            ny = int(np.count_nonzero((hit % speclen) // (speclen // 2)))
            nb = len(hit) - ny
            bc, yc, ibc, iyc = bc + nb, yc + ny, ibc + nb * int(it), iyc + ny * int(it)
        ibc, iyc = ibc % (1 << 32), iyc % (1 << 32)
        h64 = lg[min(bc, 80)] + lg[min(yc, 80)] + np.log10(1.0 + ibc) + np.log10(1.0 + iyc) - 4.0
        if bc + yc == int(t["sharedions"]) and 0 < h64 < 80:   # hyperscores of 80 and above are clamped to 79
            hyp_err = max(hyp_err, abs(float(t["hyperscore"]) - h64) / abs(h64))
    # the reference's e-value (slope/intercept truncated to 1e-6) against the unquantized fit
    q_fit = plain & fin & (res["e_x"] > 0)
    dq = np.abs(np.log10(res["e_x"][q_fit]) - np.log10(o["e_fp64"][q_fit])) if q_fit.any() else np.zeros(1)
    out = {"sample": int(len(sel)), "sample_seed": 3, "oracle_s": round(oracle_s, 2),
           "cpsms_equal": bool(np.array_equal(res["cpsms"], o["cpsms"])),
           "histograms_equal": bool(np.array_equal(hist, oh)), "heaps_equal": bool(heaps_ok),
           "top_psm_equal": bool(top_ok), "tail_fit_equal": bool(fit_ok),
           "e_x_max_rel_err": e_rel, "e_fp64_max_rel_err": fp64_rel, "slope_max_rel_err": slope_rel,
           "hyperscore_fp32_vs_fp64_max_rel_err": hyp_err, "hyperscore_spectra": int(min(n_hyp, fitted.sum())),
           "e_quantized_vs_fp64_log10": {"median": float(np.median(dq)), "max": float(np.max(dq))},
           "fitted_in_sample": int(fitted.sum())}
    if tail_on:
        L = ((res_all["status"] & N.STATUS_LEARNED_TAIL) != 0) & (res_all["e_x"] > 0) & (res_all["e_fp64"] > 0)
        d = np.abs(np.log10(res_all["e_x"][L]) - np.log10(res_all["e_fp64"][L])) if L.any() else np.zeros(0)
        out["learned_tail_vs_plain_fit"] = {
            "queries": int(L.sum()),
            "share_within_0.1_log10": float(np.mean(d <= 0.1)) if len(d) else None,
            "median_abs_log10": float(np.median(d)) if len(d) else None}
    out["all_exact"] = bool(out["cpsms_equal"] and out["histograms_equal"] and out["heaps_equal"] and
                            out["top_psm_equal"] and out["tail_fit_equal"] and e_rel <= 1e-9 and fp64_rel <= 1e-9)
    log(f"[bench] parity on {len(sel)} sampled spectra: exact={out['all_exact']} (oracle {oracle_s:.1f}s)")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="large-200k", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain", action="store_true", help="time the plain one-spectrum-per-CTA path instead")
    ap.add_argument("--plain-sample", type=int, default=4096,
                    help="spectra of the seeded sample the plain path is timed on (0: leave it out)")
    ap.add_argument("--parity-sample", type=int, default=256,
                    help="spectra of the seeded sample checked against the oracle (0: leave it out)")
    ap.add_argument("--spectra", type=int, default=0, help="search only the first N spectra (profiling cases)")
    ap.add_argument("--no-tail", action="store_true", help="leave the learned tail out of the step")
    ap.add_argument("--no-index-build", action="store_true", help="skip timing the GPU index build at set-up")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape")
    ap.add_argument("--no-graph", action="store_true", help="launch the step's kernels directly (no CUDA graph)")
    ap.add_argument("--sparse-below", type=int, default=0,
                    help="queries with fewer candidate PSMs take the learned tail (0: calibrated)")
    ap.add_argument("--tail-queries", type=int, default=16000,
                    help="well-populated queries the learned tail is trained on (64 subsamples each)")
    ap.add_argument("--stream-run", action="store_true",
                    help="the stress configuration streamed through gx_search_stream (its own JSON line)")
    ap.add_argument("--stream-spectra", type=int, default=0, help="spectra of the stress run (0: 1M)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.stream_run:
        stream_run(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric = "query spectra/s"
    unit = "spectra/s"

    if args.impl == "reference":
        if rank != 0:
            return
        w, db, q = make_reference_workload(args.workload)
        sel = ref_sample(args.workload, q.n)
        ref = reference_cpu(w, db, q, sel, args.steps, args.warmup)
        line = {"metric": metric, "value": ref["value"], "unit": unit, "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ref["seconds"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32+f64",
                "data": "synthetic (seeded generator)",
                "config": {"workload": args.workload, "spectra_per_step": ref["sample"],
                           "window_da": w["dM"] if q.dM is None else "half +-10 ppm, half +-%g Da" % w["dM"],
                           "sample": f"seeded subset (PCG64 seed 7) of the workload's {w['nspec']} spectra, "
                                     "the same subset the GPU arm's cpu_baseline times"},
                "cpu_baseline": {"value": ref["value"], "unit": unit, "cores": ref["cores"], "kind": "reference",
                                 "sample": f"{ref['sample']} of the workload's {w['nspec']} spectra per step"},
                "e2e": {"value": ref["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import gicops_b200 as gx
    from gicops_b200.search import algorithmic_bytes
    import gicops_b200._native as N

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    w, db, H, q = make_workload(args.workload, rank)
    if args.spectra:
        q = q.subset(np.arange(min(args.spectra, q.n)))
    params = gx.SearchParams(dM=w["dM"], dF=5, topmatches=5, expect_max=20.0,
                             flags=gx.FLAG_PLAIN if args.plain else 0)
    t1 = time.perf_counter()
    dev = gx.DeviceIndex(H, local)
    upload_s = time.perf_counter() - t1
    extras = world == 1   # set-up measurements beside the step: one process only
    # ---- index build: the same index with its fragment ions, CSR and block layout computed
    # on the GPU (entries on the host), against the host build + upload above (untimed setup)
    index_build = None
    if extras and not args.no_index_build:
        t1 = time.perf_counter()
        E = gx.HostIndex.build(db, maxz=w["maxz"], mods=w["mods"], nmods=w["nmods"], ions=False)
        entries_s = time.perf_counter() - t1
        t1 = time.perf_counter()
        D = gx.DeviceIndex(E, local)
        device_s = time.perf_counter() - t1
        D.close()
        E.close()
        index_build = {"host_build_s": round(w["host_build_s"], 3), "upload_s": round(upload_s, 3),
                       "entries_s": round(entries_s, 3), "device_ions_s": round(device_s, 3),
                       "host_path_s": round(w["host_build_s"] + upload_s, 3),
                       "device_path_s": round(entries_s + device_s, 3),
                       "host_threads": os.cpu_count()}
        log(f"[bench] index build: host {index_build['host_path_s']} s (build + upload), "
            f"device {index_build['device_path_s']} s (entries + GPU ions/CSR)")
    prep = prep_measure(gx, q, local, rank) if extras and not args.no_index_build else None
    ws = gx.Searcher(dev, q.n, len(q.moz))
    stream = torch.cuda.current_stream()
    d = torch.device("cuda", local)

    def device_queries(qq):
        t = dict(idx=torch.from_numpy(qq.idx.view(np.int32).copy()).to(d), moz=torch.from_numpy(qq.moz.copy()).to(d),
                 intn=torch.from_numpy(qq.intn.copy()).to(d), prec=torch.from_numpy(qq.prec.copy()).to(d),
                 charge=torch.from_numpy(qq.charge.astype(np.int32)).to(d))
        if qq.dM is not None:   # per-spectrum precursor tolerances (Da)
            t["dM"] = torch.from_numpy(np.where(np.isnan(qq.dM), w["dM"], qq.dM).astype(np.float64)).to(d)
        qd_ = dict(nspec=qq.n, npeaks=len(qq.moz), **{k: v.data_ptr() for k, v in t.items()})
        return qd_, t

    qd, qt = device_queries(q)
    t_pre, t_chg = qt["prec"], qt["charge"]
    t_out = torch.empty(q.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=d)
    t_hist = torch.empty((q.n, N.HIST_BINS), dtype=torch.int32, device=d)

    # ---- learned tail: trained here (untimed) on this workload's well-populated queries --
    tail = None
    tail_info = None
    if not args.no_tail and not args.plain:
        tail, tail_info = train_tail(ws, qd, params, t_out, t_hist, t_pre, t_chg, local, args.tail_queries,
                                     args.sparse_below)
        if tail is not None:
            ws.set_tail(tail, tail_info["sparse_below"])   # every search below applies it after the plain fit

    # ---- launch shape: the autotuner times every candidate on a seeded sample of the batch
    tiles = None
    if not args.plain and not args.no_autotune:
        sel = np.sort(np.random.Generator(np.random.PCG64(9)).choice(q.n, size=min(q.n, 4096), replace=False))
        tqd, tkeep = device_queries(q.subset(sel))
        t0 = time.perf_counter()
        tr = ws.autotune(tqd, params, reps=3, use_cache=False, stream=stream.cuda_stream)
        tiles = {"chosen": tr["best"], "sample": int(len(sel)), "tune_s": round(time.perf_counter() - t0, 2),
                 "candidates_ms": [[c["chunks_per_lane"], c["ctas_per_sm"], c["tile"], c["sorted"], c["pipeline"],
                                    round(c["ms"], 3)] for c in tr["candidates"]],
                 "candidate_fields": ["chunks_per_lane", "ctas_per_sm", "tile", "sorted", "pipeline", "ms"]}
        log(f"[bench] autotuned launch shape: {tr['best']} ({tiles['tune_s']} s)")
        del tqd, tkeep

    # the step's launch sequence is captured once in a CUDA graph and replayed
    use_graph = not args.plain and not args.no_graph
    if use_graph:
        ws.set_graph(True)

    def step():
        ws.search_device(qd, params, t_out.data_ptr(), stream=stream.cuda_stream)

    # an index smaller than twice L2 (126 MB) is flushed from L2 between timed steps by
    # writing a 256 MB buffer on the same stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=d) if dev.nbytes < 252e6 else None

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region (device events, queries resident in HBM) ---------------------
    clocks, stop = [], threading.Event()
    th = threading.Thread(target=sample_clocks, args=(stop, clocks, local), daemon=True)
    th.start()
    time.sleep(0.5)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = gx.lib().gx_launch_count()
    if flush is None:   # index larger than L2: steps back to back
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    else:               # index fits L2: flush it before each step, time each step alone
        ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
    launches = int(gx.lib().gx_launch_count() - n0)
    stop.set()
    th.join(timeout=5)
    if dist:
        t = torch.tensor([ms], device=d)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = q.n * world / (ms_step / 1e3)

    # ---- dominant kernel duration (events around each launch, same stream) --------
    prof_steps = min(args.steps, 3)
    gx.lib().gx_profile_enable(1)
    for _ in range(prof_steps):
        step()
    torch.cuda.synchronize()
    kt = N.kernel_times()
    gx.lib().gx_profile_enable(0)
    top_k = max(kt, key=lambda k: kt[k][1])
    k_ms = kt[top_k][1] / kt[top_k][0]

    # ---- end to end through the C ABI with host buffers (gx_search_host: pinned host
    # queries copied in, search, learned tail when attached, results copied out) ------
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    qp = gx.synth.QueryBatch(pin(q.idx), pin(q.moz), pin(q.intn), pin(q.prec), pin(q.charge.astype(np.int32)),
                             q.rtime, None if q.dM is None else pin(np.where(np.isnan(q.dM), w["dM"], q.dM)))
    out_pinned = torch.empty(q.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory().numpy()
    from gicops_b200.search import make_c_queries
    import ctypes as C
    cq, keep = make_c_queries(qp, params)
    cp = params.c()
    e2e_steps = min(args.steps, 5)

    def e2e_step():
        N.check(gx.lib().gx_search_host(dev.handle, ws.handle, C.byref(cq), C.byref(cp), out_pinned.ctypes.data,
                                        None, None))

    for _ in range(2):
        e2e_step()
    if dist:
        dist.barrier()
    if flush is None:
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = (time.perf_counter() - t0) / e2e_steps
    else:
        e2e_s = 0.0
        for _ in range(e2e_steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            e2e_s += time.perf_counter() - t0
        e2e_s /= e2e_steps
    if dist:
        t = torch.tensor([e2e_s], device=d)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = q.idx.nbytes + q.moz.nbytes + q.intn.nbytes + q.prec.nbytes + 4 * q.n + (8 * q.n if q.dM is not None else 0)
    d2h = q.n * N.RESULT_DTYPE.itemsize + 4

    # ---- roofline numerator: algorithmic bytes of one launch ------------------------
    rs = np.random.Generator(np.random.PCG64(3)).choice(q.n, size=min(q.n, 4096), replace=False)
    ab = algorithmic_bytes(H, q.subset(np.sort(rs)), params)
    bytes_launch = float(ab.mean()) * q.n
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_launch / (k_ms / 1e3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tf):
        tj = json.load(open(tf))
        ent = tj.get(args.workload, {}).get(top_k)
        if ent:   # per launch of the workload's whole batch; a --spectra case scales by spectra
            traffic = ent["dram_bytes_per_launch"] * q.n / ent["launch_spectra"]

    # ---- parity of the benchmarked outputs (untimed) --------------------------------
    parity = None
    if rank == 0 and args.parity_sample and not args.plain:
        cap = params.heap_cap
        t_heap = torch.empty(q.n * cap * N.CELL_DTYPE.itemsize, dtype=torch.uint8, device=d)

        def run_full(sel):
            ws.search_device(qd, params, t_out.data_ptr(), t_heap.data_ptr(), t_hist.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
            ix = torch.from_numpy(sel.astype(np.int64)).to(d)
            res_all = t_out.cpu().numpy().view(N.RESULT_DTYPE).copy()
            hp = t_heap.view(q.n, -1).index_select(0, ix).cpu().numpy().view(N.CELL_DTYPE).reshape(len(sel), cap)
            hs = t_hist.index_select(0, ix).cpu().numpy().view(np.uint32)
            return res_all, hp, hs

        parity = parity_block(gx, N, H, q, params, w, run_full, tail is not None, n_sample=args.parity_sample)
        del t_heap
    del t_hist

    # ---- the plain one-spectrum-per-CTA path and the batched path on one seeded sample --
    plain = None
    if args.plain_sample and not args.plain:
        import dataclasses
        sel = np.sort(np.random.Generator(np.random.PCG64(5)).choice(q.n, size=min(q.n, args.plain_sample),
                                                                    replace=False))
        sq = q.subset(sel)
        sqd, skeep = device_queries(sq)
        s_out = torch.empty(sq.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=d)
        pp = dataclasses.replace(params, flags=gx.FLAG_PLAIN)

        def timed(prm):
            ws.search_device(sqd, prm, s_out.data_ptr(), stream=stream.cuda_stream)   # warm-up
            torch.cuda.synchronize()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            ws.search_device(sqd, prm, s_out.data_ptr(), stream=stream.cuda_stream)
            a1.record(stream)
            torch.cuda.synchronize()
            return a0.elapsed_time(a1)

        pl_ms, bt_ms = timed(pp), timed(params)
        plain = {"value": sq.n / (pl_ms / 1e3), "unit": unit, "sample": int(sq.n), "sample_seed": 5,
                 "batched_same_sample": sq.n / (bt_ms / 1e3), "batched_over_plain_same_sample": pl_ms / bt_ms,
                 "batched_full_batch_over_plain": value / world / (sq.n / (pl_ms / 1e3))}
        log(f"[bench] plain path: {plain['value']:.0f} spectra/s on {sq.n} spectra "
            f"(batched on the same: {plain['batched_same_sample']:.0f})")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref = reference_cpu(w, db, q, ref_sample(args.workload, q.n), steps=1, warmup=1)
            cpu = {"value": ref["value"], "unit": unit, "cores": ref["cores"], "kind": "reference",
                   "sample": f"{ref['sample']} of {q.n} spectra (seeded subset, PCG64 seed 7), reference "
                             f"DSLIM_QuerySpectrum, all {ref['cores']} host threads, query time only"}
        except Exception as ex:  # the checker binary may be absent on a machine without the reference build
            log(f"[bench] reference CPU baseline unavailable: {ex}")

    if rank == 0:
        line = {
            "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32+f64", "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": args.workload + (f" (first {q.n} spectra)" if args.spectra else ""),
                       "spectra_per_gpu": q.n, "proteins": w["nproteins"],
                       "index_entries": H.total_entries(), "index_ion_ids": H.total_ions(),
                       "window_da": w["dM"] if q.dM is None else "half +-10 ppm, half +-%g Da" % w["dM"],
                       "frag_tol_bins": 5, "topK": 5,
                       "l2": ("inputs larger than L2 (index %.2f GB)" % (dev.nbytes / 1e9)) if flush is None else
                             ("L2 flushed before each timed step (index %.1f MB)" % (dev.nbytes / 1e6)),
                       "parallelism": f"replicas x{world}",
                       "reference_sample": f"the reference CPU path is timed on a seeded subset of "
                                           f"{len(ref_sample(args.workload, q.n))} of these {q.n} spectra (PCG64 "
                                           "seed 7; its whole batch would take minutes per step); the subset is a "
                                           "uniform draw from the same batch"},
            "e2e": {"value": q.n * world / e2e_s, "unit": unit, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
            "roofline": {"bound": "hbm", "kernel": top_k, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": bytes_launch, "kernel_ms": k_ms,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback"},
            "kernel_ms": {k: v[1] / v[0] for k, v in kt.items()},
            "gpu_launches": launches,
            "cuda_graph": use_graph,
            "tiles": tiles if tiles else {"chosen": ws.tiles, "autotuned": False},
            "path": "plain" if args.plain else ("batched+learned tail" if tail else "batched"),
            "parity": parity,
            "index_build": index_build,
            "prep": prep,
            "learned_tail": dict(tail_info or {}, queries_replaced=int(
                ((t_out.cpu().numpy().view(N.RESULT_DTYPE)["status"] & N.STATUS_LEARNED_TAIL) != 0).sum()))
            if tail else None,
            "plain_path": plain,
            "clocks": summarize_clocks(clocks),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
