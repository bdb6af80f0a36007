"""Benchmark of the peptide-search query path (spectra/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload open-20k] [--impl ours|reference]

A step is one search of the whole synthetic batch (default: the open-search
workload -- 20,000 proteins, Met oxidation <= 2, b/y ions of charge 1-2, 50,000
spectra of 30-150 peaks, +-500 Da precursor window, +-0.05 Da fragment tolerance,
top-K 5).  Its index (2.8 GB) is larger than L2, so steps run back to back; an
index smaller than twice L2 (the closed-1k workload's) is flushed from L2 before each
timed step instead, and the step timed alone.

Printed (rank 0, one JSON line): value = spectra/s with queries resident in HBM
(CUDA events on the launching stream, max over ranks); e2e = spectra/s through
the host-buffer API (pinned host queries in, results out, per step); roofline of
the dominant kernel against the measured HBM copy bandwidth; cpu_baseline = the
reference's own OpenMP CPU query path timed on a bounded sample on this host.

Under torchrun each rank searches its own batch against a replica of the index
(spectra are independent: weak scaling, no collective on the data path).
``--impl reference`` times the reference's CPU implementation alone (rank 0).
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


def log(*a):
    print(*a, file=sys.stderr, flush=True)


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


def _harness_run(w: dict, db, sq, steps: int, warmup: int, cores: int, dM: float) -> list:
    """Per-step query seconds of the reference harness on the batch sq at tolerance dM."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    with tempfile.TemporaryDirectory() as tmp:
        dbdir = os.path.join(tmp, "db")
        db.write_peps(dbdir)
        qf = os.path.join(tmp, "q.pbin")
        sq.write_pbin(qf)
        cmd = [harness, "--db", dbdir, "--maxz", str(w["maxz"]), "--dM", repr(float(dM)), "--dF", "5",
               "--threads", str(cores), "--topmatches", "5", "--queries", qf, "--repeat", str(warmup + steps)]
        for r, m, n in w["mods"]:
            cmd += ["--mods", f"{r}:{m}:{n}"]
        if w["mods"]:
            cmd += ["--nmods", str(w["nmods"])]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed: {r.stderr[-400:]}")
        rec = json.loads(r.stdout.strip().splitlines()[-1])
    log(f"[bench] reference CPU: {sq.n} spectra at dM {dM:g} Da x {len(rec['query_s_each'])} repeats, "
        f"index build {rec['index_s']:.1f}s")
    return rec["query_s_each"][warmup:]


def reference_cpu(w: dict, db, q, steps: int, warmup: int, sample: int | None = None):
    """The reference's OpenMP CPU query path (oracle/_ref/ref_harness) on a sample of q.

    The reference reads one global precursor tolerance, so a batch with per-spectrum
    tolerances is timed in two batches: the spectra at the workload's window, and the
    narrow-window spectra at the median of their tolerances (timing only)."""
    cores = os.cpu_count() or 1
    if sample is None:
        sample = int(min(q.n, max(2048, min(16384, 128 * cores))))
    sel = np.random.Generator(np.random.PCG64(7)).choice(q.n, size=sample, replace=False)
    sel.sort()
    sq = q.subset(sel)
    if sq.dM is None or np.all(np.isnan(sq.dM)):
        each = _harness_run(w, db, sq, steps, warmup, cores, w["dM"])
    else:
        narrow = ~np.isnan(sq.dM)
        parts = [(np.nonzero(~narrow)[0], w["dM"]), (np.nonzero(narrow)[0], float(np.median(sq.dM[narrow])))]
        each = None
        for idx, dm in parts:
            if not len(idx):
                continue
            sub = sq.subset(idx)
            sub.dM = None
            e = np.asarray(_harness_run(w, db, sub, steps, warmup, cores, dm))
            each = e if each is None else each + e
    per = float(np.mean(each))
    log(f"[bench] reference CPU: {sample} spectra, {per:.3f} s per step")
    return dict(value=sample / per, cores=cores, sample=sample, seconds=per, steps=len(each))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="open-20k", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain", action="store_true", help="time the plain one-spectrum-per-CTA path instead")
    ap.add_argument("--compare-plain", action="store_true", help="also time one step of the plain path")
    ap.add_argument("--spectra", type=int, default=0, help="search only the first N spectra (profiling cases)")
    ap.add_argument("--no-tail", action="store_true", help="leave the learned tail out of the step")
    ap.add_argument("--no-index-build", action="store_true", help="skip timing the GPU index build at set-up")
    ap.add_argument("--sparse-below", type=int, default=500,
                    help="queries with fewer candidate PSMs take the learned tail")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric = "query spectra/s"
    unit = "spectra/s"

    if args.impl == "reference":
        if rank != 0:
            return
        w, db, H, q = make_workload(args.workload, 0)
        ref = reference_cpu(w, db, q, args.steps, args.warmup)
        line = {"metric": metric, "value": ref["value"], "unit": unit, "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ref["seconds"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32+f64",
                "data": "synthetic (seeded generator)",
                "config": {"workload": args.workload, "spectra_per_step": ref["sample"],
                           "window_da": w["dM"] if q.dM is None else "half +-10 ppm, half +-%g Da" % w["dM"]},
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
    # ---- index build: the same index with its fragment ions, CSR and block layout computed
    # on the GPU (entries on the host), against the host build + upload above (untimed setup)
    index_build = None
    if not args.no_index_build:
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
    prep = None if args.no_index_build else prep_measure(gx, q, local, rank)
    ws = gx.Searcher(dev, q.n, len(q.moz))
    stream = torch.cuda.current_stream()
    d = torch.device("cuda", local)
    t_idx = torch.from_numpy(q.idx.view(np.int32).copy()).to(d)
    t_moz = torch.from_numpy(q.moz.copy()).to(d)
    t_int = torch.from_numpy(q.intn.copy()).to(d)
    t_pre = torch.from_numpy(q.prec.copy()).to(d)
    t_chg = torch.from_numpy(q.charge.astype(np.int32)).to(d)
    t_out = torch.empty(q.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=d)
    t_hist = torch.empty((q.n, N.HIST_BINS), dtype=torch.int32, device=d)
    qd = dict(nspec=q.n, npeaks=len(q.moz), idx=t_idx.data_ptr(), moz=t_moz.data_ptr(), intn=t_int.data_ptr(),
              prec=t_pre.data_ptr(), charge=t_chg.data_ptr())
    if q.dM is not None:   # per-spectrum precursor tolerances (Da)
        t_dm = torch.from_numpy(np.where(np.isnan(q.dM), w["dM"], q.dM).astype(np.float64)).to(d)
        qd["dM"] = t_dm.data_ptr()

    # ---- learned tail: trained here (untimed) on this workload's well-populated queries --
    tail = None
    tail_info = None
    if not args.no_tail and not args.plain:
        import gicops_b200.tail as T
        t0 = time.perf_counter()
        ws.search_device(qd, params, t_out.data_ptr(), hist_dev=t_hist.data_ptr(), stream=stream.cuda_stream)
        torch.cuda.synchronize()
        res0 = t_out.cpu().numpy().view(N.RESULT_DTYPE)
        pop = np.nonzero(((res0["status"] & 1) != 0) & (res0["cpsms"] >= 10000) & np.isfinite(res0["slope"]) &
                         (res0["slope"] < 0))[0]
        rng = np.random.default_rng(7)
        pop = rng.permutation(pop)[:4000]
        tail = T.TailModel(local, max_batch=8192, seed=11)
        if len(pop) >= 64:
            dv = dict(hist=t_hist, res=t_out, prec=t_pre, charge=t_chg)
            smp = T.plan(pop, per_query=32, keep_range=(8, 512), seed=1)
            xs, ts = T.training_set(tail, dv, res0, smp)
            tail.set_norm_from(ts.cpu().numpy())
            losses = tail.train(xs, ts, epochs=6, batch=512, opt=T.Adam(lr=1e-3), seed=2, lr_decay=0.8)
            tail_info = {"sparse_below": args.sparse_below, "train_queries": int(len(pop)),
                         "train_samples": int(len(smp)), "train_loss": [round(x, 4) for x in losses],
                         "train_s": round(time.perf_counter() - t0, 2)}
            ws.set_tail(tail, args.sparse_below)   # every search below applies it after the plain fit
        else:
            tail = None
        log(f"[bench] learned tail: {tail_info}")
    del t_hist

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
    gx.lib().gx_profile_enable(1)
    for _ in range(args.steps):
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
                             q.rtime, q.dM)
    out_pinned = torch.empty(q.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory().numpy()
    from gicops_b200.search import make_c_queries
    import ctypes as C
    cq, keep = make_c_queries(qp, params)
    cp = params.c()

    def e2e_step():
        N.check(gx.lib().gx_search_host(dev.handle, ws.handle, C.byref(cq), C.byref(cp), out_pinned.ctypes.data,
                                        None, None))

    for _ in range(2):
        e2e_step()
    if dist:
        dist.barrier()
    if flush is None:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        e2e_s = (time.perf_counter() - t0) / args.steps
    else:
        e2e_s = 0.0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            e2e_s += time.perf_counter() - t0
        e2e_s /= args.steps
    if dist:
        t = torch.tensor([e2e_s], device=d)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = q.idx.nbytes + q.moz.nbytes + q.intn.nbytes + q.prec.nbytes + 4 * q.n
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
        if ent:
            traffic = ent["dram_bytes_per_launch"]

    plain = None
    if args.compare_plain and not args.plain:
        import dataclasses
        pp = dataclasses.replace(params, flags=gx.FLAG_PLAIN)
        ws.search_device(qd, pp, t_out.data_ptr(), stream=stream.cuda_stream)
        torch.cuda.synchronize()
        e0.record(stream)
        ws.search_device(qd, pp, t_out.data_ptr(), stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        plain = {"value": q.n / (e0.elapsed_time(e1) / 1e3), "unit": unit, "steps": 1}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref = reference_cpu(w, db, q, steps=1, warmup=1)
            cpu = {"value": ref["value"], "unit": unit, "cores": ref["cores"], "kind": "reference",
                   "sample": f"{ref['sample']} of {q.n} spectra, reference DSLIM_QuerySpectrum, "
                             f"all {ref['cores']} host threads, query time only"}
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
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": q.n * world / e2e_s, "unit": unit, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "kernel": top_k, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": bytes_launch, "kernel_ms": k_ms,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback"},
            "kernel_ms": {k: v[1] / v[0] for k, v in kt.items()},
            "gpu_launches": launches,
            "path": "plain" if args.plain else ("batched+learned tail" if tail else "batched"),
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
