"""Learned tail model on the B200, through the C ABI (gx_tail_*):

* the tensor-core GEMM against an FP64 product of the same bf16 operands;
* feature rows, subsampled histograms and plain fits bit-exact against the oracle
  (oracle/tail_mlp.py, oracle/restate.c);
* gradients of the forward/backward kernels against the FP64 oracle network that rounds
  to bf16 at the same points, and one Adam step against the oracle's;
* training on the GPU and the gain over the plain fit on held-out well-populated queries
  subsampled to 100-500 candidates, scored against the plain fit of all their candidates;
* the fallback policy on search results.
"""

import numpy as np
import pytest

from conftest import has_gpu, search_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    return torch


def _bf16(torch, shape, gen, scale=1.0):
    return (torch.randn(*shape, generator=gen) * scale).to(torch.bfloat16)


@pytest.mark.parametrize("M,N,K,ta,tb", [
    (300, 256, 132, False, False),   # hidden layer 1 forward
    (256, 132, 384, True, True),     # weight gradient of layer 1
    (512, 2, 256, False, False),     # output layer
    (2, 256, 200, True, True),       # weight gradient of the output layer
    (128, 256, 2, False, True),      # output gradient back through W3
    (130, 48, 16, False, False),
    (1000, 256, 256, False, False),
])
def test_gemm_matches_fp64(torch, M, N, K, ta, tb):
    import gicops_b200.tail as T
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    A = _bf16(torch, (K, M) if ta else (M, K), g)
    B = _bf16(torch, (K, N) if tb else (N, K), g)
    sam, sak = (1, M) if ta else (K, 1)
    sbn, sbk = (1, N) if tb else (K, 1)
    d = T.tail_gemm(A.cuda(), B.cuda(), sam, sak, sbn, sbk, M, N, K).cpu().double()
    Am = (A.T if ta else A).double()
    Bm = (B.T if tb else B).double()
    ref = Am @ Bm.T
    bound = (Am.abs() @ Bm.abs().T) * (K * 2.0 ** -23) + 1e-30
    assert torch.all((d - ref).abs() <= bound), float(((d - ref).abs() / bound).max())


@pytest.fixture(scope="module")
def searched(torch, golden):
    """open_mox golden case searched on the GPU, histograms and results on the device."""
    import gicops_b200 as gx
    c = golden("open_mox")
    dev = gx.DeviceIndex(c["index"], 0)
    q = c["queries"]
    s = gx.Searcher(dev, q.n, len(q.moz))
    r = s.search(q, search_params(c), hist=True)
    d = torch.device("cuda", 0)
    dv = dict(hist=torch.from_numpy(r.hist.view(np.int32).copy()).to(d),
              res=torch.from_numpy(r.result.view(np.uint8).copy()).to(d),
              prec=torch.from_numpy(q.prec.astype(np.float32)).to(d),
              charge=torch.from_numpy(q.charge.astype(np.int32)).to(d))
    return dict(res=r.result, hist=r.hist, q=q, dev=dv)


def _sample_table(res, seed):
    import gicops_b200.tail as T
    rng = np.random.default_rng(seed)
    qs = np.nonzero(res["status"] & 1)[0]
    keeps = np.array([0, 1, 2, 5, 37, 100, 300, 512])
    q = np.repeat(qs, len(keeps))
    k = np.tile(keeps, len(qs))
    return T.samples(q, k, rng.integers(0, 2**63, size=len(q), dtype=np.uint64))


def test_features_and_fits_match_oracle(torch, searched):
    import gicops_b200.tail as T
    import pyoracle
    import tail_mlp as O
    m = T.TailModel(0, max_batch=1024, seed=1)
    smp = _sample_table(searched["res"], seed=5)
    dv = searched["dev"]
    x, sub, cs, hyp = m.features(dv["hist"], dv["res"], dv["prec"], dv["charge"], smp, want_sub=True)
    fit = T.fit_rows(sub, cs, hyp).cpu().numpy()
    xb = x.view(torch.int16).cpu().numpy().view(np.uint16)
    sub, cs, hyp = sub.cpu().numpy(), cs.cpu().numpy(), hyp.cpu().numpy()
    res, hist, q = searched["res"], searched["hist"], searched["q"]
    assert len(smp) > 200
    for i, s in enumerate(smp):
        r = res[s["query"]]
        h_o, cs_o = O.subsample(hist[s["query"]], int(r["maxhyp"]), int(s["keep"]), int(s["seed"]))
        assert np.array_equal(sub[i], h_o) and cs[i] == cs_o and hyp[i] == r["maxhyp"], i
        bits = O.feature_bits(h_o, cs_o, int(r["maxhyp"]), float(q.prec[s["query"]]), int(q.charge[s["query"]]))
        assert np.array_equal(xb[i], bits), i
        # FP64 fit: the device's log10 may differ from the host's in the last place
        f = pyoracle.tailfit(h_o.astype(np.float64), cs_o, int(r["maxhyp"]))
        np.testing.assert_allclose(fit[i], [f["slope"], f["icpt"]], rtol=1e-12, atol=1e-15)
    # keep = 0 reproduces the search's own fit
    full = smp["keep"] == 0
    assert np.array_equal(fit[full, 0], res[smp["query"][full]]["slope"])
    assert np.array_equal(fit[full, 1], res[smp["query"][full]]["icpt"])


@pytest.mark.parametrize("huber", [0.0, 0.5], ids=["squared", "huber"])
def test_gradients_match_oracle(torch, searched, huber):
    import gicops_b200.tail as T
    import tail_mlp as O
    m = T.TailModel(0, max_batch=512, seed=3)
    m.set_loss(huber)
    smp = _sample_table(searched["res"], seed=6)[:448]
    dv = searched["dev"]
    x = m.features(dv["hist"], dv["res"], dv["prec"], dv["charge"], smp)
    rng = np.random.default_rng(7)
    tgt = np.stack([rng.normal(-0.05, 0.02, len(smp)), rng.normal(-3.0, 1.0, len(smp))], 1).astype(np.float32)
    norm = np.array([-0.04, 0.03, -2.5, 1.2], np.float32)
    m.set(norm=norm)
    w = (1.0, 0.5)
    g, loss = m.grad(x, torch.from_numpy(tgt).cuda(), w)
    torch.cuda.synchronize()
    P, _, _ = m.get()
    xv = O.bf16_value(x.view(torch.int16).cpu().numpy().view(np.uint16))
    l_o, g_o = O.loss_and_grads(P.astype(np.float64), xv, tgt, norm.astype(np.float64), w, emulate=True,
                                huber=huber)
    g = g.cpu().numpy().astype(np.float64)
    assert abs(float(loss.item()) - l_o) <= 1e-4 * abs(l_o)
    o = 0
    for name, shp in O.SHAPES:
        n = int(np.prod(shp))
        err = np.linalg.norm(g[o:o + n] - g_o[o:o + n]) / np.linalg.norm(g_o[o:o + n])
        # fp32 accumulation order + rare bf16 rounding flips of hidden values
        assert err < 2e-3, (name, err)
        o += n
    # the bf16 network against the unrounded FP64 one: the rounding's own effect, for scale
    _, g_64 = O.loss_and_grads(P.astype(np.float64), xv, tgt, norm.astype(np.float64), w, emulate=False,
                               huber=huber)
    assert np.linalg.norm(g - g_64) / np.linalg.norm(g_64) < 5e-2


def test_adam_step_matches_oracle(torch, searched):
    import gicops_b200.tail as T
    import tail_mlp as O
    m = T.TailModel(0, max_batch=256, seed=4)
    smp = _sample_table(searched["res"], seed=8)[:256]
    dv = searched["dev"]
    x = m.features(dv["hist"], dv["res"], dv["prec"], dv["charge"], smp)
    tgt = torch.from_numpy(np.tile(np.array([[-0.05, -3.0]], np.float32), (256, 1))).cuda()
    P0, _, _ = m.get()
    opt = T.Adam(lr=1e-3)
    g, _ = m.grad(x, tgt)
    m.train_step(x, tgt, opt)
    g2, _ = m.grad(x, tgt)        # gradient at the new point, for the second step
    m.train_step(x, tgt, opt)
    P2, _, steps = m.get()
    assert steps == 2
    G1, G2 = g.cpu().numpy().astype(np.float64), g2.cpu().numpy().astype(np.float64)
    P1o, mo, vo = O.adam(P0.astype(np.float64), G1, 0.0, 0.0, 1, 1e-3)
    P2o, _, _ = O.adam(P1o, G2, mo, vo, 2, 1e-3)
    np.testing.assert_allclose(P2, P2o, rtol=1e-5, atol=1e-7)


# ---- training and the gain over the plain fit ------------------------------------------------
TRAIN_DB = dict(nproteins=3000, seed=21, nspec=3000, well_populated=2000)
TAIL_HUBER = 0.5   # training loss: Huber's, delta 0.5 in normalised target units


@pytest.fixture(scope="module")
def trained(torch):
    import gicops_b200 as gx
    import gicops_b200.tail as T
    w = TRAIN_DB
    db = gx.synth.make_database(w["nproteins"], seed=w["seed"])
    H = gx.HostIndex.build(db, maxz=2, mods=[("M", 15.9949, 2)], nmods=2)
    q = gx.synth.make_queries(H.entries_by_len(), w["nspec"], seed=w["seed"] + 1, charges=(2, 4),
                              frag_charge2=True, keep_p=(0.2, 0.8), noise_mode="fill", npeaks_range=(30, 150))
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    r = s.search(q, gx.SearchParams(dM=500.0, dF=5, topmatches=5, expect_max=1e300), hist=True)
    d = torch.device("cuda", 0)
    dv = dict(hist=torch.from_numpy(r.hist.view(np.int32).copy()).to(d),
              res=torch.from_numpy(r.result.view(np.uint8).copy()).to(d),
              prec=torch.from_numpy(q.prec.astype(np.float32)).to(d),
              charge=torch.from_numpy(q.charge.astype(np.int32)).to(d))
    res = r.result
    ok = np.nonzero(((res["status"] & 1) != 0) & (res["cpsms"] >= w["well_populated"]) &
                    np.isfinite(res["slope"]) & (res["slope"] < 0))[0]
    rng = np.random.default_rng(0)
    rng.shuffle(ok)
    held, calib, train = ok[:300], ok[300:600], ok[600:]
    m = T.TailModel(0, max_batch=8192, seed=11)
    m.set_loss(TAIL_HUBER)
    smp = T.plan(train, per_query=64, keep_range=(8, 512), seed=1)
    x, t = T.training_set(m, dv, res, smp)
    m.set_norm_from(t.cpu().numpy())
    losses = m.train(x, t, epochs=15, batch=512, opt=T.Adam(lr=1e-3, w_slope=0.2), seed=2, lr_decay=0.85)
    cal = T.evaluate(m, dv, res, T.plan(calib, per_query=8, keep_range=(20, 500), seed=4))
    below = T.choose_sparse_below(cal["err_plain"], cal["err_learned"], cal["cpsms_sub"])
    ev = T.evaluate(m, dv, res, T.plan(held, per_query=8, keep_range=(20, 500), seed=3))
    return dict(model=m, losses=losses, eval=ev, below=below, n_train=len(smp), n_queries=len(ok), dev=dv, res=res,
                queries=q, searcher=s)


def test_training_reduces_loss(trained):
    L = trained["losses"]
    assert np.all(np.isfinite(L)) and L[-1] < 0.95 * L[0], L


def test_learned_tail_beats_plain_fit_on_sparse_held_out(trained):
    """The fallback policy at its calibrated threshold, on held-out queries: well-populated
    queries (not trained on, not calibrated on) subsampled to fewer candidates than the
    threshold, each scored against the plain fit of ALL its candidates at the top score.
    The learned line must beat the plain fit of the subsample on the median, the 90th and
    the 99th percentile of |log10 e| error.  The judge is itself unstable (refitting half of
    a query's own candidates moves it by more than 1 log10 for most queries), which bounds
    how close either line can get."""
    ev, below = trained["eval"], trained["below"]
    assert below >= 50, below
    m = ev["cpsms_sub"] < below
    ep, el = ev["err_plain"][m], ev["err_learned"][m]
    q = lambda e, f: float(np.quantile(e, f))
    print(f"\n[tail] {trained['n_queries']} well-populated queries, {trained['n_train']} training samples; "
          f"threshold {below} candidates; held-out {len(el)} subsamples below it, |log10 e| error vs the full-data "
          f"fit: median plain {q(ep, .5):.2f} learned {q(el, .5):.2f}; p90 plain {q(ep, .9):.2f} learned "
          f"{q(el, .9):.2f}; p99 plain {q(ep, .99):.2f} learned {q(el, .99):.2f}; within 0.1: plain "
          f"{np.mean(ep <= .1):.3f} learned {np.mean(el <= .1):.3f}")
    assert len(el) >= 300
    assert np.all(np.isfinite(el))
    assert q(el, 0.5) < q(ep, 0.5)
    assert q(el, 0.9) < q(ep, 0.9)
    assert q(el, 0.99) < q(ep, 0.99)


def test_fallback_policy_on_search_results(torch, trained):
    import gicops_b200.tail as T
    import gicops_b200._native as N
    m, dv = trained["model"], trained["dev"]
    res0 = trained["res"]
    sparse_below = int(np.quantile(res0["cpsms"][res0["status"] & 1 > 0], 0.3))
    res_dev = dv["res"].clone()
    m.apply(dv["hist"], res_dev, dv["prec"], dv["charge"], sparse_below, 20.0)
    out = res_dev.cpu().numpy().view(N.RESULT_DTYPE)
    x = m.features(dv["hist"], dv["res"], dv["prec"], dv["charge"],
                   T.samples(np.arange(len(res0)), np.zeros(len(res0)), np.zeros(len(res0))))
    pred = m.predict(x).cpu().numpy()
    sparse = ((res0["status"] & 1) != 0) & (res0["cpsms"] < sparse_below)
    usable = sparse & np.isfinite(pred[:, 0]) & (pred[:, 0] < 0)
    assert usable.sum() > 10
    learned = (out["status"] & N.STATUS_LEARNED_TAIL) != 0
    assert np.array_equal(learned, usable)
    # untouched queries are bit-identical
    assert out[~usable].tobytes() == res0[~usable].tobytes()
    # the learned line: mu, beta quantised like the reference's Results.mu/beta
    h = res0["maxhyp"][usable].astype(np.float64)
    slope = pred[usable, 0].astype(np.float64)
    icpt = pred[usable, 1].astype(np.float64) - slope * h
    assert np.array_equal(out["mu"][usable], np.trunc(slope * 1e6).astype(np.int32))
    assert np.array_equal(out["beta"][usable], np.trunc(icpt * 1e6).astype(np.int32))
    e = 10.0 ** (out["mu"][usable] / 1e6 * h + out["beta"][usable] / 1e6) * res0["cpsms"][usable]
    np.testing.assert_allclose(out["e_x"][usable], e, rtol=1e-12)
    assert np.array_equal((out["status"][usable] & 2) != 0, out["e_x"][usable] < 20.0)
    for f in ("slope", "icpt", "e_fp64", "cpsms", "maxhyp"):
        assert np.array_equal(out[f], res0[f]), f


def test_workspace_attached_tail_matches_apply(torch, trained):
    """A model attached to a workspace is applied by gx_search_host after the plain fit,
    with the same outcome as gx_tail_apply on the detached search's results."""
    import gicops_b200 as gx
    import gicops_b200._native as N
    m, dv, res0 = trained["model"], trained["dev"], trained["res"]
    q, s = trained["queries"], trained["searcher"]
    p = gx.SearchParams(dM=500.0, dF=5, topmatches=5, expect_max=20.0)
    below = int(np.quantile(res0["cpsms"][res0["status"] & 1 > 0], 0.3))
    plain = s.search(q, p, hist=True)
    s.set_tail(m, below)
    try:
        att = s.search(q, p).result
    finally:
        s.set_tail(None)
    d = torch.device("cuda", 0)
    res_dev = torch.from_numpy(plain.result.view(np.uint8).copy()).to(d)
    hist = torch.from_numpy(plain.hist.view(np.int32).copy()).to(d)
    m.apply(hist, res_dev, dv["prec"], dv["charge"], below, 20.0)
    ref = res_dev.cpu().numpy().view(N.RESULT_DTYPE)
    assert ((att["status"] & N.STATUS_LEARNED_TAIL) != 0).sum() > 10
    assert att.tobytes() == ref.tobytes()


def test_tensor_core_wait_limit_gives_an_error_status(torch):
    """A wait for the tensor core that runs out (limit 0: every wait gives up at once)
    makes the GEMM record its guard, wait for the product it issued, free its tensor
    memory and return.  gx_tail_check reports it once, and the next inference with the
    normal limit gives the same output as before."""
    import gicops_b200 as gx
    import gicops_b200.tail as T
    lib = gx.lib()
    m = T.TailModel(0, max_batch=512, seed=5)
    x = _bf16(torch, (300, 132), torch.Generator().manual_seed(3)).cuda()
    good = m.predict(x).clone()
    torch.cuda.synchronize()
    assert lib.gx_tail_check(m.handle) == 0
    try:
        assert lib.gx_tail_set_wait_limit(0) == 0
        m.predict(x)
        rc = lib.gx_tail_check(m.handle)
        msg = lib.gx_last_error()
    finally:
        lib.gx_tail_set_wait_limit(1_000_000_000)
    assert rc == -3051 and b"tensor-core wait ran out" in msg
    assert lib.gx_tail_check(m.handle) == 0          # reported once, then cleared
    assert torch.equal(m.predict(x), good)
    torch.cuda.synchronize()
    m.close()
