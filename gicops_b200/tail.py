"""Learned tail model: host side of the gx_tail_* entry points (include/gicops_b200.h).

A query's e-value comes from a straight-line fit to the log10 survival of its score
histogram (expeRT, source/core/expeRT.cpp:ModelTailFit in the reference).  With few
candidates that fit is unstable.  The model here predicts the line from the histogram
instead: it is trained on the GPU, by the library's own tensor-core kernels, on
well-populated queries whose candidates are subsampled (the input) against the plain
fit of all their candidates (the target), and it replaces the plain fit only for
queries below a candidate-count threshold (gx_tail_apply).

Device memory is held in torch tensors; every computation is a library call.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from ._native import check, lib

HIST_BINS = N.HIST_BINS


def _torch():
    import torch
    return torch


def _p(t) -> int | None:
    return None if t is None else t.data_ptr()


def _stream() -> int:
    return _torch().cuda.current_stream().cuda_stream


@dataclass
class Adam:
    lr: float = 1e-3
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    w_slope: float = 1.0
    w_lgs: float = 1.0

    def c(self) -> N.TailAdam:
        return N.TailAdam(self.lr, self.beta1, self.beta2, self.eps, self.w_slope, self.w_lgs)


def samples(queries, keeps, seeds) -> np.ndarray:
    """Sample table (gx_tail_sample[]): histogram row, subsample size (0 = all), seed."""
    s = np.zeros(len(queries), dtype=N.TAIL_SAMPLE_DTYPE)
    s["query"], s["keep"], s["seed"] = queries, keeps, seeds
    return s


def fit_rows(hist, cpsms, hyp):
    """Plain FP64 expeRT fit of device histogram rows: tensor [n, 2] (slope, intercept)."""
    torch = _torch()
    n = hist.shape[0]
    out = torch.empty((n, 2), dtype=torch.float64, device=hist.device)
    check(lib().gx_tail_fit_rows(_p(hist), _p(cpsms), _p(hyp), n, _p(out), _stream()))
    return out


def line_targets(slope, icpt, hyp) -> np.ndarray:
    """Training targets [n, 2] float32: (slope, log10 survival fraction at the top bin)."""
    slope = np.asarray(slope, dtype=np.float64)
    return np.stack([slope, slope * np.asarray(hyp, dtype=np.float64) + np.asarray(icpt, dtype=np.float64)],
                    axis=1).astype(np.float32)


class TailModel:
    """gx_tail_model: fp32 master weights + Adam state + scratch for max_batch rows."""

    def __init__(self, device: int = 0, max_batch: int = 8192, seed: int = 0):
        h = C.c_void_p()
        check(lib().gx_tail_model_create(device, max_batch, seed, C.byref(h)))
        self.handle, self.device, self.max_batch = h, device, max_batch

    def close(self) -> None:
        if self.handle:
            lib().gx_tail_model_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters ------------------------------------------------------------------
    def get(self):
        P = np.empty(N.TAIL_NPARAM, dtype=np.float32)
        norm = np.empty(4, dtype=np.float32)
        steps = C.c_uint64()
        check(lib().gx_tail_model_get(self.handle, P.ctypes.data, norm.ctypes.data, C.byref(steps)))
        return P, norm, int(steps.value)

    def set(self, params=None, norm=None) -> None:
        P = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        nm = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        if P is not None and P.size != N.TAIL_NPARAM:
            raise ValueError(f"expected {N.TAIL_NPARAM} parameters, got {P.size}")
        check(lib().gx_tail_model_set(self.handle, None if P is None else P.ctypes.data,
                                      None if nm is None else nm.ctypes.data))

    def save(self, path: str) -> None:
        P, norm, steps = self.get()
        np.savez(path, params=P, norm=norm, steps=steps)

    def load(self, path: str) -> None:
        d = np.load(path)
        self.set(d["params"], d["norm"])

    def set_loss(self, huber: float = 0.0) -> None:
        """Training loss: the squared error (0) or Huber's loss with this delta, in
        normalised target units (gx_tail_set_loss)."""
        check(lib().gx_tail_set_loss(self.handle, float(huber)))

    def set_norm_from(self, targets) -> np.ndarray:
        """Target normalisation (mean, scale per output) from a training set's targets."""
        t = np.asarray(targets, dtype=np.float64)
        norm = np.array([t[:, 0].mean(), max(t[:, 0].std(), 1e-6), t[:, 1].mean(), max(t[:, 1].std(), 1e-6)],
                        dtype=np.float32)
        self.set(norm=norm)
        return norm

    # ---- features ----------------------------------------------------------------------
    def features(self, hist, res, prec, charge, smp: np.ndarray, want_sub: bool = False):
        """Feature rows (torch bfloat16 [n, 132]) for a sample table; with want_sub also the
        subsampled histograms, their candidate counts and top bins."""
        torch = _torch()
        dev = hist.device
        smp = np.ascontiguousarray(smp, dtype=N.TAIL_SAMPLE_DTYPE)
        n = len(smp)
        x = torch.empty((n, N.TAIL_IN), dtype=torch.bfloat16, device=dev)
        sub = cs = hyp = None
        if want_sub:
            sub = torch.empty((n, HIST_BINS), dtype=torch.int32, device=dev)
            cs = torch.empty(n, dtype=torch.int32, device=dev)
            hyp = torch.empty(n, dtype=torch.int32, device=dev)
        nq = hist.shape[0]
        for i0 in range(0, n, self.max_batch):
            i1 = min(n, i0 + self.max_batch)
            part = smp[i0:i1]
            check(lib().gx_tail_features(
                self.handle, _p(hist), _p(res), _p(prec), _p(charge), nq, part.ctypes.data, i1 - i0, _p(x[i0:i1]),
                None if sub is None else _p(sub[i0:i1]), None if cs is None else _p(cs[i0:i1]),
                None if hyp is None else _p(hyp[i0:i1]), _stream()))
        check(lib().gx_tail_check(self.handle))
        return (x, sub, cs, hyp) if want_sub else x

    # ---- training ----------------------------------------------------------------------
    def grad(self, x, target, weights=(1.0, 1.0)):
        torch = _torch()
        g = torch.empty(N.TAIL_NPARAM, dtype=torch.float32, device=x.device)
        loss = torch.empty(1, dtype=torch.float32, device=x.device)
        w = (C.c_float * 2)(*weights)
        check(lib().gx_tail_grad(self.handle, _p(x), _p(target), x.shape[0], w, _p(g), _p(loss), _stream()))
        return g, loss

    def train_step(self, x, target, opt: Adam, loss_out=None) -> None:
        o = opt.c()
        check(lib().gx_tail_train_step(self.handle, _p(x), _p(target), x.shape[0], C.byref(o), _p(loss_out),
                                       _stream()))

    def train(self, x, target, epochs: int = 10, batch: int = 512, opt: Adam | None = None, seed: int = 0,
              lr_decay: float = 1.0) -> list:
        """Mini-batch Adam over (x, target) (device tensors); returns the mean loss per epoch."""
        torch = _torch()
        opt = opt or Adam()
        n = x.shape[0]
        g = torch.Generator(device="cpu").manual_seed(seed)
        loss = torch.zeros(1, dtype=torch.float32, device=x.device)
        hist = []
        lr = opt.lr
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g).to(x.device)
            xs, ts = x[perm].contiguous(), target[perm].contiguous()
            tot = torch.zeros(1, dtype=torch.float32, device=x.device)
            nb = 0
            for i0 in range(0, n - batch + 1, batch):
                self.train_step(xs[i0:i0 + batch], ts[i0:i0 + batch],
                                Adam(lr, opt.beta1, opt.beta2, opt.eps, opt.w_slope, opt.w_lgs), loss)
                tot += loss
                nb += 1
            hist.append(float(tot.item()) / max(nb, 1))
            lr *= lr_decay
        return hist

    # ---- inference ---------------------------------------------------------------------
    def predict(self, x):
        """[n, 2] float32: (slope, log10 survival fraction at the top bin)."""
        torch = _torch()
        n = x.shape[0]
        out = torch.empty((n, 2), dtype=torch.float32, device=x.device)
        for i0 in range(0, n, self.max_batch):
            i1 = min(n, i0 + self.max_batch)
            check(lib().gx_tail_predict(self.handle, _p(x[i0:i1]), i1 - i0, _p(out[i0:i1]), _stream()))
        return out

    def apply(self, hist, res, prec, charge, sparse_below: int, expect_max: float) -> None:
        """Fallback policy over device search results (in place)."""
        check(lib().gx_tail_apply(self.handle, _p(hist), _p(res), _p(prec), _p(charge), hist.shape[0],
                                  sparse_below, expect_max, _stream()))


def tail_gemm(a, b, sam, sak, sbn, sbk, M, N_, K):
    """D = A * B^T on the model's tensor-core GEMM (bf16 operands, fp32 result)."""
    torch = _torch()
    d = torch.empty((M, N_), dtype=torch.float32, device=a.device)
    check(lib().gx_tail_gemm(_p(a), sam, sak, _p(b), sbn, sbk, M, N_, K, _p(d), N_, _stream()))
    return d


# ---- training sets and evaluation ----------------------------------------------------------
def plan(queries, per_query: int, keep_range=(8, N.TAIL_MAX_KEEP), seed: int = 0) -> np.ndarray:
    """Sample table: each query `per_query` times, subsample sizes log-uniform in keep_range
    (inclusive), distinct seeds."""
    rng = np.random.default_rng(seed)
    q = np.repeat(np.asarray(queries, dtype=np.uint32), per_query)
    lo, hi = keep_range
    keeps = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=len(q))).astype(np.uint32).clip(lo, hi)
    seeds = rng.integers(0, 2**63, size=len(q), dtype=np.uint64)
    return samples(q, keeps, seeds)


def training_set(model: TailModel, dev: dict, res_host: np.ndarray, smp: np.ndarray):
    """(features, targets) on the device for a sample table over searched queries.

    dev holds device tensors hist [nq, 802], res (gx_result bytes), prec, charge;
    res_host the same results on the host.  Targets are the plain FP64 fit of ALL the
    query's candidates: (slope, slope * maxhyp + icpt)."""
    torch = _torch()
    x = model.features(dev["hist"], dev["res"], dev["prec"], dev["charge"], smp)
    r = res_host[smp["query"]]
    t = torch.from_numpy(line_targets(r["slope"], r["icpt"], r["maxhyp"])).to(x.device)
    return x, t


def choose_sparse_below(err_plain, err_learned, cands, thresholds=(25, 50, 75, 100, 150, 200, 300, 500),
                        min_rows: int = 100) -> int:
    """The fallback policy's candidate threshold, from calibration samples (held-out
    well-populated queries subsampled to sparsity, errors against their full-data fit): the
    largest threshold T for which the samples with fewer than T candidates have a smaller
    median AND a smaller 90th-percentile error with the learned line than with the plain
    fit.  0 when no threshold qualifies: the model is then never used."""
    ep, el, cs = (np.asarray(a) for a in (err_plain, err_learned, cands))
    best = 0
    for t in sorted(thresholds):
        m = cs < t
        if m.sum() < min_rows:
            continue
        if np.median(el[m]) < np.median(ep[m]) and np.quantile(el[m], 0.9) < np.quantile(ep[m], 0.9):
            best = t
    return int(best)


def evaluate(model: TailModel, dev: dict, res_host: np.ndarray, smp: np.ndarray) -> dict:
    """Errors (log10 e-value at the top score) of the learned line and of the plain fit on
    the subsampled candidates, both against the plain fit of all the candidates."""
    x, sub, cs, hyp = model.features(dev["hist"], dev["res"], dev["prec"], dev["charge"], smp, want_sub=True)
    plain = fit_rows(sub, cs, hyp).cpu().numpy()
    pred = model.predict(x).cpu().numpy().astype(np.float64)
    r = res_host[smp["query"]]
    h = r["maxhyp"].astype(np.float64)
    truth = r["slope"] * h + r["icpt"]
    e_plain = np.abs(plain[:, 0] * h + plain[:, 1] - truth)
    e_plain[~np.isfinite(e_plain)] = np.inf
    e_learn = np.abs(pred[:, 1] - truth)
    e_learn[~np.isfinite(e_learn)] = np.inf
    return dict(err_plain=e_plain, err_learned=e_learn, keep=smp["keep"].copy(), cpsms_sub=cs.cpu().numpy())
