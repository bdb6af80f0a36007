"""CPU oracle of the learned tail model (TEST INFRASTRUCTURE ONLY: imported by tests/ as
the checker of the CUDA kernels in gicops_b200/csrc/gx_tail.cu, never by the product).

The model has no counterpart in the reference; the plain fit it stands in for is
source/core/expeRT.cpp:ModelTailFit (restated in restate.c:rs_tailfit).  This file
restates, in FP64 numpy:

* the feature rows of k_features, including the subsampling (Floyd's sampling without
  replacement, Bentley & Floyd 1987, driven by SplitMix64, Steele, Lea & Flood 2014)
  bit for bit;
* the network 132 -> 256 -> 256 -> 2 (GELU, erf form), its loss and backward pass,
  optionally rounding to bf16 at the same points as the GPU (operands of every tensor-core
  product: features, weights, hidden activations, output gradient, hidden gradients);
* one Adam step.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf

WIN, NIN, NHID, NOUT = 128, 132, 256, 2
HIST = 802
SHAPES = [("W1", (NHID, NIN)), ("b1", (NHID,)), ("W2", (NHID, NHID)), ("b2", (NHID,)), ("W3", (NOUT, NHID)),
          ("b3", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
M64 = (1 << 64) - 1


# ---- bf16 -----------------------------------------------------------------------------
def bf16_bits(x) -> np.ndarray:
    """Round to float32, then to bf16 (round to nearest even): uint16 bit patterns."""
    f = np.asarray(x, dtype=np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    return ((u + 0x7FFF + lsb) >> 16).astype(np.uint16)


def bf16_value(bits) -> np.ndarray:
    return (np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def bf16(x) -> np.ndarray:
    return bf16_value(bf16_bits(x))


# ---- parameters -----------------------------------------------------------------------
def unpack(P) -> dict:
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(P[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    return out


def pack(d) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


# ---- subsampling and features (k_features) ----------------------------------------------
def splitmix64(state: int) -> tuple[int, int]:
    state = (state + 0x9E3779B97F4A7C15) & M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return state, z ^ (z >> 31)


def subsample(hist, hyp: int, keep: int, seed: int) -> tuple[np.ndarray, int]:
    """(subsampled histogram, candidate count).  The top-scoring candidate (bin hyp) is
    always kept; keep - 1 others are drawn without replacement from the rest."""
    h = np.asarray(hist, dtype=np.int64)
    tot = int(h.sum())
    if keep == 0 or keep >= tot:
        return h.copy(), tot
    top = 1 if h[hyp] > 0 else 0
    others, k = tot - top, keep - top
    o = h.copy()
    o[hyp] -= top
    cum = np.cumsum(o)
    st, chosen = seed & M64, set()
    for j in range(others - k, others):
        st, r = splitmix64(st)
        t = (r * (j + 1)) >> 64
        chosen.add(j if t in chosen else t)
    ranks = np.fromiter(chosen, dtype=np.int64, count=len(chosen))
    sub = np.bincount(np.searchsorted(cum, ranks, side="right"), minlength=HIST).astype(np.int64)
    sub[hyp] += top
    return sub, keep


def feature_bits(sub, cs: int, hyp: int, prec: float, charge: int) -> np.ndarray:
    """The 132 bf16 feature bits of one row: log10(1 + count) of the 128 bins from the
    first non-empty one, log10(candidates), precursor mass / 1000, charge, distance of
    the top bin from the window start / 100."""
    sub = np.asarray(sub)
    nz = np.nonzero(sub)[0]
    b0 = int(nz[0]) if len(nz) else 0
    b = b0 + np.arange(WIN)
    c = np.where(b < HIST, sub[np.clip(b, 0, HIST - 1)], 0).astype(np.float64)
    x = np.empty(NIN, dtype=np.float64)
    x[:WIN] = np.log10(1.0 + c)
    x[WIN] = np.log10(float(cs if cs > 0 else 1))
    x[WIN + 1] = float(np.float32(prec)) / 1000.0
    x[WIN + 2] = float(charge)
    x[WIN + 3] = (hyp - b0) / 100.0
    return bf16_bits(x)


# ---- network ---------------------------------------------------------------------------
def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(P, X, emulate: bool = True) -> dict:
    """X: [n, 132] feature values.  emulate=True rounds the tensor-core operands to bf16."""
    p = unpack(P)
    r = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    Xb = r(X)
    W1, W2, W3 = r(p["W1"]), r(p["W2"]), r(p["W3"])
    Z1 = Xb @ W1.T + p["b1"]
    A1 = r(gelu(Z1))
    Z2 = A1 @ W2.T + p["b2"]
    A2 = r(gelu(Z2))
    Y = A2 @ W3.T + p["b3"]
    return dict(Xb=Xb, W1=W1, W2=W2, W3=W3, Z1=Z1, A1=A1, Z2=Z2, A2=A2, Y=Y)


def loss_and_grads(P, X, T, norm, w=(1.0, 1.0), emulate: bool = True, huber: float = 0.0) -> tuple[float, np.ndarray]:
    """Mean weighted loss on normalised targets and its gradient (flat, NPARAM): the squared
    error (huber 0) or Huber's loss with delta huber (d^2 / 2 delta inside, |d| - delta / 2
    outside), as k_loss computes them."""
    r = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    f = forward(P, X, emulate)
    n = X.shape[0]
    T = np.asarray(T, dtype=np.float64)
    tn = np.stack([(T[:, 0] - norm[0]) / norm[1], (T[:, 1] - norm[2]) / norm[3]], axis=1)
    wv = np.asarray(w, dtype=np.float64)
    d = f["Y"] - tn
    if huber > 0:
        ad = np.abs(d)
        inside = ad < huber
        loss = float((wv * np.where(inside, 0.5 * d * d / huber, ad - 0.5 * huber)).sum() / n)
        dY = r(wv * np.where(inside, d / huber, np.sign(d)) / n)
    else:
        loss = float((wv * d * d).sum() / n)
        dY = r(2.0 * wv * d / n)
    g = {}
    g["W3"] = dY.T @ f["A2"]
    g["b3"] = dY.sum(axis=0)
    dZ2 = r((dY @ f["W3"]) * gelu_grad(f["Z2"]))
    g["W2"] = dZ2.T @ f["A1"]
    g["b2"] = dZ2.sum(axis=0)
    dZ1 = r((dZ2 @ f["W2"]) * gelu_grad(f["Z1"]))
    g["W1"] = dZ1.T @ f["Xb"]
    g["b1"] = dZ1.sum(axis=0)
    return loss, pack(g)


def predict(P, X, norm, emulate: bool = True) -> np.ndarray:
    Y = forward(P, X, emulate)["Y"]
    return np.stack([Y[:, 0] * norm[1] + norm[0], Y[:, 1] * norm[3] + norm[2]], axis=1)


def adam(P, G, m, v, step: int, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * G
    v = b2 * v + (1 - b2) * G * G
    bc1, bc2 = 1 - b1 ** step, 1 - b2 ** step
    return P - lr * (m / bc1) / (np.sqrt(v / bc2) + eps), m, v
