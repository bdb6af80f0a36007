"""Multi-GPU layouts of the query path (one process per GPU, torch.distributed).

Two ways to spread a search over ranks:

* **Replicas** (spectra are independent): every rank holds the whole index and
  searches its share of the spectra.  ``replica_split`` deals the spectra out
  round-robin in descending order of their scan volume, so every rank gets a similar
  amount of work; ``gather_results`` brings the per-rank results back to rank 0 in
  the original spectrum order.  No data-path collective.

* **Index shards** (the reference's distributed design, source/core/lbe_internal.cpp:
  75-103 and source/core/dslim_score.cpp:199-388, where MPI ranks own peptide subsets
  and exchange partial results through files): here each rank owns a subset of the
  peptide lengths (``length_shards``, balanced by entry count) and searches every
  spectrum against it.  One exchange per batch: the per-spectrum score histograms and
  candidate counts are summed (all_reduce), the per-rank top-K cells are gathered
  (all_gather) and merged by (hyperscore descending, global length index, entry);
  the tail fit then runs on the merged histogram, which equals the single-index one.

The collectives go through torch.distributed (NCCL between GPUs; gloo for the CPU
tests of this logic).  ``merge_shards`` merges on the host; ``merge_shards_device``
keeps everything on the GPU: the collectives run on CUDA tensors (NCCL) and the merge,
the mapping to global length indices and the tail fit of the summed histograms run in
one kernel (``gx_merge_shards_device``), which ``merge_gathered_device`` calls on
already gathered data.
"""

from __future__ import annotations

import numpy as np

from . import _native as N
from ._native import CELL_DTYPE, HIST_BINS


def replica_split(volumes, world: int) -> list:
    """Spectrum indices of each rank: descending volume, dealt round-robin."""
    order = np.argsort(-np.asarray(volumes, dtype=np.float64), kind="stable")
    return [np.sort(order[r::world]) for r in range(world)]


def gather_results(local: np.ndarray, mine: np.ndarray, n: int, world: int, rank: int, group=None):
    """Rank 0 receives every rank's records (structured array, one per spectrum of
    ``mine``) placed at their original positions in an array of n; other ranks get None."""
    import torch
    import torch.distributed as dist
    raw = torch.from_numpy(np.ascontiguousarray(local).view(np.uint8).copy())
    idx = torch.from_numpy(np.asarray(mine, dtype=np.int64))
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([len(mine)], dtype=torch.int64), group=group)
    cap = int(max(s.item() for s in sizes))
    rec = local.dtype.itemsize
    pad_raw = torch.zeros(cap * rec, dtype=torch.uint8)
    pad_raw[: raw.numel()] = raw
    pad_idx = torch.full((cap,), -1, dtype=torch.int64)
    pad_idx[: idx.numel()] = idx
    all_raw = [torch.zeros_like(pad_raw) for _ in range(world)]
    all_idx = [torch.zeros_like(pad_idx) for _ in range(world)]
    dist.all_gather(all_raw, pad_raw, group=group)
    dist.all_gather(all_idx, pad_idx, group=group)
    if rank != 0:
        return None
    out = np.zeros(n, dtype=local.dtype)
    for r in range(world):
        k = int(sizes[r].item())
        recs = all_raw[r].numpy()[: k * rec].view(local.dtype)
        out[all_idx[r].numpy()[:k]] = recs
    return out


def length_shards(entries_per_length, world: int) -> list:
    """Length indices owned by each rank: greedy by entry count, largest first."""
    sizes = np.asarray(entries_per_length, dtype=np.int64)
    load = np.zeros(world, dtype=np.int64)
    own = [[] for _ in range(world)]
    for i in np.argsort(-sizes, kind="stable"):
        r = int(np.argmin(load))
        own[r].append(int(i))
        load[r] += sizes[i]
    return [sorted(o) for o in own]


def merge_topk(cells: np.ndarray, cap: int) -> np.ndarray:
    """Top-cap cells of one spectrum out of all ranks' cells (empty cells have h <= 0):
    hyperscore descending, then global length index, then entry, ascending."""
    c = cells[cells["hyperscore"] > 0]
    order = np.lexsort((c["psid"], c["idxoffset"], -c["hyperscore"].astype(np.float64)))
    out = np.zeros(cap, dtype=CELL_DTYPE)
    k = min(cap, len(order))
    out[:k] = c[order[:k]]
    return out


def merge_shards(hist: np.ndarray, cpsms: np.ndarray, cells: np.ndarray, own_lengths, cap: int, world: int,
                 group=None):
    """Exchange of the index-sharded search (every rank calls it, in the same order).

    hist [n, 802] and cpsms [n] are this rank's partial histograms and candidate counts;
    cells [n, k] its top-k cells with idxoffset local to ``own_lengths``.  Returns the
    merged (hist, cpsms, top cells [n, cap] with global length indices), identical on
    every rank."""
    import torch
    import torch.distributed as dist
    n = hist.shape[0]
    h = torch.from_numpy(np.ascontiguousarray(hist, dtype=np.int64))
    c = torch.from_numpy(np.ascontiguousarray(cpsms, dtype=np.int64))
    dist.all_reduce(h, group=group)
    dist.all_reduce(c, group=group)
    g = np.array(cells, dtype=CELL_DTYPE, copy=True)
    lut = np.asarray(own_lengths, dtype=np.uint16)
    live = g["hyperscore"] > 0
    g["idxoffset"][live] = lut[g["idxoffset"][live]]
    raw = torch.from_numpy(g.view(np.uint8).reshape(n, -1).copy())
    parts = [torch.zeros_like(raw) for _ in range(world)]
    dist.all_gather(parts, raw, group=group)
    allc = np.concatenate([p.numpy().reshape(-1).view(CELL_DTYPE).reshape(n, -1) for p in parts], axis=1)
    top = np.stack([merge_topk(allc[i], cap) for i in range(n)]) if n else np.zeros((0, cap), CELL_DTYPE)
    return h.numpy().astype(np.uint32).reshape(n, HIST_BINS), c.numpy().astype(np.int32), top


def length_lut(own_lengths) -> np.ndarray:
    """[GX_MAX_LENGTHS] global length index of each rank-local one (unused slots 0)."""
    lut = np.zeros(N.MAX_LENGTHS, np.uint16)
    lut[: len(own_lengths)] = np.asarray(own_lengths, dtype=np.uint16)
    return lut


def merge_gathered_device(params, cells, status, luts, hist, cpsms, stream=None):
    """Merge of gathered shard results on the GPU (CUDA tensors, no collective):
    cells uint8 [world, n, k*16] (gx_cell records, rank-local idxoffset), status int32
    [world, n], luts uint16 [world, GX_MAX_LENGTHS], hist int32 [n, 802] and cpsms int32
    [n] summed over ranks.  Returns (result records uint8 [n, record], top cells uint8
    [n, cap*16]) on the same device."""
    import ctypes as C
    import torch
    world, n = int(status.shape[0]), int(status.shape[1])
    k = int(cells.shape[2]) // CELL_DTYPE.itemsize if n else 1
    cap = int(N.lib().gx_heap_capacity(params.topmatches))
    dev = cells.device
    out = torch.empty((n, N.RESULT_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    top = torch.empty((n, cap * CELL_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    cp = params.c() if hasattr(params, "c") else params
    for t in (cells, status, luts, hist, cpsms):
        assert t.is_contiguous() and t.device == dev
    N.check(N.lib().gx_merge_shards_device(n, world, k, cells.data_ptr(), status.data_ptr(), luts.data_ptr(),
                                           hist.data_ptr(), cpsms.data_ptr(), C.byref(cp), top.data_ptr(),
                                           out.data_ptr(), C.c_void_p(st)))
    return out, top


def merge_shards_device(params, hist, cpsms, cells, status, own_lengths, world: int, group=None):
    """Exchange + merge of the index-sharded search, on the GPU (every rank calls it, in
    the same order): hist int32 [n, 802] and cpsms int32 [n] are this rank's partial
    histograms and counts, cells uint8 [n, k*16] its top-k gx_cell records (rank-local
    idxoffset), status int32 [n] its result statuses; all CUDA tensors.  One all_reduce of
    histograms and counts, all_gathers of cells, statuses and length maps (NCCL), then
    the device merge.  Returns (result records, top cells), identical on every rank."""
    import torch
    import torch.distributed as dist
    dev = hist.device
    h = hist.contiguous().clone()
    c = cpsms.contiguous().clone()
    dist.all_reduce(h, group=group)
    dist.all_reduce(c, group=group)
    lut = torch.from_numpy(length_lut(own_lengths).view(np.uint8)).to(dev)   # NCCL has no 16-bit ints: bytes
    parts_c = [torch.empty_like(cells) for _ in range(world)]
    parts_s = [torch.empty_like(status) for _ in range(world)]
    parts_l = [torch.empty_like(lut) for _ in range(world)]
    dist.all_gather(parts_c, cells.contiguous(), group=group)
    dist.all_gather(parts_s, status.contiguous(), group=group)
    dist.all_gather(parts_l, lut, group=group)
    luts = torch.stack(parts_l).view(torch.int16)
    return merge_gathered_device(params, torch.stack(parts_c), torch.stack(parts_s), luts, h, c)
