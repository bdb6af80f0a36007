"""Index-sharded search merged on the GPU (gx_merge_shards_device), against one search
of the whole index.

The ranks are emulated on the one GPU as the merge kernel sees them after the
collectives: each length shard is searched for real (its own device index), the
partial histograms and counts are summed, the cells, statuses and length maps stacked,
and one kernel launch merges all ranks' data.  The records must equal the whole-index
search: candidate counts, status bits, top hyperscore and its histogram bin, tail-fit
region and e-values bit for bit, the top-K hyperscores in order, and the top PSM where
its hyperscore is unique.  The NCCL wiring of merge_shards_device runs in a one-rank
process group in a subprocess."""

import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import has_gpu, search_params

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def gx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200
    return gicops_b200


def _search(gx, H, q, p):
    dev = gx.DeviceIndex(H, 0)
    return gx.Searcher(dev, q.n, len(q.moz)).search(q, p, heap=True, hist=True)


def _check_against_full(full, rec, top, cap):
    import gicops_b200._native as N
    r = rec.view(N.RESULT_DTYPE).reshape(-1)
    t = top.view(N.CELL_DTYPE).reshape(len(r), cap)
    f = full.result
    assert np.array_equal(r["cpsms"], f["cpsms"])
    assert np.array_equal(r["status"] & 15, f["status"] & 15)
    m = (f["status"] & 1) != 0
    for k in ("maxhyp", "mu", "beta", "stt1", "end1"):
        assert np.array_equal(r[k][m], f[k][m]), k
    for k in ("e_x", "e_fp64", "slope", "icpt"):
        assert np.array_equal(r[k][m].view(np.uint64), f[k][m].view(np.uint64)), k
    assert np.array_equal(r["top"]["hyperscore"][m].view(np.uint32), f["top"]["hyperscore"][m].view(np.uint32))
    unique = 0
    for i in range(len(r)):
        hs = np.sort(full.heap[i]["hyperscore"][full.heap[i]["hyperscore"] > 0])[::-1]
        assert np.array_equal(t[i]["hyperscore"][: len(hs)], hs), i
        assert np.all(t[i]["hyperscore"][len(hs):] == 0)
        if m[i] and (full.heap[i]["hyperscore"] == f["top"]["hyperscore"][i]).sum() == 1:
            assert (int(r["top"]["psid"][i]), int(r["top"]["idxoffset"][i])) == \
                   (int(f["top"]["psid"][i]), int(f["top"]["idxoffset"][i]))
            unique += 1
    return unique


@pytest.mark.parametrize("case,world", [("open_mox", 3), ("closed_1k", 2)])
def test_device_merge_of_emulated_ranks_equals_whole_index(gx, golden, case, world):
    import torch
    from gicops_b200 import shard
    c = golden(case)
    H, q = c["index"], c["queries"]
    p = search_params(c)
    full = _search(gx, H, q, p)
    own = shard.length_shards([x["N"] for x in H.lengths], world)
    parts = [_search(gx, gx.HostIndex([H.lengths[i] for i in o], H.maxz, H.scale, H.max_mass), q, p) for o in own]
    assert np.array_equal(sum(x.hist.astype(np.int64) for x in parts), full.hist)
    d = torch.device("cuda", 0)
    cells = torch.from_numpy(np.stack([x.heap.view(np.uint8).reshape(q.n, -1) for x in parts])).to(d)
    status = torch.from_numpy(np.stack([x.result["status"] for x in parts]).astype(np.int32)).to(d)
    luts = torch.from_numpy(np.stack([shard.length_lut(o) for o in own]).view(np.int16)).to(d)
    hist = torch.from_numpy(sum(x.hist.astype(np.int64) for x in parts).astype(np.int32)).to(d)
    cpsms = torch.from_numpy(sum(x.result["cpsms"].astype(np.int64) for x in parts).astype(np.int32)).to(d)
    rec, top = shard.merge_gathered_device(p, cells, status, luts, hist, cpsms)
    torch.cuda.synchronize()
    unique = _check_against_full(full, rec.cpu().numpy(), top.cpu().numpy(), p.heap_cap)
    assert unique > 10


_NCCL_RANK = r"""
import os, sys, numpy as np, torch, torch.distributed as dist
sys.path.insert(0, {root!r}); sys.path.insert(0, os.path.join({root!r}, "tests")); sys.path.insert(0, os.path.join({root!r}, "oracle"))
from conftest import load_case, case_index, case_queries, search_params
import gicops_b200 as gx
from gicops_b200 import shard
torch.cuda.set_device(0)
dist.init_process_group("nccl", init_method="tcp://127.0.0.1:{port}", rank=0, world_size=1,
                        device_id=torch.device("cuda", 0))
c = load_case("open_mox")
H, q = case_index(c), case_queries(c)
p = search_params(c)
dev = gx.DeviceIndex(H, 0)
r = gx.Searcher(dev, q.n, len(q.moz)).search(q, p, heap=True, hist=True)
d = torch.device("cuda", 0)
rec, top = shard.merge_shards_device(p, torch.from_numpy(r.hist.astype(np.int32)).to(d),
                                     torch.from_numpy(r.result["cpsms"].copy()).to(d),
                                     torch.from_numpy(r.heap.view(np.uint8).reshape(q.n, -1).copy()).to(d),
                                     torch.from_numpy(r.result["status"].copy()).to(d),
                                     list(range(H.nlen)), 1)
torch.cuda.synchronize()
np.save({out!r}, rec.cpu().numpy())
dist.destroy_process_group()
"""


def test_nccl_wiring_single_rank(gx, golden, tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "rec.npy")
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    subprocess.run([sys.executable, "-c", _NCCL_RANK.format(root=ROOT, port=port, out=out)], check=True, env=env,
                   timeout=300)
    import gicops_b200._native as N
    c = golden("open_mox")
    full = _search(gx, c["index"], c["queries"], search_params(c))
    r = np.load(out).view(N.RESULT_DTYPE).reshape(-1)
    f = full.result
    assert np.array_equal(r["cpsms"], f["cpsms"]) and np.array_equal(r["status"] & 15, f["status"] & 15)
    m = (f["status"] & 1) != 0
    assert np.array_equal(r["e_x"][m].view(np.uint64), f["e_x"][m].view(np.uint64))
