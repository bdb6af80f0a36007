"""Multi-rank layouts of gicops_b200.shard on CPU ranks (gloo, world size 2).

Each rank's search is the oracle's (the layouts are host logic; the per-rank search
is the same call a GPU rank makes through the library).  Checked against one search
of the whole batch over the whole index:

* replicas: spectra split by scan volume, searched per rank, gathered on rank 0 --
  every result record identical;
* index shards: lengths split between the ranks, partial histograms and candidate
  counts summed, top-K cells gathered and merged -- histograms and counts identical,
  the merged top-K hyperscores equal the single index's, and the tail fit of the
  merged histogram gives the single index's e-value.
"""

import os
import socket

import numpy as np
import pytest

WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from conftest import load_case, case_index, case_queries, oracle_params
    c = load_case("open_mox")
    return case_index(c), case_queries(c), oracle_params(c)


def _worker(rank, port, out_dir):
    import torch.distributed as dist
    import pyoracle
    import gicops_b200.shard as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        H, q, p = _case()
        # ---- replicas -----------------------------------------------------------------
        vol = np.diff(q.idx.astype(np.int64))
        mine = S.replica_split(vol, WORLD)[rank]
        res, _ = pyoracle.search(H.lengths, q.subset(mine), p, hist=False, nthreads=1)
        full = S.gather_results(res, mine, q.n, WORLD, rank)
        if rank == 0:
            np.save(os.path.join(out_dir, "replicas.npy"), full)
        # ---- index shards -------------------------------------------------------------
        own = S.length_shards([ln["N"] for ln in H.lengths], WORLD)[rank]
        res, hist = pyoracle.search([H.lengths[i] for i in own], q, p, hist=True, nthreads=1)
        cap = pyoracle.heap_capacity(p.topmatches)
        cells = np.zeros((q.n, cap), dtype=S.CELL_DTYPE)
        for i in range(q.n):
            k = int(res["heap_size"][i])
            for f in ("hyperscore", "psid", "idxoffset", "sharedions", "totalions"):
                cells[i, :k][f] = res["heap"][i, :k][f]
        mh, mc, top = S.merge_shards(hist, res["cpsms"], cells, own, cap, WORLD)
        if rank == 0:
            np.savez(os.path.join(out_dir, "shards.npz"), hist=mh, cpsms=mc, top=top.view(np.uint8))
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def ran(tmp_path_factory):
    import torch.multiprocessing as mp
    out = str(tmp_path_factory.mktemp("shard"))
    mp.spawn(_worker, args=(_free_port(), out), nprocs=WORLD, join=True)
    return out


def test_replicas_gather_equals_single_search(ran):
    import pyoracle
    H, q, p = _case()
    ref, _ = pyoracle.search(H.lengths, q, p, hist=False)
    got = np.load(os.path.join(ran, "replicas.npy"))
    assert got.tobytes() == ref.tobytes()


def test_index_shard_merge_equals_single_index(ran):
    import pyoracle
    import gicops_b200.shard as S
    H, q, p = _case()
    ref, rhist = pyoracle.search(H.lengths, q, p, hist=True)
    z = np.load(os.path.join(ran, "shards.npz"))
    cap = pyoracle.heap_capacity(p.topmatches)
    top = z["top"].view(S.CELL_DTYPE).reshape(q.n, cap)
    assert np.array_equal(z["hist"], rhist) and np.array_equal(z["cpsms"], ref["cpsms"])
    checked = 0
    for i in range(q.n):
        k = int(ref["heap_size"][i])
        want = np.sort(ref["heap"][i, :k]["hyperscore"])[::-1]
        got = top[i]["hyperscore"][: k]
        assert np.array_equal(got, want), i
        if int(ref["cpsms"][i]) < p.min_cpsm:
            continue
        # tail fit of the merged histogram at the merged top score
        t = top[i][0]
        assert t["hyperscore"] == ref["top"][i]["hyperscore"]
        hyp = int(np.floor(np.float64(np.float32(t["hyperscore"]) * np.float32(10.0)) + 0.5))
        f = pyoracle.tailfit(z["hist"][i].astype(np.float64), int(z["cpsms"][i]), hyp)
        assert f["e_x"] == ref["e_x"][i]
        if (ref["heap"][i, :k]["hyperscore"] == t["hyperscore"]).sum() == 1:   # unique top: same PSM
            assert (int(t["psid"]), int(t["idxoffset"])) == (int(ref["top"][i]["psid"]), int(ref["top"][i]["idxoffset"]))
        checked += 1
    assert checked > 50
