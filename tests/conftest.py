import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = ["closed_small", "closed_1k", "open_mox", "mixed_window"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_case(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    peps = {int(k.split("_")[1]): z[k] for k in z.files if k.startswith("peps_")}
    d = {k: z[k] for k in z.files if not k.startswith("peps_")}
    d["meta"] = meta
    d["peps"] = peps
    return d


def case_queries(c: dict):
    from gicops_b200.synth import QueryBatch
    dM = c["q_dM"] if len(c["q_dM"]) else None
    return QueryBatch(c["q_idx"], c["q_moz"], c["q_intn"], c["q_prec"], c["q_charge"],
                      np.zeros(len(c["q_prec"]), np.float32), dM)


def case_index(c: dict, ions: bool = True):
    """Index of a golden case built by the library's host builder (entries only when
    ions is False)."""
    import gicops_b200 as gx
    from gicops_b200.synth import Database
    m = c["meta"]
    db = Database(peps=c["peps"], nproteins=m["nproteins"])
    mods = [tuple(x) for x in m["mods"]]
    return gx.HostIndex.build(db, maxz=m["maxz"], mods=mods, nmods=m["nmods"], min_mass=m["min_mass"],
                              max_mass=m["max_mass"], ions=ions)


def oracle_params(c: dict):
    import pyoracle
    m = c["meta"]
    return pyoracle.Params(dM=m["dM"], dF=m["dF"], topmatches=m["topmatches"], min_cpsm=m["min_cpsm"],
                           min_shp=m["min_shp"], expect_max=1e300)


def search_params(c: dict, **kw):
    import gicops_b200 as gx
    m = c["meta"]
    return gx.SearchParams(dM=m["dM"], dF=m["dF"], topmatches=m["topmatches"], min_cpsm=m["min_cpsm"],
                           min_shp=m["min_shp"], expect_max=1e300, **kw)


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(name):
        if name not in cache:
            c = load_case(name)
            c["index"] = case_index(c)
            c["queries"] = case_queries(c)
            cache[name] = c
        return cache[name]
    return get


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
