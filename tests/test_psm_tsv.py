"""PSM TSV rows (gicops_b200.psm_tsv): the number formatting against C++ std::to_string
(compiled here), and the rows of a golden case against the PSMs the compiled reference
printed (captured by oracle/ref_harness)."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import load_case, case_index, case_queries, oracle_params


def test_number_format_matches_std_to_string(tmp_path):
    gxx = shutil.which("g++") or "/usr/bin/g++"
    if not os.path.exists(gxx):
        pytest.skip("no C++ compiler")
    from gicops_b200.psm_tsv import fmt_f
    rng = np.random.default_rng(4)
    fl = np.concatenate([rng.uniform(0, 5000, 200), rng.lognormal(0, 8, 200), [0.0, 1e-7, 0.5, 1234.5678]])
    fl = fl.astype(np.float32)
    db = np.concatenate([10.0 ** rng.uniform(-12, 6, 200), [0.0, 5e-7, 4.9999995e-7, 19.999999]])
    src = tmp_path / "f.cpp"
    src.write_text("#include <cstdio>\n#include <string>\n#include <iostream>\nint main(){float f;double d;"
                   "while(std::cin>>f)std::cout<<std::to_string(f)<<'\\n';std::cin.clear();"
                   "return 0;}\n")
    exe = tmp_path / "f"
    subprocess.run([gxx, "-O1", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], input="\n".join(repr(float(x)) for x in fl), capture_output=True, text=True,
                         check=True).stdout.split()
    assert out == [fmt_f(x) for x in fl]
    srcd = tmp_path / "d.cpp"
    srcd.write_text("#include <string>\n#include <iostream>\nint main(){double d;"
                    "while(std::cin>>d)std::cout<<std::to_string(d)<<'\\n';return 0;}\n")
    exed = tmp_path / "d"
    subprocess.run([gxx, "-O1", str(srcd), "-o", str(exed)], check=True)
    out = subprocess.run([str(exed)], input="\n".join(repr(float(x)) for x in db), capture_output=True, text=True,
                         check=True).stdout.split()
    assert out == [fmt_f(x) for x in db]


def test_rows_match_reference_psms():
    import pyoracle
    from gicops_b200.psm_tsv import HEADER, psm_rows
    c = load_case("closed_small")
    H, q = case_index(c), case_queries(c)
    p = oracle_params(c)
    p.expect_max = 20.0
    res, _ = pyoracle.search(H.lengths, q, p)
    rows = psm_rows(H, q, res, "q.ms2")
    assert len(HEADER.split("\t")) == 14 and all(len(r.split("\t")) == 14 for r in rows)
    rep = np.nonzero(c["cap_reported"])[0]
    assert len(rows) == len(rep) > 10
    for row, s in zip(rows, rep):
        f = row.split("\t")
        assert f[1] == str(s + 1)
        lnx = H.lengths[int(c["cap_idxoffset"][s])]
        ent = lnx["entries"][int(c["cap_psid"][s])]
        assert f[5] == bytes(lnx["seqs"][int(ent["seqid"])]).decode()
        assert f[6] == str(int(c["cap_sharedions"][s])) and f[7] == str(int(c["cap_totalions"][s]))
        assert f[11] == "%f" % float(np.float32(c["cap_hyperscore"][s]))
        assert f[12] == "%f" % float(c["cap_e_x"][s])
        assert f[13] == str(int(c["cap_npsms"][s]))
