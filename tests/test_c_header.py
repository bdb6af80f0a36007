"""The public header as a C caller sees it: include/gicops_b200.h compiles as C99 with
warnings as errors, a C program links against the library, and the host-only entry
points (heap capacity, hyperscore table, host index build, MS2 reader, error path)
answer as they do through ctypes.  No device call is made."""

import os
import shutil
import subprocess

import numpy as np
import pytest

import gicops_b200._native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "gicops_b200.h"

int main(int argc, char **argv)
{
    double lg[81];
    gx_lgfact(lg);
    printf("cap %d %d %d\n", gx_heap_capacity(5), gx_heap_capacity(10), gx_heap_capacity(31));
    printf("lg80 %.17g\n", lg[80]);
    /* host index build of three peptides of length 7 */
    const char seqs[] = "PEPTIDEKLMNPQRACDEFGHK";
    gx_build_params bp;
    memset(&bp, 0, sizeof(bp));
    bp.maxz = 1; bp.scale = 100; bp.min_mass = 500; bp.max_mass = 5000; bp.threads = 1;
    gx_host_length *h = NULL;
    gx_status st = gx_build_length(seqs, 3, 7, &bp, &h);
    gx_length_desc d;
    if (st == GX_SUCCESS) st = gx_host_length_desc(h, &d);
    if (st != GX_SUCCESS) { printf("error %d %s\n", st, gx_last_error()); return 1; }
    unsigned long long sum = 0;
    for (unsigned i = 0; i < d.npep * d.speclen; i++) sum += d.iA[i] * (unsigned long long)(i + 1);
    printf("index %u %u %u %llu\n", d.npep, d.speclen, d.bA[500000], sum);
    gx_host_length_free(h);
    /* error path: a bad residue */
    st = gx_build_length("PEPT1DE", 1, 7, &bp, &h);
    printf("bad %d\n", st);
    /* MS2 reader */
    gx_ms2_file *f = NULL;
    st = gx_ms2_read(argv[1], 100, &f);
    gx_ms2_raw r;
    if (st == GX_SUCCESS) st = gx_ms2_desc(f, &r);
    if (st != GX_SUCCESS) { printf("error %d %s\n", st, gx_last_error()); return 1; }
    printf("ms2 %u %u %d %d\n", r.nspec, r.nvalues, r.mz[0], r.intn[r.nvalues - 1]);
    gx_ms2_free(f);
    (void)argc;
    return 0;
}
"""


def test_header_compiles_as_c_and_links(tmp_path):
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    if not os.path.exists(cc):
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "abi"
    libdir = os.path.dirname(N.LIB_PATH)
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", libdir, "-lgicops_b200", "-Wl,-rpath," + libdir], check=True)
    ms2 = tmp_path / "t.ms2"
    ms2.write_text("S\t1\t1\t500\nZ\t2\t1001.5\n100.25 7\n200.5 9.5\n")
    out = subprocess.run([str(exe), str(ms2)], capture_output=True, text=True, check=True).stdout.split("\n")
    import pyoracle
    assert out[0] == f"cap {pyoracle.heap_capacity(5)} {pyoracle.heap_capacity(10)} {pyoracle.heap_capacity(31)}"
    lg = np.zeros(81)
    N.lib().gx_lgfact(lg.ctypes.data)
    assert float(out[1].split()[1]) == lg[80]
    import gicops_b200 as gx
    from gicops_b200.synth import Database
    db = Database(peps={7: np.frombuffer(b"PEPTIDEKLMNPQRACDEFGHK"[:21], np.uint8).reshape(3, 7).copy()}, nproteins=1)
    H = gx.HostIndex.build(db, maxz=1, minlen=7, maxlen=7)
    x = H.lengths[0]
    s = int((x["iA"].astype(np.uint64) * np.arange(1, len(x["iA"]) + 1, dtype=np.uint64)).sum())
    assert out[2] == f"index {x['N']} {x['speclen']} {int(x['bA'][500000])} {s}"
    assert out[3] == "bad -3002"
    assert out[4] == "ms2 1 2 10025 950"
