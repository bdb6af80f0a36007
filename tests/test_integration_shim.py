"""The reference-side shim of INTEGRATION.md (a C++ replacement of hcp::gpu::cuda::s3
on top of this library's C ABI) compiles against the reference's own headers and
include/gicops_b200.h.  Needs the reference source tree and the config header that
oracle/Makefile generates from it; skipped where they are absent."""

import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("GX_REFERENCE", "/root/reference")
GEN = os.path.join(ROOT, "oracle", "_ref", "gen")


def test_shim_compiles_against_reference_headers(tmp_path):
    inc = os.path.join(REF, "source", "core", "include")
    gxx = shutil.which("g++") or "/usr/bin/g++"
    if not (os.path.isdir(inc) and os.path.exists(os.path.join(GEN, "config.hpp")) and os.path.exists(gxx)):
        pytest.skip("reference headers or generated config not available")
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    shim = re.findall(r"```cpp\n(.*?)```", text, re.S)[0]
    src = tmp_path / "shim.cpp"
    src.write_text(shim)
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-fopenmp", "-DUSE_OMP", "-w", "-include", "array",
                        "-I", GEN, "-I", inc, "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
