"""Golden MS2 -> .pbin fixture for the query preprocessing (peak picking and intensity
normalisation).

Writes a seeded synthetic ``prep.ms2`` and converts it with the compiled reference
(``oracle/_ref/ref_harness --ms2-to-pbin``, which calls the reference's own
MSQuery::convertAndprepMS2bin, source/core/msquery.cpp:137-336), keeping its output
as ``prep.ms2.pbin``.  Run from the repository root after ``make -C oracle``:

    python tests/golden/make_ms2_golden.py

The spectra cover what the conversion does on the way: peak counts around the 100-peak
cut (0, 1, 99-101, several hundred), intensity ties, peaks below the 1% cut, intensities
that truncate to 0, a spectrum whose intensities are all 0, peak lines split by a tab
(the reference splits peak lines on spaces only), CRLF line ends, number formats, and
peak lines before the first S line.
"""

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def spectrum_lines(rng, scan, npk, kind):
    out = [f"S\t{scan}\t{scan}\t{rng.uniform(300, 1500):.4f}"]
    z = int(rng.integers(1, 5))
    out.append(f"I\tRTime\t{rng.uniform(0, 120):.4f}")
    out.append(f"Z\t{z}\t{rng.uniform(500, 4000):.5f}")
    mz = np.sort(rng.uniform(100, 2000, npk))
    if kind == "zero":
        it = np.zeros(npk)
    elif kind == "ties":
        it = rng.choice([10.0, 55.5, 200.25, 1e4, 3e4], size=npk)
    elif kind == "tiny":
        it = np.concatenate([rng.uniform(0.001, 0.009, npk // 2), rng.lognormal(6, 2, npk - npk // 2)])
        rng.shuffle(it)
    else:
        it = rng.lognormal(5, 2, npk)
    for k in range(npk):
        fmt = int(rng.integers(0, 4))
        m = f"{mz[k]:.4f}" if fmt == 0 else (f"{mz[k]:.2f}" if fmt == 1 else (f"{mz[k]:g}" if fmt == 2 else f"{mz[k]:.6f}"))
        i = f"{it[k]:.1f}" if fmt != 2 else f"{it[k]:g}"
        sep = "\t" if kind == "tabs" and k % 7 == 3 else " "
        out.append(f"{m}{sep}{i}")
    return out


def make_ms2(path, seed=7, nspec=160):
    rng = np.random.default_rng(seed)
    lines = ["H\tCreationDate\tsynthetic", "H\tExtractor\tnone",
             "412.1234 5000.0", "413.5 12.0"]                       # peaks before the first S line
    counts = [0, 1, 2, 99, 100, 101, 150, 400, 37, 64]
    kinds = ["plain", "ties", "tiny", "zero", "tabs"]
    for s in range(nspec):
        npk = counts[s] if s < len(counts) else int(rng.integers(20, 260))
        kind = kinds[s % len(kinds)]
        if kind == "zero":            # one spectrum with all intensities 0 (index 12)
            kind = "plain"
        if s == 12:
            kind = "zero"
        lines += spectrum_lines(rng, s + 1, npk, kind)
        if s % 11 == 5:
            lines.append("D\tsomething\t1")
    text = ""
    for k, ln in enumerate(lines):
        text += ln + ("\r\n" if k % 13 == 4 else "\n")
    with open(path, "w", newline="") as f:
        f.write(text)


def main():
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        sys.exit("build the reference harness first: make -C oracle")
    ms2 = os.path.join(HERE, "prep.ms2")
    make_ms2(ms2)
    if os.path.exists(ms2 + ".pbin"):
        os.remove(ms2 + ".pbin")
    r = subprocess.run([harness, "--ms2-to-pbin", ms2], capture_output=True, text=True, check=True)
    print(r.stdout.strip())
    print(ms2 + ".pbin", os.path.getsize(ms2 + ".pbin"), "bytes")


if __name__ == "__main__":
    main()
