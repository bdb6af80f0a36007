"""PSM rows in the reference's TSV format (source/core/dslim_fileout.cpp:68-146).

The reference writes one file per OpenMP thread, in the order threads finish spectra;
``write_psms`` writes the same columns and number formatting for a batch, in spectrum order.
Numbers follow C++ ``std::to_string``: ``%f`` (six decimals) for float and double values,
decimal integers otherwise.  As in the reference, ``mod_info`` is empty and the peptide is
the unmodified sequence.  A row is written for every spectrum whose PSM the reference
prints (``gx_result.status & 2``).
"""

from __future__ import annotations

import numpy as np

HEADER = ("file\tscan_num\tprec_mass\tcharge\tretention_time\tpeptide\tmatched_ions\ttotal_ions\t"
          "calc_pep_mass\tmass_diff\tmod_info\thyperscore\texpectscore\tnum_hits")


def fmt_f(x) -> str:
    """std::to_string of a float or double: printf("%f") of its double value."""
    return "%f" % float(x)


def psm_rows(index, queries, results: np.ndarray, file_name: str, first_scan: int = 0) -> list:
    """Rows of the reported PSMs of a searched batch.

    index: the HostIndex searched; queries: its QueryBatch (precursor masses, charges,
    retention times); results: gx_result records; first_scan: spectrum number of the
    batch's first spectrum minus one (the reference prints specid + 1)."""
    rows = []
    for s in np.nonzero((results["status"] & 2) != 0)[0]:
        r = results[s]
        t = r["top"]
        ln = index.lengths[int(t["idxoffset"])]
        ent = ln["entries"][int(t["psid"])]
        pep = bytes(ln["seqs"][int(ent["seqid"])]).decode()
        pmass = np.float32(queries.prec[s])
        cmass = np.float32(ln["mass"][int(t["psid"])])
        rows.append("\t".join([
            file_name, str(first_scan + int(s) + 1), fmt_f(pmass), str(int(queries.charge[s])),
            fmt_f(np.float32(queries.rtime[s])), pep, str(int(t["sharedions"])), str(int(t["totalions"])),
            fmt_f(cmass), fmt_f(np.float32(pmass - cmass)), "", fmt_f(np.float32(t["hyperscore"])),
            fmt_f(float(r["e_x"])), str(int(r["cpsms"]))]))
    return rows


def write_psms(path: str, index, queries, results: np.ndarray, file_name: str, first_scan: int = 0,
               header: bool = True) -> int:
    """Append the batch's rows to a TSV file (with the header when asked); returns rows written."""
    rows = psm_rows(index, queries, results, file_name, first_scan)
    with open(path, "a" if not header else "w") as f:
        if header:
            f.write(HEADER + "\n")
        for row in rows:
            f.write(row + "\n")
    return len(rows)
