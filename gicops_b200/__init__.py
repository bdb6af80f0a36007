"""gicops_b200: B200-native peptide-search query path.

Fragment-ion index lookup -> BYC shared-peak scorecard -> hyperscore -> top-K ->
score histogram -> tail-fit e-value, as hand-written sm_100a CUDA behind the C ABI
of include/gicops_b200.h.  A drop-in for the reference's (mhaseeb123/gicops)
``hcp::gpu::cuda::s3::search`` / ``DSLIM_QuerySpectrum`` boundary.
"""

from . import prep, synth, tail
from ._native import (CELL_DTYPE, FLAG_PLAIN, FLAG_WIDE_SCORECARD, HIST_BINS, PEP_ENTRY_DTYPE, RESULT_DTYPE,
                      GxError, lib)
from .index import DeviceIndex, HostIndex
from .search import Searcher, SearchParams, SearchResults, Streamer

__all__ = ["synth", "tail", "lib", "GxError", "HostIndex", "DeviceIndex", "Searcher", "SearchParams", "SearchResults",
           "Streamer", "RESULT_DTYPE", "CELL_DTYPE", "PEP_ENTRY_DTYPE", "HIST_BINS", "FLAG_PLAIN", "FLAG_WIDE_SCORECARD"]
