"""gems_b200 -- B200-native (sm_100a) Felsenstein likelihood kernels behind IQ-TREE's
PhyloTree API.

The compute path is the CUDA library ``libgems_b200.so`` (C-ABI in ``include/gems_b200.h``);
this package only binds it.  There is no CPU fallback: when the library or a CUDA device is
missing, the calls raise.
"""
from .api import (GemsError, PhyloTree, Session, STATUS, op_array, branch_struct,
                  measure_peaks, check_barrier_timeout, compress_alignment, Ingest, full_traversal,
                  traverse_batch, branch_lnl_batch, set_models_from_rates,
                  optimize_all_branches_batch, compute_likelihood_batch, evaluate_rates_batch,
                  GEMS_CHILD_PARTIAL, GEMS_CHILD_TIP)

__all__ = ["GemsError", "PhyloTree", "Session", "STATUS", "op_array", "branch_struct",
           "measure_peaks", "check_barrier_timeout", "compress_alignment", "Ingest", "full_traversal",
           "traverse_batch", "branch_lnl_batch", "set_models_from_rates",
           "optimize_all_branches_batch", "compute_likelihood_batch", "evaluate_rates_batch",
           "GEMS_CHILD_PARTIAL", "GEMS_CHILD_TIP"]
