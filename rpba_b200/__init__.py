"""rpba_b200 -- robust bundle adjustment on one NVIDIA B200.

The global robust bundle adjustment of RPBA (class LSA, rbacore.cpp) as
hand-written sm_100a CUDA behind a C ABI (include/rpba_b200.h).  This
package is the Python side of that ABI (``lib``), the block container
(``block``) and seeded synthetic scenes (``scenes``).
"""
from .block import (Block, RpbaBlockC, RpbaOptionsC, RpbaReportC, make_options, PRECOND_WEIGHTS,
                    SOLVER_PCG, SOLVER_DIRECT, SOLVER_LEARNED, PREC_FP64, PREC_MIXED)
from .lib import (InputBlock, OutputBlock, CalcPLSA, Solver, RpbaError, load, LIB_PATH,
                  EXPORTS, STATUS, float_sequential_sum, train_preconditioner,
                  precond_loss_grad, record_systems, solve_batch, triangulate, triangulate_parts,
                  partition_images, lsa_gcp_step, calc_plsa_parallel, calc_plsa_parallel_ranks, spd_inverse)

__all__ = ["Block", "RpbaBlockC", "RpbaOptionsC", "RpbaReportC", "make_options", "PRECOND_WEIGHTS", "SOLVER_PCG",
           "SOLVER_DIRECT", "SOLVER_LEARNED", "PREC_FP64", "PREC_MIXED", "InputBlock",
           "OutputBlock", "CalcPLSA", "Solver", "RpbaError", "load", "LIB_PATH", "EXPORTS",
           "STATUS", "float_sequential_sum", "train_preconditioner", "precond_loss_grad",
           "record_systems", "solve_batch", "triangulate", "triangulate_parts", "partition_images",
           "lsa_gcp_step", "calc_plsa_parallel", "calc_plsa_parallel_ranks", "spd_inverse"]
