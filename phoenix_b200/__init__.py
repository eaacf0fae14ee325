"""phoenix_b200 -- B200 (sm_100a) time stepping of the driven-dissipative
Gross-Pitaevskii equation with reservoir, a drop-in for the RK4 / DP45 hot
path of PHOENIX.  The compute lives in libphx.so (C ABI: include/phx.h);
this package mirrors the reference's solver interface on top of it.
"""
from ._lib import PhxError, header_symbols, load  # noqa: F401
from .batch import BatchSolver  # noqa: F401
from .solver import (Solver, SolverFactory, SystemParameters, Temporal, load_case_fields,  # noqa: F401
                     system_from_case)

__all__ = ["Solver", "BatchSolver", "SolverFactory", "SystemParameters", "Temporal", "PhxError", "load", "header_symbols",
           "system_from_case", "load_case_fields"]
