"""B200 (sm_100a) implementation of the Wilson / domain-wall dynamical-fermion
hot path of the 2-D U(1) lattice study, behind the C ABI in include/dwf_b200.h.

The CUDA library (_lib/libdwfb200.so) is built by ``build.py``; without it every
compute entry point raises.
"""
from . import _capi
from ._capi import (OP_D, OP_DDAG, OP_DDDAG, OP_DDAGD, SOLVER_CG64, SOLVER_MIXED, SOLVER_EO_MIXED, SOLVER_LEARNED,
                    LP_GCR, LP_BICGSTAB, DwfError,
                    LIB_PATH)
from .dwf import DomainWall, CgResult
from .wilson import Wilson

__all__ = ["DomainWall", "Wilson", "CgResult", "DwfError", "OP_D", "OP_DDAG", "OP_DDDAG", "OP_DDAGD",
           "SOLVER_CG64", "SOLVER_MIXED", "SOLVER_EO_MIXED", "SOLVER_LEARNED", "LP_GCR", "LP_BICGSTAB",
           "LIB_PATH"]
