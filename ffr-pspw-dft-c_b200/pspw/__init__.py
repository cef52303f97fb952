"""Host-side Python interface of the B200 Hamiltonian engine (ctypes over the
C ABI of libpspw_gpu.so; see include/pspw_gpu.h)."""
from ._lib import (MIX_ANDERSON, MIX_BROYDEN, MIX_KERKER, MIX_PULAY, MIX_SIMPLE, NL_AUTO, NL_SIMT,
                   NL_TENSOR_CORE, OVERLAP_AUTO, OVERLAP_OFF, OVERLAP_ON, PREC_F32, PREC_F64,
                   PspwError, check, lib)
from .cell import Cell, basis_gamma, random_col

__all__ = ["Cell", "basis_gamma", "random_col", "PREC_F32", "PREC_F64", "NL_AUTO", "NL_SIMT",
           "NL_TENSOR_CORE", "OVERLAP_AUTO", "OVERLAP_ON", "OVERLAP_OFF", "MIX_SIMPLE", "MIX_KERKER", "MIX_ANDERSON", "MIX_PULAY",
           "MIX_BROYDEN",
           "PspwError", "check", "lib"]
