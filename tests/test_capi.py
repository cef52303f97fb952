"""The C ABI library loads (no GPU needed) and exports every function that
include/pspw_gpu.h declares; the drop-in library exports the reference's
C++ signatures under their g++ mangled names."""
import ctypes
import os
import re
import subprocess

import pytest

from pspw import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pspw_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pspw_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_functions():
    names = declared_functions()
    assert "pspw_apply_ham_block" in names and "pspw_cell_create" in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_error_strings_without_gpu():
    L = _lib.lib()
    assert L.pspw_error_string(2) == b"inconsistent sizes"
    assert L.pspw_version() >= 100


# g++ mangled names of the reference functions the drop-in replaces
# (signatures from common_pspw.h:176-222)
DROPIN_SYMBOLS = [
    "_Z14ApplyHam_blockPCdS0_iiPdii",       # ApplyHam_block        common_pspw.h:177
    "_Z8ApplyHamPCdS0_iiPdi",               # ApplyHam              common_pspw.h:176
    "_Z9chebyfiltiPCdiddPdi",               # chebyfilt             common_pspw.h:187
    "_Z19ApplyHam_block_cudaPCdS0_iii",     # ApplyHam_block_cuda   common_pspw.h:254
    "_Z25SetupArrays_ApplyHam_cudaPjPdPCdS0_",  # SetupArrays_...   common_pspw.h:255
    "_Z21CopyRho_ApplyHam_cudaPd",          # CopyRho_ApplyHam_cuda common_pspw.h:257
    "_Z9SetupCUDAv", "_Z12ShutdownCUDAv",   # common_pspw.h:252-253
    "_Z12davidson_cpuiPdPCdiiS_iS_",        # davidson_cpu          common_pspw.h:198
    "_Z10lobpcg_cpuiPdPCdiiS_iS_",          # lobpcg_cpu            common_pspw.h:193
    "_Z8ortho_qrPCdii",                     # ortho_qr              common_pspw.h:222
    "_Z10eig_zheevdPCdiPdi",                # eig_zheevd            common_pspw.h:217
    "_Z14eig_zhegv_evalPCdiS0_iPdS0_ii",    # eig_zhegv_eval        common_pspw.h:220
    "_Z9eig_zhegvPCdiS0_iS0_ii",            # eig_zhegv             common_pspw.h:218
    "_Z7GenPreciPdid",                      # GenPrec               common_pspw.h:182
    "_Z10EvalRhoPsiiPdPCdii",               # EvalRhoPsi (5 args)   common_pspw.h:180
    "_Z10EvalRhoPsiiPdPCdi",                # EvalRhoPsi (4 args)   common_pspw.h:179
    "_Z7lanczosiPCdiPdiS0_S1_i",            # lanczos               common_pspw.h:185
    "_Z17Diagon_lobpcg_cpuiPdPCdiS_id",     # Diagon_lobpcg_cpu     common_pspw.h:195
    "_Z19Diagon_davidson_cpuiPdPCdiS_id",   # Diagon_davidson_cpu   common_pspw.h:200
    "_Z10symmetrizePCdiii",                 # symmetrize (lobpcg_cpu.cpp:15)
    "_Z7EvalENLv",                          # EvalENL               common_pspw.h:181
]


@pytest.mark.skipif(not os.path.exists(_lib.DROPIN_PATH), reason="drop-in library not built")
def test_dropin_exports_reference_mangled_names():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.DROPIN_PATH], capture_output=True,
                         text=True).stdout
    for s in DROPIN_SYMBOLS:
        assert re.search(r"\bT " + re.escape(s) + r"$", out, re.M), s
