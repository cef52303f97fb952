"""Parity at the benchmarked configuration itself.

bench.py times the degree-10 Chebyshev filter (chebyfilt.cpp:6-74) of the
whole 144-band Si64 block (64 atoms, a = 20.52 bohr, 64^3 grid, NGW 23847)
on the window [0.5, 16] Ha, as a device block with ld = NGW over the whole
sphere, which is the filter's stick-order mode (the block is permuted once
into the order of the stick lists and back).  These tests run exactly that
call and compare it with

- the engine's FP64 filter of the same block (whole block), and
- the oracle's chebyfilt (a numpy restatement pinned to the reference's own
  output) on a 16-band slice: bands are independent under the filter, so
  columns of the block's result equal the filter of those columns alone.

Bars: FP64 engine vs oracle 1e-12 relative max-norm (the FP64 parity bar of
ApplyHam_block.cpp); FP32 filter vs either FP64 result 1e-4 relative
max-norm (FP32 H*psi is within 2e-5 of FP64 per application; ten
applications through the three-term recurrence stay below 1e-4).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pspw_oracle as O  # noqa: E402
from helpers import oracle_cell, relmax  # noqa: E402
from pspw import PREC_F32, PREC_F64, workloads  # noqa: E402

DEGREE, LB, UB = 10, 0.5, 16.0  # bench.py's filter
TOL64 = 1e-12
TOL32 = 1e-4
SLICE = slice(40, 56)  # 16 bands from the middle of the block


@pytest.fixture(scope="module")
def si64():
    w = workloads.workload("si64")
    cell = workloads.make_cell(w)
    # the FP32 input, widened: both precisions filter the same numbers
    psi = np.asfortranarray(w["psi"].astype(np.complex64).astype(complex))
    return w, cell, psi


def _filter_dev(cell, psi, prec):
    """bench.py's call: chebyfilt_dev on a device block, ld = ngw."""
    ngw, nb = psi.shape
    dt = torch.complex64 if prec == PREC_F32 else torch.complex128
    d = torch.from_numpy(np.ascontiguousarray(psi.T)).to(dt).cuda()
    torch.cuda.synchronize()
    cell.chebyfilt_dev(d, ngw, ngw, nb, DEGREE, LB, UB, prec)
    torch.cuda.synchronize()
    return d.cpu().numpy().T.astype(complex)


@pytest.fixture(scope="module")
def filtered(si64):
    w, cell, psi = si64
    assert psi.shape == (23847, 144)
    f64 = _filter_dev(cell, psi, PREC_F64)
    f32 = _filter_dev(cell, psi, PREC_F32)
    ref = O.chebyfilt(oracle_cell(w), np.asfortranarray(psi[:, SLICE]), DEGREE, LB, UB,
                      w["veff"])
    return f64, f32, ref


def test_bench_filter_fp64_slice_matches_oracle(filtered):
    f64, _, ref = filtered
    assert relmax(f64[:, SLICE], ref) < TOL64


def test_bench_filter_fp32_slice_matches_oracle(filtered):
    _, f32, ref = filtered
    assert relmax(f32[:, SLICE], ref) < TOL32


def test_bench_filter_fp32_whole_block_matches_fp64(filtered):
    f64, f32, _ = filtered
    assert np.isfinite(f32).all()
    assert relmax(f32, f64) < TOL32
    # per band as well: no band may hide under the block's largest column
    per_band = np.abs(f32 - f64).max(axis=0) / np.abs(f64).max(axis=0)
    assert per_band.max() < 10 * TOL32


def test_bench_filter_fp32_repeat_is_bitwise(si64, filtered):
    _, cell, psi = si64
    _, f32, _ = filtered
    assert np.array_equal(_filter_dev(cell, psi, PREC_F32), f32)


def test_si64_fp64_hpsi_32_bands_matches_oracle(si64):
    # block H*psi in FP64 on 32 bands of the benchmarked cell, device call
    w, cell, psi = si64
    blk = np.asfortranarray(w["psi"][:, 56:88])
    ngw, nb = blk.shape
    d_in = torch.from_numpy(np.ascontiguousarray(blk.T)).cuda()
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    cell.apply_ham_block_dev(d_in, d_out, ngw, ngw, nb, PREC_F64)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().T
    ref = O.apply_ham_block(oracle_cell(w), blk, w["veff"])
    assert relmax(out, ref) < TOL64
