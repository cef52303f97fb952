"""Batched H*psi over uneven cells (pspw_batch_*): every cell's result in
the one-launch batch equals the same cell applied alone with the tuned
schedule (bitwise), repeated launches give the same bits, and the FP32
batch agrees with each cell's FP64 H*psi (2e-5 relative max-norm, the FP32
parity bar); the FP64 batch agrees with the oracle (1e-12)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pspw_oracle as O  # noqa: E402
from helpers import oracle_cell, relmax  # noqa: E402
from pspw import PREC_F32, PREC_F64, Cell  # noqa: E402
from pspw.batch import Batch, ortho_cell  # noqa: E402


@pytest.fixture(scope="module")
def cells():
    rng = np.random.default_rng(31)
    out = []
    for _ in range(6):
        d = ortho_cell(rng, nat_range=(2, 6), lat_range=(8.0, 10.5), ecut_range=(10.0, 13.0),
                       band_range=(8, 40))
        c = Cell.from_arrays(d)
        c.set_veff(d["veff"])
        out.append((d, c))
    return out


def _alone(cell, psi, prec):
    ngw, nb = psi.shape
    dt = torch.complex64 if prec == PREC_F32 else torch.complex128
    d_in = torch.from_numpy(np.ascontiguousarray(psi.T)).to(dt).cuda()
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    cell.apply_ham_block_dev(d_in, d_out, ngw, ngw, nb, prec)
    torch.cuda.synchronize()
    return d_out.cpu().numpy().T


@pytest.mark.parametrize("prec", [PREC_F32, PREC_F64])
def test_batch_equals_cells_alone(cells, prec):
    b = Batch([c for _, c in cells], [d["nbands"] for d, _ in cells], prec)
    for i, (d, _) in enumerate(cells):
        b.upload(i, d["psi"])
    b.tune(reps=2)
    b.apply()
    assert b.kernels() >= 4 * len(cells)  # every cell's passes are in the graph
    first = [b.download(i) for i in range(len(cells))]
    b.apply()
    second = [b.download(i) for i in range(len(cells))]
    for i, (d, c) in enumerate(cells):
        s = b.schedule(i)
        assert s["ms"] > 0
        assert np.array_equal(first[i], second[i])
        alone = _alone(c, np.asarray(d["psi"], dtype=b.dtype), prec)
        assert np.array_equal(first[i], alone)
        if prec == PREC_F32:
            ref = c.apply_ham_block(np.asarray(d["psi"], dtype=np.complex64).astype(complex))
            assert relmax(first[i], ref) < 2e-5
        elif i < 2:
            oc = oracle_cell(d)
            ref = O.apply_ham_block(oc, d["psi"], d["veff"])
            assert relmax(first[i], ref) < 1e-12
    b.close()


def test_batch_cells_have_uneven_shapes(cells):
    shapes = {(d["nr"], d["ngw"], d["nbands"]) for d, _ in cells}
    assert len(shapes) == len(cells)
    assert any(d["nr"][0] != d["nr"][1] for d, _ in cells)  # orthorhombic grids
