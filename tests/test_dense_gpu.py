"""The engine's FP64 complex GEMM (the zgemm_ products of the solvers, the
SCF loop and the FP64 projectors) against numpy, through the C ABI on
device matrices; and the device timeout path of the tensor-core kernels.

Shapes cover the three kernels: one column (matrix-vector), 2..8 columns
(narrow SIMT tiles) and more than 8 (DMMA tiles, with K split over blocks
when the output is small), ragged tile edges, leading dimensions above the
row count, op(A) = A and A^H, beta zero and non-zero.  Bar: 1e-12 relative
max-norm (FP64 products; sums of up to 30000 terms).
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from helpers import golden, engine_cell_args, relmax  # noqa: E402
from pspw import PREC_F64, Cell, PspwError  # noqa: E402

TOL = 1e-12
G = golden("si8_8ry")


@pytest.fixture(scope="module")
def cell():
    c = Cell.from_arrays(engine_cell_args(G))
    c.set_veff(G["veff"])
    return c


def _dev(mat, ld):
    """column-major device copy of a host matrix with leading dimension ld"""
    rows, cols = mat.shape
    h = np.zeros((cols, ld), dtype=complex)
    h[:, :rows] = mat.T
    return torch.from_numpy(h).cuda()


def _run(cell, opa, m, n, k, alpha, beta, pad=0, seed=0):
    rng = np.random.default_rng(seed)
    cplx = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)  # noqa: E731
    A = cplx(k, m) if opa == "C" else cplx(m, k)
    B, C = cplx(k, n), cplx(m, n)
    lda, ldb, ldc = max(1, A.shape[0]) + pad, max(1, k) + pad, m + pad
    dA, dB, dC = _dev(A, lda), _dev(B, ldb), _dev(C, ldc)
    torch.cuda.synchronize()
    cell.zgemm_dev(opa, m, n, k, alpha, dA, lda, dB, ldb, beta, dC, ldc)
    torch.cuda.synchronize()
    got = dC.cpu().numpy()[:, :m].T
    opA = A.conj().T if opa == "C" else A
    ref = alpha * (opA @ B) + beta * C
    return got, ref, dC


@pytest.mark.parametrize("opa", ["N", "C"])
@pytest.mark.parametrize("m,n,k", [
    (1, 1, 1), (37, 1, 1000),            # one column: matrix-vector kernels
    (23847, 1, 146), (146, 1, 23847),
    (50, 5, 700), (2000, 8, 33),         # narrow SIMT tiles
    (9, 9, 4), (65, 17, 3), (146, 146, 146), (200, 130, 1),   # DMMA, ragged tiles
    (146, 146, 23847), (256, 144, 5000),  # DMMA, K split over blocks
    (3001, 146, 146), (1000, 70, 256),    # tall outputs
    (64, 64, 0),                          # K = 0: C = beta C
])
def test_zgemm_matches_numpy(cell, opa, m, n, k):
    for alpha, beta in ((1.0, 0.0), (0.5 - 2j, 1.5 + 0.25j)):
        got, ref, _ = _run(cell, opa, m, n, k, alpha, beta, pad=3 if m % 2 else 0)
        assert relmax(got, ref) < TOL, (alpha, beta)


def test_zgemm_split_k_is_bitwise_repeatable(cell):
    a, _, _ = _run(cell, "C", 146, 146, 23847, 1.0, 0.0, seed=5)
    b, _, _ = _run(cell, "C", 146, 146, 23847, 1.0, 0.0, seed=5)
    assert np.array_equal(a, b)


def test_zgemm_rejects_other_ops(cell):
    d = torch.zeros(4, 4, dtype=torch.complex128, device="cuda")
    for op in ("T", "x"):
        with pytest.raises(PspwError) as e:
            cell.zgemm_dev(op, 4, 4, 4, 1.0, d, 4, d, 4, 0.0, d, 4)
        assert e.value.code == 1
    with pytest.raises(PspwError):
        cell.zgemm_dev("N", 4, 4, 4, 1.0, d, 3, d, 4, 0.0, d, 4)  # lda < m


def test_device_wait_times_out_and_cell_stays_usable(cell):
    ref = cell.apply_ham_block(G["psi"])
    cell.check_device_wait(1)  # completed barrier: no error
    t0 = time.perf_counter()
    with pytest.raises(PspwError) as e:
        cell.check_device_wait(0)  # a barrier nothing completes
    assert e.value.code == 6  # PSPW_ERR_TIMEOUT
    assert 0.05 < time.perf_counter() - t0 < 30.0
    cell.check_device_wait(1)  # the error word was cleared
    assert np.array_equal(cell.apply_ham_block(G["psi"]), ref)
    d_in = torch.from_numpy(np.ascontiguousarray(G["psi"].T)).cuda()
    d_out = torch.zeros_like(d_in)
    ngw = int(G["ngw"])
    cell.apply_ham_block_dev(d_in, d_out, ngw, ngw, d_in.shape[0], PREC_F64)
    torch.cuda.synchronize()
    assert relmax(d_out.cpu().numpy().T, G["hpsi"]) < TOL


# ---------------------------------------------------------------- Hermitian eigensolver
def _eig_dev(cell, a, pad=0):
    n = a.shape[0]
    lda = n + pad
    h = np.full((n, lda), np.nan + 0j)
    h[:, :n] = a.T  # column j of A = row j of the torch tensor
    d_a = torch.from_numpy(h).cuda()
    d_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    cell.eig_zheevd_dev(d_a, lda, d_w, n)
    torch.cuda.synchronize()
    return d_w.cpu().numpy(), d_a.cpu().numpy()[:, :n].T.copy()


def _check_eig(cell, a, pad=0, tol=1e-12):
    w, v = _eig_dev(cell, a, pad)
    full = np.triu(a) + np.triu(a, 1).conj().T  # the upper triangle defines A
    ref = np.linalg.eigvalsh(full)
    nrm = max(np.abs(ref).max(), 1e-300)
    n = len(w)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w - ref).max() <= tol * nrm
    assert np.abs(full @ v - v * w).max() <= tol * nrm
    assert np.abs(v.conj().T @ v - np.eye(n)).max() <= tol * max(1, n / 16)
    return w, v


@pytest.mark.parametrize("n", [1, 2, 3, 17, 64, 146, 150, 151, 200])
def test_eig_zheevd_dev_random(cell, n):
    # n <= 150: the engine's kernels; above: cuSOLVER
    rng = np.random.default_rng(n)
    m = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a = m + m.conj().T
    a[np.tril_indices(n, -1)] = np.nan  # only the upper triangle may be read
    _check_eig(cell, a, pad=n % 3)


def _with_spectrum(lam, seed):
    n = len(lam)
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    a = (q * lam) @ q.conj().T
    return 0.5 * (a + a.conj().T)


def test_eig_zheevd_dev_degenerate_and_clustered(cell):
    n = 146
    lam = np.repeat(np.linspace(-0.3, 0.6, 49), 3)[:n]  # triplets, as in a cubic crystal
    _check_eig(cell, _with_spectrum(lam, 1))
    rng = np.random.default_rng(2)
    lam = np.sort(rng.uniform(-0.3, 0.6, n))
    lam[10:15] = lam[10] + np.array([0.0, 1e-12, 1e-9, 2e-6, 3e-4])  # a chain inside 1e-3
    lam[80:84] = lam[80]
    _check_eig(cell, _with_spectrum(np.sort(lam), 3))


def test_eig_zheevd_dev_special_matrices(cell):
    _check_eig(cell, np.diag(np.arange(40, dtype=float) - 7.5).astype(complex))
    w, v = _eig_dev(cell, np.zeros((9, 9), dtype=complex))
    assert np.all(w == 0) and np.abs(v.conj().T @ v - np.eye(9)).max() < 1e-14
    t = np.diag(np.full(50, 2.0)) - np.diag(np.ones(49), 1) - np.diag(np.ones(49), -1)
    _check_eig(cell, t.astype(complex))  # already tridiagonal (reflectors with tau = 0)
    _check_eig(cell, 1e-150 * _with_spectrum(np.linspace(1, 2, 30), 4))  # tiny scale
    _check_eig(cell, 1e150 * _with_spectrum(np.linspace(-1, 2, 30), 6))  # huge scale


def test_eig_zheevd_dev_is_bitwise_repeatable(cell):
    a = _with_spectrum(np.linspace(-1, 1, 146), 5)
    w1, v1 = _eig_dev(cell, a)
    w2, v2 = _eig_dev(cell, a)
    assert np.array_equal(w1, w2) and np.array_equal(v1, v2)


# ---------------------------------------------------------------- span orthonormalisation
@pytest.mark.parametrize("ngw,n,cond", [(3000, 146, 1e2), (2945, 23, 1e4), (5000, 60, 1e8)])
def test_ortho_span_dev(cell, ngw, n, cond):
    """CholeskyQR2 on unit-norm columns (and the Householder QR past the
    conditioning limit): orthonormal columns spanning the input's space."""
    rng = np.random.default_rng(n)
    q, _ = np.linalg.qr(rng.standard_normal((ngw, n)) + 1j * rng.standard_normal((ngw, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    x = (q * np.logspace(0, -np.log10(cond), n)) @ v  # condition number `cond`
    x *= np.logspace(0, 3, n)  # and columns of very different lengths
    d = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    torch.cuda.synchronize()
    cell.ortho_span_dev(d, ngw, n)
    torch.cuda.synchronize()
    y = d.cpu().numpy().T
    assert np.abs(y.conj().T @ y - np.eye(n)).max() < 1e-12
    # span(Y) = span(X): X is reproduced by its projection on Y
    assert np.abs(x - y @ (y.conj().T @ x)).max() < 1e-9 * np.abs(x).max() * cond
