"""GPU parity of block H*psi and the Chebyshev filter against the oracle.

Bar: FP64 path within 1e-12 relative max-norm of the reference's
ApplyHam_block (golden fixture made by the reference) and of the oracle; the
FP32 path within 2e-5 relative max-norm (single-precision FFT and projector
sums with FP32 accumulation over NGW <= 24k terms).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pspw_oracle as O  # noqa: E402
from helpers import engine_cell_args, golden, oracle_cell, relmax  # noqa: E402
from pspw import (NL_SIMT, NL_TENSOR_CORE, OVERLAP_AUTO, OVERLAP_OFF, OVERLAP_ON,  # noqa: E402
                  PREC_F32, PREC_F64, Cell, PspwError, basis_gamma, synth)
from pspw import workloads  # noqa: E402

TOL64 = 1e-12
TOL32 = 2e-5

G = golden("si8_8ry")


def engine_cell(d, veff):
    c = Cell.from_arrays(engine_cell_args(d))
    c.set_veff(veff)
    return c


@pytest.fixture(scope="module")
def gcell():
    return engine_cell(G, G["veff"])


@pytest.fixture(scope="module")
def cfg0():
    w = workloads.workload("si8")
    cell = workloads.make_cell(w)
    return w, cell


def test_fp64_matches_reference_golden(gcell):
    out = gcell.apply_ham_block(G["psi"])
    assert relmax(out, G["hpsi"]) < TOL64


def test_single_band_matches_reference_apply_ham(gcell):
    out = gcell.apply_ham_block(G["psi"][:, :1])
    assert relmax(out[:, 0], G["h1"]) < TOL64


def test_fp64_config0_matches_oracle(cfg0):
    w, cell = cfg0
    out = cell.apply_ham_block(w["psi"])
    ref = O.apply_ham_block(oracle_cell(w), w["psi"], w["veff"])
    assert relmax(out, ref) < TOL64


def test_fp32_device_config0(cfg0):
    w, cell = cfg0
    psi = w["psi"]
    ngw, nb = psi.shape
    d_in = torch.from_numpy(np.ascontiguousarray(psi.T)).to(torch.complex64).cuda()
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    cell.apply_ham_block_dev(d_in, d_out, ngw, ngw, nb, PREC_F32)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().T
    ref = O.apply_ham_block(oracle_cell(w), psi.astype(np.complex64).astype(complex), w["veff"])
    assert relmax(out, ref) < TOL32


def test_fp64_device_leading_dimension(cfg0):
    w, cell = cfg0
    psi = w["psi"][:, :5]
    ngw = psi.shape[0]
    ld = ngw + 7
    host = np.zeros((5, ld), dtype=complex)
    host[:, :ngw] = psi.T
    d_in = torch.from_numpy(host).cuda()
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    cell.apply_ham_block_dev(d_in, d_out, ld, ngw, 5, PREC_F64)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy()[:, :ngw].T
    ref = O.apply_ham_block(oracle_cell(w), psi, w["veff"])
    assert relmax(out, ref) < TOL64


def test_band_batches_give_identical_bits(cfg0):
    w, cell = cfg0
    outs = []
    for nbatch in (0, 1, 3, 16):
        cell.set_band_batch(nbatch)
        outs.append(cell.apply_ham_block(w["psi"]))
    cell.set_band_batch(0)
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


def test_repeat_is_deterministic(cfg0):
    w, cell = cfg0
    a = cell.apply_ham_block(w["psi"])
    b = cell.apply_ham_block(w["psi"])
    assert np.array_equal(a, b)


def test_fewer_plane_waves_than_the_cell(cfg0):
    # NGW_ik below the cell's sphere: only the first ngw G's exist
    w, cell = cfg0
    ngw = 2000
    psi = np.asfortranarray(w["psi"][:ngw, :4])
    out = cell.apply_ham_block(psi)
    oc = oracle_cell(w)
    ref = O.apply_ham_block(oc, psi, w["veff"])
    assert relmax(out, ref) < TOL64


@pytest.mark.parametrize("nr", [(22, 21, 26), (25, 27, 30), (20, 24, 18)])
def test_non_power_of_two_grids(nr):
    # radices 7, 11, 13 take the generic butterfly; 25/27/30 mix 3 and 5
    lat, pos = synth.si_diamond(1)
    b = basis_gamma(lat, 8.0, nr, [8], [pos])
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=[4])
    veff = synth.local_potential(b["nr"], lat, pos)
    psi = synth.wavefunctions(b, lat, 3, 5)
    cell = Cell.from_arrays(b)
    cell.set_veff(veff)
    out = cell.apply_ham_block(psi)
    ref = O.apply_ham_block(oracle_cell(b), psi, veff)
    assert relmax(out, ref) < TOL64


@pytest.mark.parametrize("n", [25, 27, 45])
def test_density_on_odd_square_grids(n):
    """EvalRhoPsi (EvalRhoPsi.cpp:83-157) on square grids of odd length,
    where the density kernel's FP64 accumulator plane follows a table of n
    ints in shared memory and must start on a 16-byte boundary; against the
    oracle (1e-12 relative max-norm)."""
    lat, pos = synth.si_diamond(1)
    b = basis_gamma(lat, 8.0, (n, n, n), [8], [pos])
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=[4])
    ngw, ngwx = b["ngw"], b["ngwx"]
    psi = synth.wavefunctions(b, lat, 4, 9)
    flat = np.concatenate([psi.reshape(-1, order="F"), np.zeros(ngwx, complex)])
    focc = np.full(4, 2.0)
    omega = float(b["omega"])
    cell = Cell.from_arrays(b)
    rho, ekin = cell.eval_rho_psi(np.zeros(n ** 3), flat, ngw, ngw, 4, focc, 1.0, omega)
    ref, ek_ref, _ = O.eval_rho_psi(oracle_cell(b), flat, ngw, ngw, 4, focc, 1.0, omega, ngwx)
    assert relmax(rho, ref) < TOL64
    assert abs(ekin - ek_ref) < TOL64 * abs(ek_ref)


@pytest.mark.parametrize("lm_end", [[1], [0], [3]])
def test_projector_counts(lm_end):
    d = dict(G)
    args = engine_cell_args(d)
    args["lm_end"] = lm_end
    cell = Cell.from_arrays(args)
    cell.set_veff(G["veff"])
    out = cell.apply_ham_block(G["psi"][:, :3])
    oc = oracle_cell(d)
    oc["lm_end"] = lm_end
    ref = O.apply_ham_block(oc, G["psi"][:, :3], G["veff"])
    assert relmax(out, ref) < TOL64


def test_two_species():
    # species-major projector order with different lm_end per species
    lat, pos = synth.si_diamond(1)
    na = [5, 3]
    tau = [pos[:5], pos[5:]]
    b = basis_gamma(lat, 8.0, None, na, tau)
    pkg_a, wnl = synth.kb_form_factors(b, lat, nsp=2, rc=[1.0, 0.8])
    wnl[1] = [0.7, -0.3, -0.3, -0.3]
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=[4, 1])
    veff = synth.local_potential(b["nr"], lat, pos)
    psi = synth.wavefunctions(b, lat, 4, 9)
    cell = Cell.from_arrays(b)
    cell.set_veff(veff)
    out = cell.apply_ham_block(psi)
    oc = oracle_cell(b)
    oc.update(na=na, lm_end=[4, 1])
    ref = O.apply_ham_block(oc, psi, veff)
    assert relmax(out, ref) < TOL64


def test_chebyfilt_fp64_matches_reference_golden(gcell):
    out = gcell.chebyfilt(G["psi"], int(G["cheb_degree"]), float(G["cheb_lb"]),
                          float(G["cheb_ub"]), PREC_F64)
    assert relmax(out, G["cheb"]) < TOL64


@pytest.mark.parametrize("degree", [1, 2, 3, 10])
def test_chebyfilt_fp64_degrees(cfg0, degree):
    w, cell = cfg0
    X = w["psi"][:, :6]
    out = cell.chebyfilt(X, degree, 1.5, 5.0, PREC_F64)
    ref = O.chebyfilt(oracle_cell(w), X, degree, 1.5, 5.0, w["veff"])
    assert relmax(out, ref) < TOL64


def test_chebyfilt_fp32(cfg0):
    w, cell = cfg0
    X = w["psi"]
    out = cell.chebyfilt(X, 10, 1.5, 5.0, PREC_F32)
    ref = O.chebyfilt(oracle_cell(w), X, 10, 1.5, 5.0, w["veff"])
    assert relmax(out, ref) < 1e-4


@pytest.mark.parametrize("prec,tol", [(PREC_F64, TOL64), (PREC_F32, 1e-4)])
def test_chebyfilt_host_block_in_two_chunks(cfg0, prec, tol):
    # 37 bands (>= 32): the host-facing filter moves the block in two band
    # chunks (19 + 18) on a copy stream while the cell stream filters the
    # other chunk; every band still gets the whole filter
    w, cell = cfg0
    rng = np.random.default_rng(11)
    psi = w["psi"]
    X = np.asfortranarray(psi[:, rng.integers(0, psi.shape[1], 37)]
                          * (1.0 + 0.1 * rng.standard_normal(37)))
    out = cell.chebyfilt(X, 4, 1.5, 5.0, prec)
    ref = O.chebyfilt(oracle_cell(w), X, 4, 1.5, 5.0, w["veff"])
    assert relmax(out, ref) < tol


def test_chebyfilt_fewer_plane_waves_than_the_cell(cfg0):
    # NGW_ik below the cell's sphere: the filter stays in the caller's G order
    w, cell = cfg0
    ngw = 2000
    X = np.asfortranarray(w["psi"][:ngw, :5])
    out = cell.chebyfilt(X, 4, 1.5, 5.0, PREC_F64)
    oc = oracle_cell(w)
    ref = O.chebyfilt(oc, X, 4, 1.5, 5.0, w["veff"])
    assert relmax(out, ref) < TOL64


def test_chebyfilt_device_leading_dimension_stick_order(cfg0):
    # the whole sphere on the register-FFT path: the filter permutes the
    # block into the stick order and back, here with ld > ngw
    w, cell = cfg0
    psi = w["psi"][:, :5]
    ngw = psi.shape[0]
    ld = ngw + 9
    host = np.full((5, ld), 7.0 + 3.0j)
    host[:, :ngw] = psi.T
    d_x = torch.from_numpy(host).cuda()
    torch.cuda.synchronize()
    cell.chebyfilt_dev(d_x, ld, ngw, 5, 6, 1.5, 5.0, PREC_F64)
    torch.cuda.synchronize()
    got = d_x.cpu().numpy()
    ref = O.chebyfilt(oracle_cell(w), psi, 6, 1.5, 5.0, w["veff"])
    assert relmax(got[:, :ngw].T, ref) < TOL64
    assert np.all(got[:, ngw:] == 7.0 + 3.0j)  # padding rows untouched


def test_errors_are_reported(gcell):
    with pytest.raises(PspwError) as e:
        gcell.set_veff(np.zeros(17))
    assert e.value.code == 2  # nnr != NNR (ApplyHam_block.cpp:18-21)
    args = engine_cell_args(G)
    args["lm_end"] = [5]
    args["pkg_a"] = np.zeros((5,) + G["pkg_a"].shape[1:])
    with pytest.raises(PspwError) as e:
        Cell.from_arrays(args)
    assert e.value.code == 9  # lm_end > 4 (ApplyHam_block.cpp:70-73)
    d = torch.zeros(4, int(G["ngw"]), dtype=torch.complex128, device="cuda")
    with pytest.raises(PspwError) as e:
        gcell.apply_ham_block_dev(d, d, int(G["ngw"]), int(G["ngw"]), 4, PREC_F64)
    assert e.value.code == 1


def test_si64_subset_parity_and_hermiticity():
    # the 64-atom, 64^3 cell: FP64 parity on 8 bands, and <x|H y> = <H x|y>
    w = workloads.workload("si64")
    cell = workloads.make_cell(w)
    psi = np.asfortranarray(w["psi"][:, :8])
    out = cell.apply_ham_block(psi)
    ref = O.apply_ham_block(oracle_cell(w), psi, w["veff"])
    assert relmax(out, ref) < TOL64
    m = psi.conj().T @ out
    assert np.abs(m - m.conj().T).max() < 1e-12 * np.abs(m).max()


@pytest.mark.parametrize("prec", [PREC_F32, PREC_F64])
def test_projection_overlap_gives_identical_bits(prec):
    """The projection concurrent with the FFT passes (second stream) or after
    them: the same kernels in the same order of arithmetic, so the same bits;
    the Si64 cell (64 atoms, 64^3 grid) with 24 bands, and the Chebyshev
    filter, whose back-projection epilogue applies the recurrence."""
    w = workloads.workload("si64")
    cell = workloads.make_cell(w)
    psi = w["psi"][:, :24]
    ngw, nb = psi.shape
    cdt = torch.complex64 if prec == PREC_F32 else torch.complex128
    d_in = torch.from_numpy(np.ascontiguousarray(psi.T)).to(cdt).cuda()
    outs, filt = [], []
    for mode in (OVERLAP_ON, OVERLAP_OFF, OVERLAP_AUTO):
        cell.set_nl_overlap(mode)
        d_out = torch.zeros_like(d_in)
        torch.cuda.synchronize()
        cell.apply_ham_block_dev(d_in, d_out, ngw, ngw, nb, prec)
        x = d_in.clone()
        torch.cuda.synchronize()
        cell.chebyfilt_dev(x, ngw, ngw, nb, 4, 0.5, 16.0, prec)
        torch.cuda.synchronize()
        outs.append(d_out.cpu())
        filt.append(x.cpu())
    for o in outs[1:]:
        assert torch.equal(o, outs[0])
    for f in filt[1:]:
        assert torch.equal(f, filt[0])
    with pytest.raises(PspwError):
        cell.set_nl_overlap(3)


def _hpsi32(cell, psi, ld=None):
    ngw, nb = psi.shape
    ld = ld or ngw
    host = np.zeros((nb, ld), dtype=np.complex64)
    host[:, :ngw] = psi.T
    d_in = torch.from_numpy(host).cuda()
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    cell.apply_ham_block_dev(d_in, d_out, ld, ngw, nb, PREC_F32)
    torch.cuda.synchronize()
    return d_out.cpu().numpy()[:, :ngw].T.astype(complex)


@pytest.mark.parametrize("lm_end,nb", [([4], 1), ([4], 16), ([3], 7), ([2], 33), ([1], 5)])
def test_fp32_tensor_core_projectors(lm_end, nb):
    """tcgen05 3xTF32 projector GEMMs against the oracle and the SIMT kernels,
    over projector counts L = 1..4 and band counts that leave ragged M and N
    tiles (N tile = bands x 2L rounded to a multiple of 16)."""
    d = dict(G)
    args = engine_cell_args(d)
    args["lm_end"] = lm_end
    cell = Cell.from_arrays(args)
    cell.set_veff(G["veff"])
    rng = np.random.default_rng(nb)
    psi = G["psi"][:, rng.integers(0, G["psi"].shape[1], nb)]
    psi = np.asfortranarray(psi.astype(np.complex64).astype(complex))
    oc = oracle_cell(d)
    oc["lm_end"] = lm_end
    ref = O.apply_ham_block(oc, psi, G["veff"])
    cell.set_nl_path(NL_TENSOR_CORE)
    out_tc = _hpsi32(cell, psi, ld=psi.shape[0] + 3)
    cell.set_nl_path(NL_SIMT)
    out_simt = _hpsi32(cell, psi)
    assert relmax(out_tc, ref) < TOL32
    assert relmax(out_simt, ref) < TOL32
    assert relmax(out_tc, out_simt) < TOL32


def test_fp32_tensor_core_atoms_not_a_multiple_of_16():
    # 5 atoms: the atom (N) dimension of the projection is padded to 16
    lat, pos = synth.si_diamond(1)
    b = basis_gamma(lat, 8.0, None, [5], [pos[:5]])
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=[4])
    veff = synth.local_potential(b["nr"], lat, pos)
    psi = synth.wavefunctions(b, lat, 9, 3).astype(np.complex64).astype(complex)
    cell = Cell.from_arrays(b)
    cell.set_veff(veff)
    cell.set_nl_path(NL_TENSOR_CORE)
    oc = oracle_cell(b)
    oc.update(na=[5])
    ref = O.apply_ham_block(oc, psi, veff)
    assert relmax(_hpsi32(cell, psi), ref) < TOL32


def test_fp32_tensor_core_si64_all_bands():
    # 64 atoms, 144 bands: 9 M tiles x split-K in the projection, 5 band
    # tiles in the back-projection; against the engine's own FP64 path
    w = workloads.workload("si64")
    cell = workloads.make_cell(w)
    psi = np.asfortranarray(w["psi"].astype(np.complex64).astype(complex))
    ref = cell.apply_ham_block(psi)
    cell.set_nl_path(NL_TENSOR_CORE)
    out = _hpsi32(cell, psi)
    assert relmax(out, ref) < TOL32
    out2 = _hpsi32(cell, psi)
    assert np.array_equal(out, out2)  # fixed-order split-K reduction


def test_fp32_tensor_core_fewer_plane_waves_than_the_cell(cfg0):
    # the projection K range stops at ngw inside an 8-G operand tile
    w, cell = cfg0
    ngw = 2003
    psi = np.asfortranarray(w["psi"][:ngw, :12].astype(np.complex64).astype(complex))
    cell.set_nl_path(NL_TENSOR_CORE)
    out = _hpsi32(cell, psi)
    ref = O.apply_ham_block(oracle_cell(w), psi, w["veff"])
    assert relmax(out, ref) < TOL32


def _multi_species_cell(na, lm_end, rc, seed):
    lat, pos = synth.si_diamond(1)
    rng = np.random.default_rng(seed)
    pos = pos + rng.uniform(-0.3, 0.3, pos.shape)  # no two species share a site pattern
    tau, k = [], 0
    for n in na:
        tau.append(pos[k:k + n])
        k += n
    b = basis_gamma(lat, 8.0, None, na, tau)
    pkg_a, wnl = synth.kb_form_factors(b, lat, nsp=len(na), rc=rc)
    for s, lm in enumerate(lm_end):
        wnl[s, :4] = [1.5 - 0.3 * s, -0.8 + 0.2 * s, -0.8 + 0.2 * s, -0.8 + 0.2 * s]
        pkg_a[lm:, :, s] = 0.0
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=lm_end)
    veff = synth.local_potential(b["nr"], lat, pos)
    return b, veff, lat


@pytest.mark.parametrize("na,lm_end,rc", [
    ([5, 3], [4, 1], [1.0, 0.8]),                          # two species, s+p and s
    ([2, 2, 3, 1], [4, 1, 4, 3], [1.0, 0.8, 1.2, 0.9]),    # four species (the serving jobs')
    ([3, 4, 1], [4, 0, 2], [1.0, 0.8, 1.1]),               # a species without projectors
])
def test_fp32_tensor_core_several_species(na, lm_end, rc):
    """tcgen05 projector GEMMs per species (each species' atoms, PKG_A and
    weights; the back-projections add into one output) against the oracle
    and the SIMT kernels."""
    b, veff, lat = _multi_species_cell(na, lm_end, rc, len(na))
    cell = Cell.from_arrays(b)
    cell.set_veff(veff)
    psi = synth.wavefunctions(b, lat, 11, 5).astype(np.complex64).astype(complex)
    oc = oracle_cell(b)
    oc.update(na=na, lm_end=lm_end)
    ref = O.apply_ham_block(oc, psi, veff)
    cell.set_nl_path(NL_TENSOR_CORE)
    out_tc = _hpsi32(cell, psi, ld=psi.shape[0] + 1)
    cell.set_nl_path(NL_SIMT)
    out_simt = _hpsi32(cell, psi)
    assert relmax(out_tc, ref) < TOL32
    assert relmax(out_simt, ref) < TOL32
    assert relmax(out_tc, out_simt) < TOL32


def test_fp32_tensor_core_several_species_filter():
    # the filter's recurrence epilogue is applied once, by the first species
    na, lm_end = [4, 4], [4, 2]
    b, veff, lat = _multi_species_cell(na, lm_end, [1.0, 0.9], 7)
    cell = Cell.from_arrays(b)
    cell.set_veff(veff)
    cell.set_nl_path(NL_TENSOR_CORE)
    X = synth.wavefunctions(b, lat, 9, 2)
    out = cell.chebyfilt(X, 6, 1.5, 5.0, PREC_F32)
    oc = oracle_cell(b)
    oc.update(na=na, lm_end=lm_end)
    ref = O.chebyfilt(oc, X, 6, 1.5, 5.0, veff)
    assert relmax(out, ref) < 1e-4


def test_tensor_core_path_refused_beyond_256_atoms_per_species():
    # 264 atoms of one species: the tensor-core kernels take at most 256
    lat, pos = synth.si_diamond(1)
    big = np.concatenate([pos + 0.01 * k for k in range(33)])[:264]
    b = basis_gamma(lat, 4.0, None, [264], [big])
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=[1])
    cell = Cell.from_arrays(b)
    with pytest.raises(PspwError) as e:
        cell.set_nl_path(NL_TENSOR_CORE)
    assert e.value.code == 9
