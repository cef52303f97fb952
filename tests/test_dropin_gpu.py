"""The drop-in library inside the reference's own host program.

oracle/_ref/libref_dropin.so is the reference built from its sources with
ApplyHam_block.cpp, ApplyHam.cpp and chebyfilt.cpp left out and
libpspw_dropin.so linked in their place; oracle/_ref/libref.so is the
unmodified reference.  The same harness calls go to both, so these tests
compare the reference with the engine behind the reference's own signatures
and globals, including the reference's Davidson and LOBPCG solvers running on
top of the drop-in ApplyHam_block.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from helpers import relmax  # noqa: E402
from ref_lib import RefLib, ref_available  # noqa: E402

if not (ref_available("libref.so") and ref_available("libref_dropin.so")):
    pytest.skip("oracle/_ref reference builds not present", allow_module_level=True)

from pspw import synth  # noqa: E402


@pytest.fixture(scope="module")
def pair():
    lat, pos = synth.si_diamond(1)
    libs = []
    for name in ("libref.so", "libref_dropin.so"):
        R = RefLib(name)
        b = R.setup(lat, 12.0, None, [8], [pos], [4.0], [3], [3], 4)
        pkg_a, wnl = synth.kb_form_factors(b, lat)
        R.set_nl(pkg_a, wnl)
        libs.append(R)
    veff = synth.local_potential(b["nr"], lat, pos)
    psi = synth.wavefunctions(b, lat, 10, 21)
    return libs[0], libs[1], b, veff, psi


def test_apply_ham_block_through_reference_signature(pair):
    ref, drop, b, veff, psi = pair
    assert relmax(drop.apply_ham_block(psi, veff), ref.apply_ham_block(psi, veff)) < 1e-12


def test_apply_ham_single_vector(pair):
    ref, drop, b, veff, psi = pair
    v = psi[:, 3].copy()
    assert relmax(drop.apply_ham(v, veff), ref.apply_ham(v, veff)) < 1e-12


def test_chebyfilt_block_width_is_nx_plus_2(pair):
    ref, drop, b, veff, psi = pair
    for R in (ref, drop):
        R.set_nx(8, 4)  # NX + 2 = 10 columns
    out_d = drop.chebyfilt(psi, 10, 1.0, 6.0, veff)
    out_r = ref.chebyfilt(psi, 10, 1.0, 6.0, veff)
    assert relmax(out_d, out_r) < 1e-12


def test_reference_davidson_on_dropin_hamiltonian(pair):
    ref, drop, b, veff, psi = pair
    ngw = b["ngw"]
    prec = ref.gen_prec(ngw, -10.0)
    ev_r, _ = ref.davidson(ngw, 12, veff, prec, 4, max_iter=8)
    ev_d, _ = drop.davidson(ngw, 12, veff, prec, 4, max_iter=8)
    assert np.abs(ev_r - ev_d).max() < 1e-9


def test_reference_lanczos_on_dropin_apply_ham(pair):
    ref, drop, b, veff, psi = pair
    T_r, f_r = ref.lanczos(psi[:, 0].copy(), 12, veff)
    T_d, f_d = drop.lanczos(psi[:, 0].copy(), 12, veff)
    assert np.abs(T_r - T_d).max() < 1e-10
