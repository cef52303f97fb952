"""The oracle (oracle/pspw_oracle.py) pinned against the reference.

Two anchors:
  * golden fixtures made by running the reference itself (tests/golden/,
    generated by make_golden.py from oracle/_ref/libref.so) -- always run;
  * the reference built from its own sources, called on the same inputs --
    run when oracle/_ref/libref.so is present.
"""
import numpy as np
import pytest

import pspw_oracle as O
from helpers import golden, oracle_cell, ref_lib_or_none, relmax

G = golden("si8_8ry")
CELL = oracle_cell(G)


def test_apply_ham_block_matches_reference_output():
    out = O.apply_ham_block(CELL, G["psi"], G["veff"])
    assert relmax(out, G["hpsi"]) < 1e-13


def test_apply_ham_single_vector():
    out = O.apply_ham(CELL, G["psi"][:, 0], G["veff"])
    assert relmax(out, G["h1"]) < 1e-13


def test_chebyfilt_matches_reference_output():
    out = O.chebyfilt(CELL, G["psi"], int(G["cheb_degree"]), float(G["cheb_lb"]),
                      float(G["cheb_ub"]), G["veff"])
    assert relmax(out, G["cheb"]) < 1e-12


def test_chebyfilt_coefficients_reproduce_filter():
    # the (a, b, c) step form used by the fused device recurrence
    X = G["psi"]
    coeffs = O.chebyfilt_step_coeffs(int(G["cheb_degree"]), float(G["cheb_lb"]),
                                     float(G["cheb_ub"]))
    ym2, ym1 = None, X
    for d, (a, b, c) in enumerate(coeffs):
        y = a * O.apply_ham_block(CELL, ym1, G["veff"]) + b * ym1
        if d > 0:
            y = y + c * ym2
        ym2, ym1 = ym1, y
    assert relmax(ym1, G["cheb"]) < 1e-12


def test_lanczos_matches_reference_output():
    T, f = O.lanczos(CELL, G["psi"][:, 1], 8, G["veff"])
    assert np.abs(T - G["lanczos_T"]).max() < 1e-11
    assert relmax(f, G["lanczos_f"]) < 1e-8


def test_random_col_bit_exact():
    assert np.array_equal(O.random_col(64, 100), G["random_col"])


def test_gen_prec_bit_exact():
    ngw = int(G["ngw"])
    p = O.gen_prec(G["xkg"][:ngw], float(G["alat"]), float(G["tpiba2"]), -10.0)
    assert np.array_equal(p, G["prec"])


def test_ortho_qr_matches_householder():
    q = O.ortho_qr(G["ortho_in"])
    assert np.abs(q - G["ortho_q"]).max() < 1e-14


def test_eval_rho_psi_matches_reference_output():
    ngw, ngwx = int(G["ngw"]), int(G["ngwx"])
    psi = G["psi"]
    flat = np.concatenate([psi.reshape(-1, order="F"), np.zeros(ngwx, complex)])
    rho, ekin, c0 = O.eval_rho_psi(CELL, flat, ngw, ngw, 4, G["focc"], 1.0, float(G["omega"]),
                                   ngwx)
    assert relmax(rho, G["rho"]) < 1e-13
    assert abs(ekin - float(G["ekin"])) < 1e-12 * abs(float(G["ekin"]))
    assert np.array_equal(c0, G["c0"])


def test_eval_rho_psi_charge_check_aborts():
    # EvalRhoPsi.cpp:129-133: a band whose |c|^2 sum is off by > 6e-3 is an error
    ngw, ngwx = int(G["ngw"]), int(G["ngwx"])
    bad = 1.01 * G["psi"]
    flat = np.concatenate([bad.reshape(-1, order="F"), np.zeros(ngwx, complex)])
    with pytest.raises(RuntimeError, match="Wrong charge"):
        O.eval_rho_psi(CELL, flat, ngw, ngw, 4, G["focc"], 1.0, float(G["omega"]), ngwx)


def test_symmetrize_equals_loop_form():
    rng = np.random.default_rng(0)
    v = rng.standard_normal((7, 7)) + 1j * rng.standard_normal((7, 7))
    ref = v.copy()
    for j in range(7):
        for i in range(j + 1):
            t = 0.5 * (ref[i, j] + np.conj(ref[j, i]))
            ref[i, j] = t
            ref[j, i] = np.conj(t)
    assert np.array_equal(O.symmetrize(v), ref)


# ------------------------------------------------------------ live reference
REF = ref_lib_or_none()
need_ref = pytest.mark.skipif(REF is None, reason="oracle/_ref/libref.so not built")


@pytest.fixture(scope="module")
def ref_cell():
    from pspw import synth
    lat, pos = synth.si_diamond(1)
    b = REF.setup(lat, 8.0, None, [8], [pos], [4.0], [3], [3], 4)
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    REF.set_nl(pkg_a, wnl)
    cell = dict(nr=b["nr"], n123=b["n123"], xkg=b["xkg"], eigr=b["eigr"], pkg_a=pkg_a, wnl=wnl,
                na=[8], lm_end=[4], tpiba2=b["tpiba2"])
    veff = synth.local_potential(b["nr"], lat, pos)
    return b, cell, veff, lat


@need_ref
def test_live_davidson_eigenvalues(ref_cell):
    b, cell, veff, _ = ref_cell
    ngw = b["ngw"]
    prec = O.gen_prec(b["xkg"][:ngw], b["alat"], b["tpiba2"], -10.0)
    ev_r, _ = REF.davidson(ngw, 12, veff, prec, 4, max_iter=6)
    ev_o, _, _ = O.davidson(cell, ngw, 12, veff, prec, 4, max_iter=6)
    assert np.abs(ev_r - ev_o).max() < 1e-9


@need_ref
def test_live_lobpcg_eigenvalues(ref_cell):
    b, cell, veff, _ = ref_cell
    ngw = b["ngw"]
    prec = O.gen_prec(b["xkg"][:ngw], b["alat"], b["tpiba2"], -10.0)
    ev_r, _ = REF.lobpcg(ngw, 12, veff, prec, 4, max_iter=6)
    ev_o, _, _ = O.lobpcg(cell, ngw, 12, veff, prec, 4, max_iter=6)
    assert np.abs(ev_r - ev_o).max() < 1e-9


@need_ref
def test_live_eig_zhegv_eval(ref_cell):
    rng = np.random.default_rng(3)
    n = 10
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a = a + a.conj().T
    m = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    bm = m @ m.conj().T + n * np.eye(n)
    w_r, v_r = REF.eig_zhegv_eval(a, bm)
    w_o, v_o, _ = O.eig_zhegv_eval(a, bm)
    assert np.abs(w_r - w_o).max() < 1e-12
    assert np.abs(np.abs(v_r) - np.abs(v_o)).max() < 1e-10


@need_ref
def test_live_eval_enl(ref_cell):
    # EvalENL.cpp:5-49 on the C0 that EvalRhoPsi copies, with unequal occupations
    b, cell, veff, lat = ref_cell
    from pspw import synth
    ngw, ngwx = b["ngw"], b["ngwx"]
    psi = synth.wavefunctions(b, lat, 6, 31)
    flat = np.concatenate([psi.reshape(-1, order="F"), np.zeros(ngwx, complex)])
    focc = np.array([2.0, 2.0, 2.0, 1.5, 0.5, 0.0])
    REF.eval_rho_psi(flat, ngw, ngw, 6, focc)
    enl_r = REF.eval_enl()
    enl_o, _ = O.eval_enl(cell, psi, ngw, 6, focc, 1.0)
    assert abs(enl_o - enl_r) < 1e-12 * abs(enl_r)


# ------------------------------------------------------------ SCF pieces
@pytest.fixture(scope="module")
def scf_case():
    from scf_case import make_case
    return make_case()


@need_ref
def test_live_xc_pz_with_stale_points(scf_case):
    rho = scf_case["rho"].copy()
    rho[0] = -0.3  # no earlier point: the reference's variables start unset
    rho[11] = -0.2  # keeps point 10's values (xc_PZ.cpp:27-30)
    rho[12] = 1e-14
    v_r, e_r = scf_case["ref"].xc_pz(rho)
    v_o, e_o = O.xc_pz(rho)
    assert np.abs(v_o[1:] - v_r[1:]).max() < 1e-14
    assert abs(e_o - e_r) < 1e-12 * abs(e_r)


@need_ref
def test_live_eval_energy(scf_case):
    c = scf_case
    v_r, e_r = c["ref"].eval_energy(c["rho"], 12.5, 0.75)
    v_o, e_o = O.eval_energy(c["rho"], c["local"], dict(c["ocell"]), 12.5, 0.75)
    assert np.abs(v_o - v_r).max() < 1e-12 * np.abs(v_r).max()
    for k in e_r:
        assert abs(e_o[k] - e_r[k]) < 1e-11 * max(1.0, abs(e_r[k])), k


@need_ref
def test_live_eval_energy_on_an_aliasing_grid(scf_case):
    """16^3 for a density sphere that needs 21 points per axis: density G
    share grid points, and the reference's scatter in G order leaves the
    last one's V(G) there; the oracle does the same."""
    from scf_case import make_case
    try:
        c = make_case(grid=(16, 16, 16))
        gidx = c["local"]["gidx"]
        assert len(np.unique(gidx)) < len(gidx)
        v_r, e_r = c["ref"].eval_energy(c["rho"], 12.5, 0.75)
        v_o, e_o = O.eval_energy(c["rho"], c["local"], dict(c["ocell"]), 12.5, 0.75)
        assert np.abs(v_o - v_r).max() < 1e-12 * np.abs(v_r).max()
        for k in e_r:
            assert abs(e_o[k] - e_r[k]) < 1e-11 * max(1.0, abs(e_r[k])), k
    finally:
        make_case()  # the module case's set-up back in the reference's globals


@need_ref
def test_live_normalize_and_kerker(scf_case):
    c = scf_case
    r = c["rho"] * 1.01
    r[3] = -0.5
    n_r = c["ref"].normalize_rho(r, c["b"]["omega"], c["nel"])
    assert np.abs(O.normalize_rho(r, c["b"]["omega"], c["nel"]) - n_r).max() < 1e-14 * n_r.max()
    x = c["rho"] - c["rho"].mean()
    k_r = c["ref"].kerker_prec(x, 0.8, 0.6)
    assert np.abs(O.kerker_prec(x, c["ocell"], 0.8, 0.6) - k_r).max() < 1e-12 * np.abs(k_r).max()


def _mix_sequence(c, n=6, seed=3):
    rng = np.random.default_rng(seed)
    return [c["rho"] * (1.0 + 0.05 * rng.standard_normal(c["nnr"])) for _ in range(n)]


@need_ref
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_live_mixers(scf_case, kind):
    import ctypes as C
    c = scf_case
    R, nnr = c["ref"], c["nnr"]
    mixdim = 3
    R.lib.ref_set_mixing(0.6)
    seq = _mix_sequence(c)
    om = O.Mixer(kind, nnr, c["ocell"], mixdim=mixdim, beta=0.3 if kind < 3 else 0.25, q0=0.6,
                 omega=c["b"]["omega"], nel=c["nel"], rho_old=c["rho"] if kind < 2 else None)
    cols = mixdim if kind == 3 else (2 if kind == 4 else 3)
    h = np.zeros((nnr, cols), order="F")
    f = np.zeros((nnr, cols), order="F")
    g = np.zeros((nnr, 2), order="F")
    df = np.zeros((nnr, mixdim), order="F")
    u = np.zeros((nnr, mixdim), order="F")
    a = np.zeros((mixdim, mixdim), order="F")
    if kind < 2:
        h[:, 0] = c["rho"]
    for it, rin in enumerate(seq, start=1):
        r_ref = rin.copy()
        if kind == 0:
            d_r = R.lib.ref_SimpleRhoMix(0.3, r_ref, h[:, 0], nnr)
        elif kind == 1:
            d_r = R.lib.ref_KerkerRhoMix(0.3, 0.6, r_ref, h[:, 0], nnr)
        elif kind == 2:
            d_r = R.lib.ref_AndersonRhoMix(it, 0.3, r_ref, h.reshape(-1, order="F"),
                                           f.reshape(-1, order="F"), g.reshape(-1, order="F"),
                                           nnr)
        elif kind == 3:
            d_r = R.lib.ref_PulayRhoMix(it, r_ref, h.reshape(-1, order="F"),
                                        f.reshape(-1, order="F"), mixdim, nnr)
        else:
            d_r = R.lib.ref_BroydenRhoMix(it, 0.25, 0.01, r_ref, h.reshape(-1, order="F"),
                                          f.reshape(-1, order="F"), df.reshape(-1, order="F"),
                                          u.reshape(-1, order="F"), a.reshape(-1, order="F"),
                                          mixdim, nnr)
        r_o, d_o = om.mix(it, rin)
        assert np.abs(r_o - r_ref).max() < 1e-9 * np.abs(r_ref).max(), (kind, it)
        assert abs(d_o - d_r) < 1e-9 * max(1.0, abs(d_r)), (kind, it)
