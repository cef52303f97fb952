"""The INPUT and FHI98 readers and the host part of the system set-up
(pspw_system_load with device = -1: ReadInputFile, ReadPseudopotentials,
Setup, InitOcc, WNL, ESELF) against the reference's own set-up run from the
same files (oracle/_ref/libref.so, in a process of its own), the reader edge
cases, Print3DArray's format, and the set-up oracle (oracle/pspw_setup_oracle)
pinned against the reference's set-up arrays."""
import os

import numpy as np
import pytest

from pspw import PspwError
from pspw.system import System, print_3d_array
from system_cases import reference_setup, write_molecule, write_si8

REF = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle", "_ref", "libref.so")
needs_ref = pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref not built")


def _case(tmp_path, name):
    d = str(tmp_path / name)
    if name == "si8":
        return write_si8(d)
    if name == "molecule":
        return write_molecule(d)
    if name == "molecule_angstrom":
        return write_molecule(d, coord="angstrom")
    raise KeyError(name)


@needs_ref
@pytest.mark.parametrize("name", ["si8", "molecule", "molecule_angstrom"])
def test_host_setup_matches_reference(tmp_path, name):
    d = _case(tmp_path, name)
    z, ctrl, _ = reference_setup(d)
    S = System(d, device=-1)
    dm = S.dims
    assert dm["nr"] == tuple(int(x) for x in z["nr"])
    for k in ("ngw", "ngwx", "ng", "ngx", "nx", "nlmax", "nax", "nsp"):
        assert dm[k] == int(z[k]), k
    for k in ("omega", "tpiba2", "nel", "eself"):
        assert S.scalars[k] == float(z[k]), k
    for k in ("n123", "xkg", "focc", "wnl", "tau"):
        assert np.array_equal(S.array(k), z[k]), k
    assert np.array_equal(S.array("g"), z["G"][: dm["ng"]])
    p = S.params()
    assert (p["nx"], p["nempty"], p["degree"], p["max_scf_iter"], p["imix"], p["mixdim"],
            p["idiag"]) == tuple(int(ctrl[k]) for k in ("nx", "nempty", "degree", "max_scf_iter",
                                                        "imix", "mixdim", "idiag"))
    assert (p["conv"], p["mix_beta"], p["kerker_q0"]) == (ctrl["conv"], ctrl["rho_mix_fac"],
                                                          ctrl["kerker_q0"])
    S.close()


def _write(d, text, fhi=("X.fhi",)):
    from helpers import write_synthetic_fhi
    os.makedirs(d, exist_ok=True)
    for f in fhi:
        write_synthetic_fhi(os.path.join(d, f))
    with open(os.path.join(d, "INPUT"), "w") as f:
        f.write(text)
    return d


BASE = """atoms
 1
 2
 X.fhi
 3 3
 {coord}
 0.10 0.20 0.30
 0.40 0.50 0.60

latvec
 8.0 0.0 0.0
 0.0 9.0 0.0
 0.0 0.0 10.0

ecut
 6.0

k_points
 1
 0.0 0.0 0.0 1.0
"""


def test_reader_defaults_and_forced_grid(tmp_path):
    d = _write(str(tmp_path / "a"), BASE.format(coord="bohr") + "\nfft_grid\n 24 24 30\n\n"
               "max_diag_iter\n 7\n")
    S = System(d, device=-1)
    assert S.dims["nr"] == (24, 24, 30)
    p = S.params()
    # ReadInputFile.cpp:22-35 defaults; IMIX is a zero-initialised global
    assert (p["degree"], p["max_scf_iter"], p["mixdim"], p["imix"], p["idiag"]) == (10, 30, 4, 0, 0)
    assert (p["conv"], p["mix_beta"], p["kerker_q0"]) == (1e-6, 0.3, 0.5)
    assert p["max_diag_iter"] == 7
    assert S.dims["nempty"] == 5 and S.dims["nx"] == 5 + 4
    assert np.array_equal(S.array("focc"), np.array([2.0] * 4 + [0.0] * 5))


def test_reader_coordinate_conversions(tmp_path):
    ang = System(_write(str(tmp_path / "ang"), BASE.format(coord="angstrom")), device=-1)
    t = ang.array("tau")[:, :, 0].T
    assert np.array_equal(t, np.array([[0.1, 0.2, 0.3], [0.4, 0.5, 0.6]]) / 0.529)
    cry = System(_write(str(tmp_path / "cry"), BASE.format(coord="crystal")), device=-1)
    # ReadInputFile.cpp:200-205 converts x, y, z in place one after the other
    A = np.array([[8.0, 0, 0], [0, 9.0, 0], [0, 0, 10.0]])
    want = []
    for p in ([0.1, 0.2, 0.3], [0.4, 0.5, 0.6]):
        p = list(p)
        for c in range(3):
            p[c] = p[0] * A[0][c] + p[1] * A[1][c] + p[2] * A[2][c]
        want.append(p)
    assert np.array_equal(cry.array("tau")[:, :, 0].T, np.array(want))


@pytest.mark.parametrize("bad,needle", [
    ("\nunknown_key\n 1\n", "unknown line"),
    ("\natoms\n 1\n 1\n missing.fhi\n 3 3\n bohr\n 0 0 0\n", "missing.fhi"),
])
def test_reader_errors(tmp_path, bad, needle):
    d = _write(str(tmp_path / "e"), BASE.format(coord="bohr") + bad)
    with pytest.raises(PspwError) as e:
        System(d, device=-1)
    assert needle in str(e.value)


def test_reader_too_few_angular_momenta(tmp_path):
    d = _write(str(tmp_path / "l"), BASE.format(coord="bohr"))
    path = os.path.join(d, "X.fhi")
    with open(path) as f:
        lines = f.read().split("\n")
    lines[0] = lines[0].split()[0] + "    2"
    with open(path, "w") as f:
        f.write("\n".join(lines))
    with pytest.raises(PspwError):
        System(d, device=-1)


def test_print_3d_array_format(tmp_path):
    a = np.array([0.0, 1.5, -2.25e-3, 123456.123456789, 1e-11, -0.5])
    p = tmp_path / "RHO.dat"
    print_3d_array(a, (1, 2, 3), p)
    assert p.read_text() == "".join(f"{x:18.10f}\n" for x in a)


# ------------------------------------------------------------------ oracle pin
def _recip(lattice):
    """CalcRecipLatt.cpp:9-21 (units of 2 pi / ALAT)."""
    A1, A2, A3 = np.asarray(lattice, dtype=float).reshape(3, 3)
    omega = np.linalg.det(np.array([A1, A2, A3]))
    s = A1[0] / omega
    B1 = np.array([A2[1] * A3[2] - A2[2] * A3[1], A1[2] * A3[1] - A1[1] * A3[2],
                   A1[1] * A2[2] - A1[2] * A2[1]]) * s
    B2 = np.array([A2[2] * A3[0] - A2[0] * A3[2], A1[0] * A3[2] - A1[2] * A3[0],
                   A1[2] * A2[0] - A1[0] * A2[2]]) * s
    B3 = np.array([A2[0] * A3[1] - A2[1] * A3[0], A1[1] * A3[0] - A1[0] * A3[1],
                   A1[0] * A2[1] - A1[1] * A2[0]]) * s
    return np.array([B1, B2, B3])


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@needs_ref
@pytest.mark.parametrize("name", ["si8", "molecule"])
def test_setup_oracle_matches_reference(tmp_path, name):
    import pspw_setup_oracle as so
    d = _case(tmp_path, name)
    z, ctrl, _ = reference_setup(d)
    S = System(d, device=-1)
    lat = np.array([[float(x) for x in S_lat] for S_lat in _lattice_rows(d)])
    ng, ngw, nsp = int(z["ng"]), int(z["ngw"]), int(z["nsp"])
    mill = np.stack([z["IN1"][:ng], z["IN2"][:ng], z["IN3"][:ng]], axis=1)
    igk = z["igk"][:ngw] - 1
    tau = z["tau"]
    na = [int(x) for x in z["na"]]
    taus = [tau[:, :na[s], s].T for s in range(nsp)]
    files = _species_files(d)
    lmax = [int(x) for x in _lmax_lloc(d)[0]]
    lloc = [int(x) for x in _lmax_lloc(d)[1]]
    sps = [so.read_fhi(os.path.join(d, f), lmax[s]) for s, f in enumerate(files)]
    # structure factor and phase factors
    sf = so.structure_factor(lat, taus, mill)
    assert _rel(sf, z["sfac"]) < 1e-12
    eg = so.eigr(lat, taus, mill[igk], int(z["ngwx"]), int(z["nax"]))
    assert _rel(eg, z["eigr"]) < 1e-12
    # local and nonlocal form factors
    G = z["G"][:ng]
    tp, tp2, om = float(z["tpiba"]), float(z["tpiba2"]), float(z["omega"])
    B = _recip(lat)
    ggk = mill[igk].astype(float) @ B
    for s in range(nsp):
        vps, rhops = so.form_factor(sps[s], G, tp, tp2, om, lloc[s])
        assert _rel(vps, z["vps"][s]) < 1e-12
        assert _rel(rhops, z["rhops"][s]) < 1e-12
        pkg, wnl = so.nl_form_factor(sps[s], z["xkg"][:ngw], ggk, tp, om, lmax[s], lloc[s],
                                     int(z["nlmax"]))
        if np.abs(z["pkg_a"][:, :ngw, s]).max() > 0:
            assert _rel(pkg, z["pkg_a"][:, :ngw, s]) < 1e-12
        assert _rel(wnl, z["wnl"][s]) < 1e-14 if np.abs(z["wnl"][s]).max() > 0 else True
    # starting density and Ewald sum
    qat = sum(so.atomic_density_g(sps[s], G, tp, om, lmax[s]) * z["sfac"][s] for s in range(nsp))
    n123d = z["N1"][:ng] + z["nr"][0] * ((z["N2"][:ng] - 1) + z["nr"][1] * (z["N3"][:ng] - 1))
    rho = so.starting_density(qat, n123d, tuple(int(x) for x in z["nr"]), om, float(z["nel"]))
    assert _rel(rho, z["rho_start"]) < 1e-11
    esr = so.ewald(lat, taus, [sp["zv"] for sp in sps], [1.0] * nsp)
    assert abs(esr - float(z["esr"])) <= 1e-12 * max(1.0, abs(float(z["esr"])))
    S.close()


def _input_lines(d):
    with open(os.path.join(d, "INPUT")) as f:
        return f.read().split("\n")


def _lattice_rows(d):
    L = _input_lines(d)
    i = L.index("latvec")
    return [L[i + k].split() for k in (1, 2, 3)]


def _species_files(d):
    L = _input_lines(d)
    return [x.strip() for x in L if x.strip().endswith(".fhi")]


def _lmax_lloc(d):
    L = _input_lines(d)
    out = [[], []]
    for k, x in enumerate(L):
        if x.strip().endswith(".fhi"):
            a, b = L[k + 1].split()
            out[0].append(int(a))
            out[1].append(int(b))
    return out
