"""Synthetic cells for the Hamiltonian engine's workloads.

The workloads use synthetic pseudopotentials instead of FHI98 tables:

* local part: V_loc(r) = sum over atoms and periodic images of
  depth * exp(-|r - tau|^2 / (2 width^2)) (depth -2 Ha, width 1.2 bohr for
  the silicon cells), built exactly as a Fourier series
  V(r) = (1/Omega) sum_G depth (2 pi width^2)^(3/2) exp(-width^2 G^2/2) S(G) e^{iG.r};
* Kleinman-Bylander part: s and p projectors per atom with radial factor
  exp(-q^2 rc^2 / 2), rc = 1.0 bohr, q = |G| in bohr^-1, and the reference's
  p convention PKG_A(2..4,G) = radial * G_alpha/|G| (0 at G = 0), as
  NLFormFactor.cpp:290-303 builds it; weights WNL = (1.5, 0.8, 0.8, 0.8) Ha;
* wavefunctions: c(G) ~ N(0,1)(1+i)-complex * exp(-|G|^2/8), orthonormalised
  by Householder QR, seeded with numpy.random.default_rng(seed).

Every array comes out in the reference's Fortran layouts (common_pspw.h), so
the same arrays can be handed to the reference and to the GPU engine.
"""
from __future__ import annotations

import numpy as np

DIAMOND_FRAC = np.array([
    [0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0],
    [0.25, 0.25, 0.25], [0.75, 0.25, 0.75], [0.25, 0.75, 0.75], [0.75, 0.75, 0.25],
])

SI_A0 = 10.26  # bohr, conventional diamond-cubic Si cell of the workloads


def si_diamond(nrep: int, a0: float = SI_A0):
    """Diamond-cubic Si supercell of nrep^3 conventional cells (8 nrep^3 atoms).
    Returns (lattice rows A1,A2,A3, positions (nat,3) in bohr)."""
    pos = []
    for i in range(nrep):
        for j in range(nrep):
            for k in range(nrep):
                pos.append((DIAMOND_FRAC + np.array([i, j, k])) * a0)
    L = nrep * a0
    return np.diag([L, L, L]), np.concatenate(pos, axis=0)


def recip_vectors(lattice):
    """B1, B2, B3 in units of 2 pi/ALAT, as CalcRecipLatt.cpp:5-23 forms them
    (ALAT = A1(1), Omega = det)."""
    A1, A2, A3 = (np.asarray(v, dtype=float) for v in lattice)
    omega = (A1[0] * (A2[1] * A3[2] - A2[2] * A3[1]) - A1[1] * (A2[0] * A3[2] - A2[2] * A3[0])
             + A1[2] * (A2[0] * A3[1] - A2[1] * A3[0]))
    s = A1[0] / omega
    B1 = np.array([(A2[1] * A3[2] - A2[2] * A3[1]), (A1[2] * A3[1] - A1[1] * A3[2]),
                   (A1[1] * A2[2] - A1[2] * A2[1])]) * s
    B2 = np.array([(A2[2] * A3[0] - A2[0] * A3[2]), (A1[0] * A3[2] - A1[2] * A3[0]),
                   (A1[2] * A2[0] - A1[0] * A2[2])]) * s
    B3 = np.array([(A2[0] * A3[1] - A2[1] * A3[0]), (A1[1] * A3[0] - A1[0] * A3[1]),
                   (A1[0] * A2[1] - A1[1] * A2[0])]) * s
    return B1, B2, B3, omega


def gk_cartesian(basis, lattice):
    """Cartesian G (units 2 pi/ALAT) of the wavefunction sphere, ngwx x 3."""
    B1, B2, B3, _ = recip_vectors(lattice)
    igk = np.asarray(basis["igk"])
    ngw = basis["ngw"]
    out = np.zeros((basis["ngwx"], 3))
    ig = igk[:ngw] - 1
    i, j, k = (np.asarray(basis[n])[ig].astype(float) for n in ("IN1", "IN2", "IN3"))
    out[:ngw] = i[:, None] * B1 + j[:, None] * B2 + k[:, None] * B3
    return out


def kb_form_factors(basis, lattice, nsp=1, rc=1.0, weights=(1.5, 0.8, 0.8, 0.8), nlmax=4):
    """Synthetic PKG_A(NLMAX,NGWX,NSP) and WNL(NSP,NLMAX) (Fortran layout)."""
    ngw, ngwx, tpiba = basis["ngw"], basis["ngwx"], basis["tpiba"]
    xkg = np.asarray(basis["xkg"])
    t = np.sqrt(xkg[:ngw])
    q = t * tpiba
    gc = gk_cartesian(basis, lattice)[:ngw]
    pkg_a = np.zeros((nlmax, ngwx, nsp), order="F")
    wnl = np.zeros((nsp, nlmax), order="F")
    rcs = rc if np.ndim(rc) else [rc] * nsp
    for s in range(nsp):
        rad_s = np.exp(-0.5 * (q * rcs[s]) ** 2)
        pkg_a[0, :ngw, s] = rad_s
        nz = t >= 1.0e-4
        for a in range(3):
            pkg_a[1 + a, :ngw, s] = np.where(nz, rad_s * gc[:, a] / np.where(nz, t, 1.0), 0.0)
        wnl[s, : len(weights)] = weights
    return pkg_a, wnl


def local_potential(nr, lattice, positions, depth=-2.0, width=1.2, species=None,
                    depths=None, widths=None):
    """V_loc on the FFT grid (NNR, i1 fastest), exact periodic Gaussian sum
    through its Fourier series.  Per-species depth/width when `species`
    (atom -> species index) and `depths`/`widths` are given."""
    n1, n2, n3 = nr
    lat = np.asarray(lattice, dtype=float)
    omega = abs(np.linalg.det(lat))
    recip = 2.0 * np.pi * np.linalg.inv(lat).T  # rows b_i with a_i . b_j = 2 pi delta
    f1 = np.fft.fftfreq(n1, 1.0 / n1)
    f2 = np.fft.fftfreq(n2, 1.0 / n2)
    f3 = np.fft.fftfreq(n3, 1.0 / n3)
    K3, K2, K1 = np.meshgrid(f3, f2, f1, indexing="ij")  # C order (i3,i2,i1)
    Gx = K1 * recip[0, 0] + K2 * recip[1, 0] + K3 * recip[2, 0]
    Gy = K1 * recip[0, 1] + K2 * recip[1, 1] + K3 * recip[2, 1]
    Gz = K1 * recip[0, 2] + K2 * recip[1, 2] + K3 * recip[2, 2]
    G2 = Gx * Gx + Gy * Gy + Gz * Gz
    pos = np.asarray(positions, dtype=float)
    vg = np.zeros_like(G2, dtype=complex)
    if species is None:
        species = np.zeros(len(pos), dtype=int)
        depths, widths = [depth], [width]
    for s in range(len(depths)):
        sel = pos[np.asarray(species) == s]
        if len(sel) == 0:
            continue
        w = widths[s]
        form = depths[s] * (2.0 * np.pi * w * w) ** 1.5 * np.exp(-0.5 * w * w * G2)
        sf = np.zeros_like(G2, dtype=complex)
        for p in sel:
            sf += np.exp(-1j * (Gx * p[0] + Gy * p[1] + Gz * p[2]))
        vg += form * sf
    # V(r_j) = (1/Omega) sum_G V(G) e^{+iG.r_j}: an unnormalised inverse DFT
    v = np.fft.ifftn(vg) * (G2.size / omega)
    return np.ascontiguousarray(v.real.reshape(-1))


def wavefunctions(basis, lattice, nbands, seed, orthonormalise=True):
    """Seeded Psi(G), ngw x nbands complex128 (Fortran order)."""
    ngw = basis["ngw"]
    rng = np.random.default_rng(seed)
    g2 = np.asarray(basis["xkg"][:ngw]) * basis["tpiba"] ** 2
    c = (rng.standard_normal((ngw, nbands)) + 1j * rng.standard_normal((ngw, nbands)))
    c *= np.exp(-g2 / 8.0)[:, None]
    c = np.asfortranarray(c)
    if orthonormalise:
        q, _ = np.linalg.qr(c)
        c = np.asfortranarray(q)
    return c
