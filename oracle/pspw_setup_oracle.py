"""TEST INFRASTRUCTURE -- CPU restatement of the reference's set-up (the oracle
for the device set-up of pspw_system_load).

Only ``tests/`` may import this module, as the checker.  numpy FP64, one
function per reference routine, each citing the file:line it follows; arrays
keep the reference's Fortran layouts.  The inputs are the reference's own
basis arrays (``RefLib.program_setup`` or ``pspw.basis_gamma``) and the FHI98
tables read by ``read_fhi``.
"""
from __future__ import annotations

from math import erf

import numpy as np
from scipy.special import erfc

MAXR = 570  # common_pspw.h


def read_fhi(path, lmax):
    """ReadPseudopotentials.cpp:20-64: `ZV nang`, ten skipped lines, then per
    channel l <= min(nang, L_MAX) a `mmax ratio` header and mmax rows
    `i r u(r) V(r)`; CLOG = log(ratio)."""
    with open(path) as f:
        lines = f.read().split("\n")
    head = lines[0].split()
    zv, nang = float(head[0]), int(head[1])
    assert nang >= lmax
    k = 11
    r = np.zeros(MAXR)
    psi = np.zeros((3, MAXR))
    vion = np.zeros((3, MAXR))
    mmax, clog = 0, 0.0
    for il in range(min(nang, lmax)):
        h = lines[k].split()
        k += 1
        mmax, clog = int(h[0]), float(np.log(float(h[1])))
        for ir in range(mmax):
            _, a, b, c = lines[k].split()[:4]
            k += 1
            r[ir], psi[il, ir], vion[il, ir] = float(a), float(b), float(c)
    return dict(zv=zv, mmax=mmax, clog=clog, r=r, psi=psi, vion=vion)


def simpson(f, h):
    """simpson.cpp:5-16 with dsum.cpp's running sums."""
    n = len(f)
    m = (n - 1) // 2
    return (4.0 * np.sum(f[1:2 * m:2]) + 2.0 * np.sum(f[2:2 * m - 1:2]) + f[0] + f[n - 1]) * h / 3.0


def _crystal(lattice, tau):
    A = np.asarray(lattice, dtype=float).reshape(3, 3)  # rows A1, A2, A3
    return np.linalg.solve(A.T, np.asarray(tau, dtype=float).T).T


def structure_factor(lattice, tau_by_species, in123):
    """StructureFactor.cpp:17-27 with the phase tables of PhaseFactor.cpp:
    SFAC(is, ig) = sum_a exp(-2 pi i n(ig) . tau'_a).  in123: (ng, 3) Miller
    indices.  Returns (NSP, NG)."""
    out = []
    for tau in tau_by_species:
        tp = _crystal(lattice, tau)                        # (na, 3)
        ph = -2.0 * np.pi * (np.asarray(in123, dtype=float) @ tp.T)  # (ng, na)
        out.append(np.exp(1j * ph).sum(axis=1))
    return np.array(out)


def eigr(lattice, tau_by_species, in123_w, ngwx, nax):
    """PhaseFactor.cpp:66-78: EIGR(ig, a, s) = exp(-2 pi i n(ig) . tau'_a),
    zero past NGW and for a >= NA(s)."""
    nsp = len(tau_by_species)
    e = np.zeros((ngwx, nax, nsp), dtype=complex)
    for s, tau in enumerate(tau_by_species):
        tp = _crystal(lattice, tau)
        ph = -2.0 * np.pi * (np.asarray(in123_w, dtype=float) @ tp.T)
        e[: len(in123_w), : len(tau), s] = np.exp(1j * ph)
    return e


def form_factor(sp, G, tpiba, tpiba2, omega, lloc, rgauss=1.0):
    """FormFactor.cpp:28-70 for one species: VPS(ig) and RHOPS(ig) over the
    density sphere G (|G|^2 in (2 pi/ALAT)^2, G[0] = 0)."""
    m, r = sp["mmax"], sp["r"][: sp["mmax"]]
    vloc = sp["vion"][lloc - 1, :m] - np.array([-sp["zv"] / x * erf(x / rgauss) for x in r])
    fpibom = 4.0 * np.pi / omega
    vps = np.zeros(len(G))
    vps[0] = simpson(vloc * r ** 3, sp["clog"]) * fpibom
    g = np.asarray(G[1:], dtype=float)
    x = np.outer(np.sqrt(g), r) * tpiba                   # (ng-1, m)
    f = vloc * np.sin(x) / x * r ** 3
    vps[1:] = [simpson(row, sp["clog"]) * fpibom for row in f]
    rhops = np.zeros(len(G))
    rhops[1:] = -sp["zv"] / omega * np.exp(-0.25 * tpiba2 * rgauss * rgauss * g)
    return vps, rhops


def nl_form_factor(sp, xkg, ggk, tpiba, omega, lmax, lloc, nlmax):
    """NLFormFactor.cpp:24-118 for one species: PKG_A(lm, ig) over the
    wavefunction sphere and WNL(lm).  ggk: (ngw, 3) G vectors."""
    m, r = sp["mmax"], sp["r"][: sp["mmax"]]
    ngw = len(xkg)
    pkg = np.zeros((nlmax, ngw))
    wnl = np.zeros(nlmax)
    t = np.sqrt(np.asarray(xkg, dtype=float))
    arg = np.outer(t * tpiba, r)
    ml = 0
    for l in range(1, lmax + 1):
        if l == lloc:
            continue
        dv = sp["vion"][l - 1, :m] - sp["vion"][lloc - 1, :m]
        fun = dv * sp["psi"][l - 1, :m] * r * r
        q = simpson(dv * sp["psi"][l - 1, :m] ** 2 * r, sp["clog"])
        wnl[ml: ml + 2 * l - 1] = (2.0 * l - 1.0) * 4.0 * np.pi / omega / q
        small = t < 1.0e-4
        with np.errstate(divide="ignore", invalid="ignore"):
            if l == 1:
                fac = np.where(small[:, None], 1.0, np.sin(arg) / arg)
            elif l == 2:
                fac = (np.sin(arg) / arg - np.cos(arg)) / arg
            else:
                fac = ((3.0 / arg ** 2 - 1.0) * np.sin(arg) - 3.0 / arg * np.cos(arg)) / arg
            q1 = np.array([simpson(row, sp["clog"]) for row in fac * fun])
            c = np.asarray(ggk, dtype=float) / t[:, None]
        if l == 1:
            pkg[ml] = q1
        elif l == 2:
            for j in range(3):
                pkg[ml + j] = np.where(small, 0.0, q1 * c[:, j])
        else:
            cx, cy, cz = c[:, 0], c[:, 1], c[:, 2]
            s3 = np.sqrt(3.0)
            vals = [q1 * 0.5 * (3.0 * cz ** 2 - 1.0), q1 * s3 * cz * cx, q1 * s3 * cz * cy,
                    q1 * s3 * cx * cy, q1 * s3 / 2.0 * (cx ** 2 - cy ** 2)]
            for j in range(5):
                pkg[ml + j] = np.where(small, 0.0, vals[j])
        ml += 2 * l - 1
    return pkg, wnl


_OCC = {1.0: (1.0, 0, 0), 0.75: (0.75, 0, 0), 1.25: (1.25, 0, 0), 2.0: (2.0, 0, 0),
        3.0: (2.0, 1.0, 0), 4.0: (2.0, 2.0, 0), 5.0: (2.0, 3.0, 0), 6.0: (2.0, 4.0, 0),
        7.0: (2.0, 5.0, 0), 8.0: (2.0, 6.0, 0), 9.0: (1.0, 0, 8.0), 10.0: (2.0, 0, 8.0),
        11.0: (1.0, 0, 10.0), 12.0: (2.0, 0, 10.0), 13.0: (2.0, 1.0, 10.0),
        14.0: (2.0, 2.0, 10.0), 15.0: (2.0, 3.0, 10.0), 16.0: (2.0, 4.0, 10.0),
        17.0: (2.0, 5.0, 10.0), 18.0: (2.0, 6.0, 10.0)}


def atomic_density_g(sp, G, tpiba, omega, lmax):
    """FormFactorAtomic.cpp:30-152 for one species: q(ig) with the occupations
    of the valence-charge table; the caller sums q * SFAC over species."""
    occ = next(v for z, v in _OCC.items() if abs(sp["zv"] - z) < 1e-4)
    m, r = sp["mmax"], sp["r"][: sp["mmax"]]
    p = sp["psi"][:, :m]
    f = occ[0] * p[0] ** 2
    if lmax >= 2:
        f = f + occ[1] * p[1] ** 2
    if lmax >= 3:
        f = f + occ[2] * p[2] ** 2
    f = f * r / omega
    q = np.zeros(len(G))
    q[0] = simpson(f, sp["clog"])
    x = np.outer(np.sqrt(np.asarray(G[1:], dtype=float)), r) * tpiba
    q[1:] = [simpson(row, sp["clog"]) for row in f * np.sin(x) / x]
    return q


def starting_density(qat, n123_density, nr, omega, nel):
    """ChebySCFLoop.cpp:157-168: qat on the grid, inverse FFT (exp(+iGr),
    unscaled), real part, NormalizeRho (NormalizeRho.cpp:7-33)."""
    from pspw_oracle import fft_inverse, normalize_rho
    grid = np.zeros(int(np.prod(nr)), dtype=complex)
    grid[np.asarray(n123_density) - 1] = qat
    return normalize_rho(fft_inverse(grid, nr).real, omega, nel)


def ewald(lattice, tau_by_species, zv, rgauss):
    """EwaldEnergy.cpp:31-112: the real-space Gaussian-screened sum over the
    lattice vectors within 30 bohr plus the 27 nearest cells, positions
    folded into the cell."""
    A = np.asarray(lattice, dtype=float).reshape(3, 3)
    taus, zs, rgs = [], [], []
    for s, tau in enumerate(tau_by_species):
        tp = _crystal(A, tau)
        tp = tp - np.floor(tp)
        taus.append(tp @ A)
        zs += [zv[s]] * len(tau)
        rgs += [rgauss[s]] * len(tau)
    tw = np.vstack(taus)
    zs, rgs = np.array(zs), np.array(rgs)
    omega = abs(np.linalg.det(A))
    nc = max(int(round(5.0 * 30.0 / omega ** (1.0 / 3.0))), 2)
    rl = []
    for i in range(-nc, nc + 1):
        for j in range(-nc, nc + 1):
            for k in range(-nc, nc + 1):
                t = i * A[0] + j * A[1] + k * A[2]
                if t @ t <= 900.0 or (abs(i) <= 1 and abs(j) <= 1 and abs(k) <= 1):
                    rl.append(t)
    rl = np.array(rl)
    esr = 0.0
    for a1 in range(len(tw)):
        d = tw[a1][None, None, :] - (rl[:, None, :] + tw[None, :, :])   # (nr, nat, 3)
        dist = np.sqrt((d ** 2).sum(axis=2))
        gkl = 1.0 / np.sqrt(rgs[a1] ** 2 + rgs ** 2)
        mask = dist > 0
        x = dist * gkl[None, :]
        fac = zs[a1] * zs[None, :] / np.where(mask, dist, 1.0) * 0.5
        esr += float((erfc(x) * fac)[mask].sum())
    return esr
