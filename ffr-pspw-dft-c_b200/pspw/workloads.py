"""The engine's named workloads: diamond-cubic silicon cells with the
synthetic local + KB pseudopotential of pspw.synth.

    si8    Si 8-atom cell,   a = 10.26 bohr, ecutwfc 15 Ha, grid 32^3, 16 bands
    si64   Si 64-atom cell,  a = 20.52 bohr, ecutwfc 15 Ha, grid 64^3, 144 bands
    si216  Si 216-atom cell, a = 30.78 bohr, ecutwfc 15 Ha, grid 96^3, 512 bands

ECUT is given in Rydberg as in the reference's INPUT (15 Ha = 30 Ry); the
grids are forced (below the reference's own grid rule, which does not change
the algorithm).  Wavefunctions are seeded with numpy's default_rng(seed).
"""
from __future__ import annotations

import numpy as np

from . import synth
from .cell import Cell, basis_gamma

WORKLOADS = {
    "si8": dict(nrep=1, grid=32, nbands=16, seed=2024),
    "si64": dict(nrep=2, grid=64, nbands=144, seed=2025),
    "si216": dict(nrep=3, grid=96, nbands=512, seed=2027),
}

ECUT_RY = 30.0


def si_cell(nrep, grid, ecut_ry=ECUT_RY, with_veff=True):
    """Basis, projectors and V_loc of a diamond Si supercell (Fortran layouts)."""
    lat, pos = synth.si_diamond(nrep)
    nr = (grid, grid, grid) if grid else None
    b = basis_gamma(lat, ecut_ry, nr, na=[len(pos)], tau=[pos])
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=[4], lattice=lat, positions=pos)
    if with_veff:
        b["veff"] = synth.local_potential(b["nr"], lat, pos)
    return b


def workload(name):
    w = WORKLOADS[name]
    c = si_cell(w["nrep"], w["grid"])
    c["psi"] = synth.wavefunctions(c, c["lattice"], w["nbands"], w["seed"])
    c["nbands"] = w["nbands"]
    c["name"] = name
    return c


def make_cell(c, device=0):
    cell = Cell.from_arrays(c, device=device)
    cell.set_veff(c["veff"])
    return cell


def hpsi_bytes(ngw, nnr, nb, nat, nsp=1, nlm=4, fp64=False):
    """Algorithmic bytes of one block H*psi: every 3D FFT counts one full read
    and one write of the grid; psi in/out once; V, maps and projector inputs
    once per block.  s_c/s_r = 16/8 B (FP64) or 8/4 B (FP32)."""
    sc, sr = (16, 8) if fp64 else (8, 4)
    return (nb * (2 * ngw + 4 * nnr) * sc + nnr * sr + ngw * (4 + sr)
            + ngw * (nat * sc + nsp * nlm * sr))


def hpsi_flops(ngw, nnr, nb, nat, nlm=4):
    """(projector flops, FFT flops) of one block H*psi (complex MAC = 8)."""
    f_nl = 16 * ngw * nat * nlm * nb
    f_fft = nb * 2 * 5 * nnr * np.log2(nnr)
    return f_nl, f_fft
