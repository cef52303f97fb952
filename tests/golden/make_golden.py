"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference implementation built from its own sources
(oracle/_ref/libref.so, `make -C oracle`) on small synthetic cells and stores
inputs and outputs as compressed .npz files.  Needs the reference checkout
only to build libref.so; the fixtures are committed and the tests read them
without it.

    python tests/golden/make_golden.py

Cells: 8-atom diamond Si, a = 10.26 bohr, synthetic local + KB potential
(ffr-pspw-dft-c_b200/pspw/synth.py):
  si8_8ry   ECUT 8 Ry, the reference's own grid rule (20^3, NGW 437)
  si8_cfg0  ECUT 30 Ry, forced 32^3 grid (NGW 2945): basis checksums only
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ffr-pspw-dft-c_b200"))

from ref_lib import RefLib  # noqa: E402
from pspw import synth  # noqa: E402


def main():
    lat, pos = synth.si_diamond(1)
    R = RefLib()
    b = R.setup(lat, 8.0, None, [8], [pos], [4.0], [3], [3], 4)
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    R.set_nl(pkg_a, wnl)
    veff = synth.local_potential(b["nr"], lat, pos)
    ngw = b["ngw"]
    psi = synth.wavefunctions(b, lat, 6, 11)
    hpsi = R.apply_ham_block(psi, veff)
    h1 = R.apply_ham(psi[:, 0].copy(), veff)
    R.set_nx(4, 2)  # chebyfilt's block width is NX+2 = 6 (chebyfilt.cpp:20)
    cheb = R.chebyfilt(psi, 4, 2.0, 4.0, veff)
    T, f = R.lanczos(psi[:, 1].copy(), 8, veff)
    prec = R.gen_prec(ngw, -10.0)
    rnd = R.random_col(64, 100)
    q = R.ortho_qr(psi * (1.0 + 0.5j) + 0.01)
    flat = np.concatenate([psi.reshape(-1, order="F"), np.zeros(b["ngwx"], complex)])
    rho, ekin, c0 = R.eval_rho_psi(flat, ngw, ngw, 4, np.array([2.0, 2.0, 2.0, 2.0]))
    np.savez_compressed(
        os.path.join(HERE, "si8_8ry.npz"),
        lattice=lat, positions=pos, nr=np.array(b["nr"]), ngw=ngw, ngwx=b["ngwx"], ngx=b["ngx"],
        ng=b["ng"], tpiba2=b["tpiba2"], alat=b["alat"], omega=b["omega"], n123=b["n123"],
        xkg=b["xkg"], igk=b["igk"], eigr=b["eigr"], pkg_a=pkg_a, wnl=wnl, veff=veff, psi=psi,
        hpsi=hpsi, h1=h1, cheb=cheb, cheb_degree=4, cheb_lb=2.0, cheb_ub=4.0, lanczos_T=T,
        lanczos_f=f, prec=prec, random_col=rnd, ortho_in=psi * (1.0 + 0.5j) + 0.01, ortho_q=q,
        rho=rho, ekin=ekin, c0=c0, focc=np.array([2.0, 2.0, 2.0, 2.0]))
    print("wrote si8_8ry.npz", b["nr"], ngw)


def basis_checksums():
    """Basis of the 32^3, 30 Ry cell in a fresh process (the reference keeps one cell per
    process)."""
    lat, pos = synth.si_diamond(1)
    R = RefLib()
    b = R.setup(lat, 30.0, (32, 32, 32), [8], [pos], [4.0], [3], [3], 4)
    ngw = b["ngw"]
    np.savez_compressed(
        os.path.join(HERE, "si8_cfg0_basis.npz"), nr=np.array(b["nr"]), ngw=ngw,
        ngwx=b["ngwx"], ngx=b["ngx"], ng=b["ng"], n123=b["n123"][:ngw], xkg=b["xkg"][:ngw],
        igk=b["igk"][:ngw], eigr_sum=b["eigr"][:ngw].sum(axis=0),
        eigr_probe=b["eigr"][:ngw:97, :, 0])
    print("wrote si8_cfg0_basis.npz", b["nr"], ngw)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "cfg0":
        basis_checksums()
    else:
        main()
        import subprocess
        subprocess.check_call([sys.executable, os.path.abspath(__file__), "cfg0"])
