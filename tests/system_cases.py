"""Input directories in the reference's own formats for the system tests, and
the reference's set-up of them run in a separate process
(ref_program_case.py): an 8-atom Si crystal and a two-species molecule in a
box (one N-like species with s and p channels, three H-like atoms with a
local channel only), with synthetic FHI98 pseudopotentials."""
import os
import subprocess
import sys

import numpy as np

from helpers import write_input, write_synthetic_fhi

HERE = os.path.dirname(os.path.abspath(__file__))

MOLECULE_INPUT = """iscf
 1

imix
 {imix}

ecut
 {ecut}

max_scf_iter
 {max_scf}

atoms
 2
 1 3
 N.fhi
 2  2
 {coord}
{n_pos}
 H.fhi
 1  1
 {coord}
{h_pos}

latvec
 {a}   0.0   0.0
  0.0   {a}   0.0
  0.0   0.0   {a}

k_points
 1
 0.0 0.0 0.0 1.0
"""

N_POS = [(-0.109736, 0.043732, 0.05751)]
H_POS = [(1.00912, -1.4209, -0.47067), (-0.61394, 0.9989, -1.52628), (-1.70223, -0.6834, 0.84038)]


def _fmt(rows):
    return "\n".join(f" {x:.6f} {y:.6f} {z:.6f}" for x, y, z in rows)


def write_si8(d, ecut_ry=8.0, **kw):
    from pspw import synth
    os.makedirs(d, exist_ok=True)
    lat, pos = synth.si_diamond(1)
    write_synthetic_fhi(os.path.join(d, "X.fhi"))
    write_input(os.path.join(d, "INPUT"), "X.fhi", pos, 10.26, ecut_ry=ecut_ry, **kw)
    return d


def write_molecule(d, ecut_ry=10.0, a=10.0, imix=3, max_scf=40, coord="bohr"):
    os.makedirs(d, exist_ok=True)
    write_synthetic_fhi(os.path.join(d, "N.fhi"), zv=5.0, well=0.5)
    write_synthetic_fhi(os.path.join(d, "H.fhi"), zv=1.0, well=0.2)
    n_pos, h_pos = N_POS, H_POS
    if coord == "angstrom":
        n_pos = [tuple(0.529 * x for x in p) for p in N_POS]
        h_pos = [tuple(0.529 * x for x in p) for p in H_POS]
    with open(os.path.join(d, "INPUT"), "w") as f:
        f.write(MOLECULE_INPUT.format(imix=imix, ecut=ecut_ry, max_scf=max_scf, coord=coord,
                                      n_pos=_fmt(n_pos), h_pos=_fmt(h_pos), a=a))
    return d


def reference_setup(d, setup_only=True, timeout=900):
    """The reference's set-up of directory d (and its SCF unless
    setup_only), run by ref_program_case.py; returns (arrays, ctrl, stdout)."""
    out = os.path.join(d, "ref_case.npz")
    args = [sys.executable, os.path.join(HERE, "ref_program_case.py"), d, out]
    if setup_only:
        args.append("setup")
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
    z = dict(np.load(out))
    ctrl = dict(zip(z.pop("ctrl_names").tolist(), z.pop("ctrl_values").tolist()))
    return z, ctrl, r.stdout
