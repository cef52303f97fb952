"""Shared test helpers: golden fixtures, oracle cells and error norms."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def oracle_cell(d):
    """The oracle's cell dict from a golden fixture or a workload dict."""
    return dict(nr=tuple(int(x) for x in d["nr"]), n123=np.asarray(d["n123"]),
                xkg=np.asarray(d["xkg"]), eigr=np.asarray(d["eigr"]),
                pkg_a=np.asarray(d["pkg_a"]), wnl=np.asarray(d["wnl"]),
                na=[int(np.asarray(d["eigr"]).shape[1])] if "na" not in d else list(d["na"]),
                lm_end=[4] if "lm_end" not in d else list(d["lm_end"]),
                tpiba2=float(d["tpiba2"]))


def engine_cell_args(d):
    c = oracle_cell(d)
    c.update(ngw=int(d["ngw"]), ngwx=int(d["ngwx"]))
    return c


def relmax(a, b):
    """max |a-b| / max |b| (the relative max-norm of the parity bar)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def ref_lib_or_none():
    try:
        from ref_lib import RefLib, ref_available
    except Exception:
        return None
    if not ref_available():
        return None
    return RefLib()


def write_synthetic_fhi(path, zv=4.0, well=1.0):
    """A synthetic norm-conserving pseudopotential in the FHI98 text layout
    the reference reads (ReadPseudopotentials.cpp:27-62): `ZV nang`, ten
    skipped lines, then per angular momentum `mmax clog` and mmax rows
    `i r u(r) V(r)` on a logarithmic mesh.  The model: V_loc = -ZV erf(r)/r
    + well exp(-(r/1.2)^2), V_s = V_loc + 1.5 exp(-(r/0.9)^2),
    V_p = V_loc - 0.7 exp(-(r/1.1)^2), V_d = V_loc; u_l(r) = r^(l+1)
    exp(-r^2/4) normalised."""
    from math import erf, exp, sqrt
    mmax, r1, fac = 495, 4.5e-4, 1.0247
    rs = [r1 * fac ** i for i in range(mmax)]

    def vloc(r):
        return -zv * erf(r) / r + well * exp(-(r / 1.2) ** 2)

    def vl(l, r):
        if l == 0:
            return vloc(r) + 1.5 * exp(-(r / 0.9) ** 2)
        if l == 1:
            return vloc(r) - 0.7 * exp(-(r / 1.1) ** 2)
        return vloc(r)

    lines = [f"{zv:.5E}    3"] + [" 0.0000    .00e+00   .00e+00"] * 10
    h = (fac - 1.0)
    for l in range(3):
        u = [r ** (l + 1) * exp(-r * r / 4.0) for r in rs]
        norm = sqrt(sum(x * x * r for x, r in zip(u, rs)) * h)
        lines.append(f"{mmax}  {fac:.14E}")
        for i, r in enumerate(rs):
            lines.append(f"{i + 1:4d} {r:.14E} {u[i] / norm:.14E} {vl(l, r):.14E}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_input(path, fhi_name, positions, a, ecut_ry=8.0, iscf=1, idiag=0, imix=2,
                max_scf=40, nempty=5):
    """An INPUT file in the reference's keyword format (ReadInputFile.cpp)."""
    pos = "\n".join(f"  {p[0]:.9f} {p[1]:.9f} {p[2]:.9f}" for p in positions)
    txt = (f"iscf\n {iscf}\n\nidiag\n {idiag}\n\nimix\n {imix}\n\nrho_mix_fac\n 0.3\n\n"
           f"max_scf_iter\n {max_scf}\n\nnempty\n {nempty}\n\necut\n {ecut_ry}\n\n"
           f"atoms\n 1\n {len(positions)}\n {fhi_name}\n 3 3\n bohr\n{pos}\n\n"
           f"latvec\n {a} 0.0 0.0\n 0.0 {a} 0.0\n 0.0 0.0 {a}\n\n"
           f"k_points\n 1\n 0.0 0.0 0.0 1.0\n")
    with open(path, "w") as f:
        f.write(txt)


def scf_lines(log):
    """The `! iter ETOT dETOT drho` lines of a reference log."""
    out = []
    for line in log.splitlines():
        parts = line.split()
        if len(parts) == 5 and parts[0] == "!":
            out.append((int(parts[1]), float(parts[2]), float(parts[3]), float(parts[4])))
    return out
