"""A synthetic SCF test case shared by the SCF-piece tests: the reference's
own set-up of the 8-atom Si cell (grid, density G list), synthetic local
pseudopotential data and a positive density.  Needs oracle/_ref/libref.so."""
import numpy as np

from ref_lib import RefLib


def make_case(ecut_ry=10.0, seed=7, grid=None):
    from pspw import synth
    lat, pos = synth.si_diamond(1)
    R = RefLib("libref.so")
    b = R.setup(lat, ecut_ry, grid, [8], [pos], [4.0], [3], [3], 4)
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    R.set_nl(pkg_a, wnl)
    b.update(pkg_a=pkg_a, wnl=wnl)
    rng = np.random.default_rng(seed)
    ng = int(b["ng"])
    G = np.asarray(b["G"])[:ng]
    sfac = (rng.standard_normal(ng) + 1j * rng.standard_normal(ng)) * 4.0 * np.exp(-0.05 * G)
    sfac[0] = 8.0
    vps = -4.0 * np.exp(-0.3 * G) / (1.0 + G)
    rhops = -0.05 * np.exp(-0.5 * G)
    nel, esr, eself = 32.0, 1.25, 3.5
    R.set_local(sfac.reshape(ng, 1), vps.reshape(ng, 1), rhops.reshape(ng, 1), esr, eself, nel)
    nr = b["nr"]
    nnr = int(np.prod(nr))
    # a smooth positive density with NEL electrons
    x = np.arange(nnr)
    i1, i2, i3 = x % nr[0], (x // nr[0]) % nr[1], x // (nr[0] * nr[1])
    f = (np.cos(2 * np.pi * i1 / nr[0]) * np.cos(2 * np.pi * i2 / nr[1])
         + 0.5 * np.sin(4 * np.pi * i3 / nr[2]) + 0.2 * rng.standard_normal(nnr))
    rho = 1.0 + 0.4 * f
    rho *= nnr * nel / b["omega"] / rho.sum()
    gidx = (np.asarray(b["N1"])[:ng] - 1) + nr[0] * ((np.asarray(b["N2"])[:ng] - 1)
                                                     + nr[1] * (np.asarray(b["N3"])[:ng] - 1))
    local = dict(gidx=gidx.astype(np.int64), g=G, vp=sfac * vps, rp=sfac * rhops,
                 omega=b["omega"], esr=esr, eself=eself)
    return dict(ref=R, b=b, sfac=sfac, vps=vps, rhops=rhops, nel=nel, esr=esr, eself=eself,
                rho=rho, local=local, nnr=nnr, ng=ng,
                ocell=dict(nr=tuple(nr), n123=b["n123"], xkg=b["xkg"], ngw=b["ngw"],
                           tpiba2=b["tpiba2"]))


def engine_scf(case):
    from pspw import Cell
    from pspw.scf import Scf
    b = case["b"]
    cell = Cell.from_arrays(dict(nr=b["nr"], ngw=b["ngw"], ngwx=b["ngwx"], n123=b["n123"],
                                 xkg=b["xkg"], tpiba2=b["tpiba2"], na=[8], lm_end=[4],
                                 eigr=b["eigr"], pkg_a=b["pkg_a"], wnl=b["wnl"]))
    ng = case["ng"]
    s = Scf(cell, b["N1"][:ng], b["N2"][:ng], b["N3"][:ng], b["G"][:ng], case["sfac"],
            case["vps"], case["rhops"], b["omega"], case["nel"], case["esr"], case["eself"])
    return cell, s
