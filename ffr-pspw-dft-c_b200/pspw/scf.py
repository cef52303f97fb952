"""The SCF pieces of the C ABI (pspw_scf_*, pspw_eval_energy, pspw_xc_pz,
pspw_normalize_rho, pspw_kerker_prec, pspw_mix*) over a Cell."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


def _c(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


class Scf:
    """Local-potential data and density-mixing state of one cell.

    g_list: dict with N1, N2, N3 (1-based grid indices of the NG density G
    vectors, G = 0 first) and G (|G|^2 in (2 pi/alat)^2 units); sfac, vps,
    rhops: NG x NSP arrays (as numpy, species in the second axis) or NSP x NG
    in the reference's memory order when passed flat."""

    def __init__(self, cell, n1, n2, n3, g, sfac, vps, rhops, omega, nel, esr, eself):
        self.cell = cell  # keeps the cell alive
        n1, n2, n3 = _c(n1, np.int32), _c(n2, np.int32), _c(n3, np.int32)
        g = _c(g, float)
        ng = len(g)
        sfac = np.asarray(sfac, dtype=complex).reshape(ng, -1)
        nsp = sfac.shape[1]
        sf = _c(sfac, complex)                      # (ng, nsp) C order = species fastest
        vp = _c(np.asarray(vps, float).reshape(ng, nsp), float)
        rp = _c(np.asarray(rhops, float).reshape(ng, nsp), float)
        self._keep = (n1, n2, n3, g, sf, vp, rp)
        h = C.c_void_p()
        check(lib().pspw_scf_create(cell.handle, ng, n1.ctypes.data, n2.ctypes.data,
                                    n3.ctypes.data, g.ctypes.data, nsp, sf.ctypes.data,
                                    vp.ctypes.data, rp.ctypes.data, float(omega), float(nel),
                                    float(esr), float(eself), C.byref(h)))
        self._h = h
        self.nnr = int(np.prod(cell.sizes()["n1"] * cell.sizes()["n2"] * cell.sizes()["n3"]))

    def close(self):
        if self._h:
            lib().pspw_scf_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def eval_energy(self, rho, ekin, enl):
        """Returns (V_eff, {ETOT, EKIN, EHT, EPSEU, ENL, EXC})."""
        r = np.array(rho, dtype=float, copy=True)
        e = np.zeros(6)
        check(lib().pspw_eval_energy(self._h, r.ctypes.data, float(ekin), float(enl),
                                     e.ctypes.data))
        return r, dict(zip(("ETOT", "EKIN", "EHT", "EPSEU", "ENL", "EXC"), e.tolist()))

    def xc_pz(self, rho):
        r = _c(rho, float)
        v = np.zeros_like(r)
        e = C.c_double(0.0)
        check(lib().pspw_xc_pz(self._h, r.ctypes.data, v.ctypes.data, C.byref(e)))
        return v, e.value

    def normalize_rho(self, rho):
        r = np.array(rho, dtype=float, copy=True)
        w = C.c_int(0)
        check(lib().pspw_normalize_rho(self._h, r.ctypes.data, C.byref(w)))
        return r, bool(w.value)

    def kerker_prec(self, x, beta, q0):
        r = np.array(x, dtype=float, copy=True)
        check(lib().pspw_kerker_prec(self._h, r.ctypes.data, float(beta), float(q0)))
        return r

    def mix_init(self, kind, mixdim=0, beta=0.25, q0=0.0, rho_old=None):
        ro = None if rho_old is None else _c(rho_old, float)
        check(lib().pspw_mix_init(self._h, int(kind), int(mixdim), float(beta), float(q0),
                                  None if ro is None else ro.ctypes.data))

    def mix(self, it, rhoe):
        r = np.array(rhoe, dtype=float, copy=True)
        d = C.c_double(0.0)
        check(lib().pspw_mix(self._h, int(it), r.ctypes.data, C.byref(d)))
        return r, d.value
