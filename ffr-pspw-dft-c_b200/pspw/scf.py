"""The SCF pieces of the C ABI (pspw_scf_*, pspw_eval_energy, pspw_xc_pz,
pspw_normalize_rho, pspw_kerker_prec, pspw_mix*) and the device SCF loop
(pspw_cheby_scf) over a Cell."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


class ScfParams(C.Structure):
    """pspw_scf_params: the INPUT controls of the SCF loop."""
    _fields_ = [("nx", C.c_int), ("nempty", C.c_int), ("degree", C.c_int),
                ("max_scf_iter", C.c_int), ("conv", C.c_double), ("imix", C.c_int),
                ("mixdim", C.c_int), ("mix_beta", C.c_double), ("pulay_beta", C.c_double),
                ("kerker_q0", C.c_double), ("idiag", C.c_int), ("max_diag_iter", C.c_int),
                ("filter_prec", C.c_int), ("tmetal", C.c_int), ("ekt", C.c_double)]


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

    @classmethod
    def borrow(cls, handle, cell, owner=None):
        """A view of an SCF handle owned elsewhere (e.g. by a System)."""
        s = cls.__new__(cls)
        s._h = handle
        s._owned = False
        s._owner = owner
        s.cell = cell
        sz = cell.sizes()
        s.nnr = int(sz["n1"] * sz["n2"] * sz["n3"])
        return s

    def close(self):
        if self._h and getattr(self, "_owned", True):
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

    def cheby_scf(self, focc, rho_start, v0, X=None, *, nx, nempty, degree=10,
                  max_scf_iter=40, conv=1e-6, imix=0, mixdim=4, mix_beta=0.3,
                  pulay_beta=0.25, kerker_q0=0.5, idiag=0, max_diag_iter=0, filter_prec=0):
        """The SCF loop of ChebySCFLoop.cpp on the device (pspw_cheby_scf).
        X: NGW x (NX+2) start block for idiag < 0 (ignored otherwise).
        Returns a dict with eig (NX), X (final block), rho (final mixed
        density), hist (iterations x {ETOT, |dETOT|, d, ms since the call
        began}), energies, iterations and converged."""
        ngw = self.cell.sizes()["ngw"]
        nx2 = nx + 2
        p = ScfParams(nx, nempty, degree, max_scf_iter, conv, imix, mixdim, mix_beta, pulay_beta,
                      kerker_q0, idiag, max_diag_iter, filter_prec)
        fo = _c(focc, float)
        rs = _c(rho_start, float)
        v = _c(np.asarray(v0, complex)[:ngw], complex)
        x = (np.zeros((ngw, nx2), complex) if X is None
             else np.asarray(X, complex)[:ngw, :nx2].copy())
        xf = np.asfortranarray(x)
        eig = np.zeros(nx)
        rho = np.zeros(self.nnr)
        hist = np.zeros(4 * max_scf_iter)
        its, cv = C.c_int(0), C.c_int(0)
        e6 = np.zeros(6)
        check(lib().pspw_cheby_scf(self._h, C.byref(p), fo.ctypes.data, rs.ctypes.data,
                                   v.ctypes.data, xf.ctypes.data, eig.ctypes.data,
                                   rho.ctypes.data, hist.ctypes.data, C.byref(its), C.byref(cv),
                                   e6.ctypes.data))
        n = its.value
        return dict(eig=eig, X=xf, rho=rho, hist=hist.reshape(-1, 4)[:n], iterations=n,
                    converged=bool(cv.value),
                    energies=dict(zip(("ETOT", "EKIN", "EHT", "EPSEU", "ENL", "EXC"),
                                      e6.tolist())))
