"""TEST INFRASTRUCTURE -- ctypes binding of the reference built from its own
sources (oracle/_ref/libref.so, made by oracle/Makefile).

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s reference/CPU
baseline legs use this module.  ``RefLib(path)`` loads one build:
``libref.so`` (the reference's own hot path) or ``libref_dropin.so`` (the
reference host program linked against the GPU drop-in in place of its hot-path
objects); both export the same ``ref_*`` harness functions (ref_driver.cpp).
Each process can hold one cell per library, because the reference keeps its
state in globals.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_zp = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def ref_available(name="libref.so"):
    return os.path.exists(os.path.join(REF_DIR, name))


class RefLib:
    def __init__(self, name="libref.so", mode=C.RTLD_LOCAL):
        path = name if os.path.isabs(name) else os.path.join(REF_DIR, name)
        self.lib = C.CDLL(path, mode=mode)
        L = self.lib
        L.ref_setup_cell.argtypes = [_dp, C.c_double, _ip, C.c_int, _ip, _dp, _dp, _ip, _ip, C.c_int]
        L.ref_get_dims.argtypes = [_ip]
        L.ref_get_scalars.argtypes = [_dp]
        L.ref_get_basis.argtypes = [_up, _dp, _ip]
        L.ref_get_gvec.argtypes = [_ip, _ip, _ip, _ip, _ip, _ip, _dp]
        L.ref_get_eigr.argtypes = [_zp]
        L.ref_set_nl.argtypes = [_dp, _dp]
        L.ref_set_nx.argtypes = [C.c_int, C.c_int]
        L.ref_set_diag.argtypes = [C.c_int, C.c_int, C.c_int]
        L.ref_set_focc.argtypes = [_dp, C.c_int]
        L.ref_get_c0.argtypes = [_zp]
        L.ref_set_ekin.argtypes = [C.c_double]
        L.ref_get_ekin.restype = C.c_double
        L.ref_get_enl.restype = C.c_double
        L.ref_EvalENL.argtypes = []
        L.ref_set_local.argtypes = [_zp, _dp, _dp, C.c_double, C.c_double, C.c_double]
        L.ref_EvalEnergy.argtypes = [_dp, C.c_double, C.c_double, _dp]
        L.ref_xc_PZ.argtypes = [_dp, _dp, C.c_int]
        L.ref_xc_PZ.restype = C.c_double
        L.ref_NormalizeRho.argtypes = [_dp, C.c_int, C.c_double, C.c_double]
        L.ref_KerkerPrec.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_double]
        L.ref_set_mixing.argtypes = [C.c_double]
        L.ref_PulayRhoMix.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_int]
        L.ref_PulayRhoMix.restype = C.c_double
        L.ref_AndersonRhoMix.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, _dp, C.c_int]
        L.ref_AndersonRhoMix.restype = C.c_double
        L.ref_BroydenRhoMix.argtypes = [C.c_int, C.c_double, C.c_double, _dp, _dp, _dp, _dp,
                                        _dp, _dp, C.c_int, C.c_int]
        L.ref_BroydenRhoMix.restype = C.c_double
        L.ref_KerkerRhoMix.argtypes = [C.c_double, C.c_double, _dp, _dp, C.c_int]
        L.ref_KerkerRhoMix.restype = C.c_double
        L.ref_SimpleRhoMix.argtypes = [C.c_double, _dp, _dp, C.c_int]
        L.ref_SimpleRhoMix.restype = C.c_double
        L.ref_ApplyHam_block.argtypes = [_zp, _zp, C.c_int, _dp, C.c_int]
        L.ref_ApplyHam.argtypes = [_zp, _zp, C.c_int, _dp]
        L.ref_chebyfilt.argtypes = [_zp, C.c_int, C.c_double, C.c_double, _dp]
        L.ref_lanczos.argtypes = [_zp, C.c_int, _dp, C.c_int, _zp, _dp]
        L.ref_davidson.argtypes = [_dp, _zp, C.c_int, C.c_int, _dp, _dp]
        L.ref_lobpcg.argtypes = [_dp, _zp, C.c_int, C.c_int, _dp, _dp]
        L.ref_Diagon_davidson.argtypes = [_dp, _zp, C.c_int, _dp, C.c_double]
        L.ref_Diagon_lobpcg.argtypes = [_dp, _zp, C.c_int, _dp, C.c_double]
        L.ref_ortho_qr.argtypes = [_zp, C.c_int, C.c_int]
        L.ref_eig_zheevd.argtypes = [_zp, C.c_int, _dp, C.c_int]
        L.ref_eig_zhegv.argtypes = [_zp, C.c_int, _zp, C.c_int, _zp, C.c_int, C.c_int]
        L.ref_eig_zhegv_eval.argtypes = [_zp, C.c_int, _zp, C.c_int, _dp, _zp, C.c_int, C.c_int]
        L.ref_GenPrec.argtypes = [_dp, C.c_int, C.c_double]
        L.ref_EvalRhoPsi.argtypes = [_dp, _zp, C.c_int, C.c_int]
        L.ref_random_col.argtypes = [_zp, C.c_int, C.c_long]
        L.ref_fft.argtypes = [_zp, C.c_int]
        L.ref_prog_setup.argtypes = []
        L.ref_prog_start_density.argtypes = [_dp]
        L.ref_get_local.argtypes = [_zp, _dp, _dp, _dp]
        L.ref_get_nl.argtypes = [_dp, _dp]
        L.ref_get_species.argtypes = [_ip, _ip, _ip]
        L.ref_get_tau.argtypes = [_dp]
        L.ref_get_ctrl.argtypes = [_ip, _dp, _dp]
        L.ref_prog_cheby_scf.argtypes = [_dp, _dp]
        self.cell = None

    # ------------------------------------------------------------ set-up
    def setup(self, lattice, ecut_ry, nr, na, tau, zv, lmax, lloc, nempty):
        """lattice: 3x3 rows A1,A2,A3 (bohr); tau: list per species of (na,3)."""
        nsp = len(na)
        nax = max(na)
        taua = np.zeros((nsp, nax, 3))
        for s in range(nsp):
            taua[s, : na[s]] = np.asarray(tau[s], dtype=float).reshape(na[s], 3)
        nr_arr = np.asarray(nr if nr is not None else (0, 0, 0), dtype=np.int32)
        self.lib.ref_setup_cell(
            np.ascontiguousarray(np.asarray(lattice, dtype=float).reshape(9)),
            float(ecut_ry), nr_arr, nsp, np.asarray(na, dtype=np.int32),
            np.ascontiguousarray(taua.reshape(-1)), np.asarray(zv, dtype=float),
            np.asarray(lmax, dtype=np.int32), np.asarray(lloc, dtype=np.int32), int(nempty))
        return self._read_cell(list(na), lmax, lloc)

    def _read_cell(self, na, lmax, lloc):
        nsp = len(na)
        d = np.zeros(12, dtype=np.int32)
        self.lib.ref_get_dims(d)
        sc = np.zeros(8)
        self.lib.ref_get_scalars(sc)
        dims = dict(nr=(int(d[0]), int(d[1]), int(d[2])), nnr=int(d[3]), ngw=int(d[4]),
                    ngwx=int(d[5]), ngx=int(d[6]), ng=int(d[7]), nx=int(d[8]), nlmax=int(d[9]),
                    nax=int(d[10]), nsp=int(d[11]), tpiba=sc[0], tpiba2=sc[1], omega=sc[2],
                    alat=sc[3], gcut=sc[4], gcutw=sc[5], nel=sc[6])
        ngwx, ngx = dims["ngwx"], dims["ngx"]
        n123 = np.zeros(ngwx, dtype=np.uint32)
        xkg = np.zeros(ngwx)
        igk = np.zeros(ngwx, dtype=np.int32)
        self.lib.ref_get_basis(n123, xkg, igk)
        g = [np.zeros(ngx, dtype=np.int32) for _ in range(6)]
        gg = np.zeros(ngx)
        self.lib.ref_get_gvec(*g, gg)
        eigr = np.zeros(ngwx * dims["nax"] * nsp, dtype=complex)
        self.lib.ref_get_eigr(eigr)
        dims.update(n123=n123, xkg=xkg, igk=igk, N1=g[0], N2=g[1], N3=g[2], IN1=g[3],
                    IN2=g[4], IN3=g[5], G=gg,
                    eigr=eigr.reshape((ngwx, dims["nax"], nsp), order="F"),
                    na=list(na), lm_end=[int(l * l - 2 * ll + 1) for l, ll in zip(lmax, lloc)])
        self.cell = dims
        return dims

    # ------------------------------------------------ the reference program
    def program_setup(self, workdir):
        """The reference program's own set-up (main.cpp: ReadInputFile,
        Setup, PrepareSCF) on the INPUT in ``workdir``, its starting density
        (ChebySCFLoop.cpp:157-168) and EwaldEnergy.  Returns the cell dict of
        ``setup`` plus pkg_a, wnl, sfac/vps/rhops (nsp x ng, the reference's
        SFAC(NSP, NG) layout), esr, eself, tau,
        rho_start and the control values of the INPUT."""
        cwd = os.getcwd()
        os.chdir(workdir)
        try:
            self.lib.ref_prog_setup()
            d = np.zeros(12, dtype=np.int32)
            self.lib.ref_get_dims(d)
            nsp, nnr = int(d[11]), int(d[3])
            na, lmax, lloc = (np.zeros(nsp, dtype=np.int32) for _ in range(3))
            self.lib.ref_get_species(na, lmax, lloc)
            b = self._read_cell([int(x) for x in na], [int(x) for x in lmax],
                                [int(x) for x in lloc])
            rho = np.zeros(nnr)
            self.lib.ref_prog_start_density(rho)
        finally:
            os.chdir(cwd)
        ng, nlmax, ngwx = b["ng"], b["nlmax"], b["ngwx"]
        sfac = np.zeros(ng * nsp, dtype=complex)
        vps, rhops, scal = np.zeros(ng * nsp), np.zeros(ng * nsp), np.zeros(4)
        self.lib.ref_get_local(sfac, vps, rhops, scal)
        pkg_a, wnl = np.zeros(nlmax * ngwx * nsp), np.zeros(nsp * nlmax)
        self.lib.ref_get_nl(pkg_a, wnl)
        iv, dv, focc = np.zeros(9, dtype=np.int32), np.zeros(3), np.zeros(b["nx"])
        self.lib.ref_get_ctrl(iv, dv, focc)
        tau = np.zeros(3 * b["nax"] * nsp)
        self.lib.ref_get_tau(tau)
        b.update(sfac=sfac.reshape((nsp, ng), order="F"), vps=vps.reshape((nsp, ng), order="F"),
                 rhops=rhops.reshape((nsp, ng), order="F"), esr=scal[0], eself=scal[1],
                 pkg_a=pkg_a.reshape((nlmax, ngwx, nsp), order="F"),
                 wnl=wnl.reshape((nsp, nlmax), order="F"), rho_start=rho, focc=focc,
                 tau=tau.reshape((3, b["nax"], nsp), order="F"),
                 ctrl=dict(nx=int(iv[0]), nempty=int(iv[1]), degree=int(iv[2]),
                           max_scf_iter=int(iv[3]), imix=int(iv[4]), mixdim=int(iv[5]),
                           idiag=int(iv[6]), user_max_diag_iter=int(iv[7]),
                           max_diag_iter=int(iv[8]), conv=dv[0], rho_mix_fac=dv[1],
                           kerker_q0=dv[2]))
        return b

    def program_cheby_scf(self, workdir):
        """ChebySCFLoop() after ``program_setup`` with rand() seeded by
        srand(1); returns (EIG[:NX], {ETOT, EKIN, EHT, EPSEU, ENL, EXC})."""
        nx = self.cell["nx"]
        eig, e6 = np.zeros(nx), np.zeros(6)
        cwd = os.getcwd()
        os.chdir(workdir)
        try:
            self.lib.ref_prog_cheby_scf(eig, e6)
        finally:
            os.chdir(cwd)
        return eig, e6

    def set_nl(self, pkg_a, wnl):
        self.lib.ref_set_nl(np.ascontiguousarray(np.asarray(pkg_a).reshape(-1, order="F")),
                            np.ascontiguousarray(np.asarray(wnl).reshape(-1, order="F")))

    # ------------------------------------------------------------ calls
    @staticmethod
    def _fz(a):
        # always a private copy: the reference works in place on its arguments
        return np.array(np.asarray(a, dtype=complex).reshape(-1, order="F"), copy=True)

    def apply_ham_block(self, vin, veff):
        ngw, nb = vin.shape
        x = self._fz(vin)
        y = np.zeros_like(x)
        self.lib.ref_ApplyHam_block(x, y, ngw, np.ascontiguousarray(veff, dtype=float), nb)
        return y.reshape((ngw, nb), order="F")

    def apply_ham(self, v, veff):
        x = np.ascontiguousarray(v, dtype=complex)
        y = np.zeros_like(x)
        self.lib.ref_ApplyHam(x, y, x.size, np.ascontiguousarray(veff, dtype=float))
        return y

    def chebyfilt(self, X, degree, lb, ub, veff):
        ngw, nb = X.shape
        x = self._fz(X)
        self.lib.ref_chebyfilt(x, degree, lb, ub, np.ascontiguousarray(veff, dtype=float))
        return x.reshape((ngw, nb), order="F")

    def lanczos(self, v0, k, veff):
        v = np.ascontiguousarray(v0, dtype=complex).copy()
        T = np.zeros(k * k)
        f = np.zeros_like(v)
        self.lib.ref_lanczos(v, k, T, k, f, np.ascontiguousarray(veff, dtype=float))
        return T.reshape((k, k), order="F"), f

    def ortho_qr(self, X):
        m, n = X.shape
        x = self._fz(X)
        self.lib.ref_ortho_qr(x, m, n)
        return x.reshape((m, n), order="F")

    def eig_zheevd(self, A):
        n = A.shape[0]
        a = self._fz(A)
        w = np.zeros(n)
        self.lib.ref_eig_zheevd(a, n, w, n)
        return w, a.reshape((n, n), order="F")

    def eig_zhegv_eval(self, A, B):
        n = A.shape[0]
        a, b = self._fz(A), self._fz(B)
        w = np.zeros(n)
        e = np.zeros(n * n, dtype=complex)
        self.lib.ref_eig_zhegv_eval(a, n, b, n, w, e, n, n)
        return w, e.reshape((n, n), order="F")

    def gen_prec(self, nbasis, tau):
        p = np.zeros(nbasis)
        self.lib.ref_GenPrec(p, nbasis, tau)
        return p

    def random_col(self, nelem, seed):
        a = np.zeros(nelem, dtype=complex)
        self.lib.ref_random_col(a, nelem, seed)
        return a

    def davidson(self, nbasis, nstates, veff, prec, nempty, max_iter=None):
        self.lib.ref_set_nx(self.cell["nx"], nempty)
        self.lib.ref_set_diag(1 if max_iter else 0, max_iter or 0, 0)
        ev = np.zeros(nstates)
        x = np.zeros(nbasis * nstates, dtype=complex)
        self.lib.ref_davidson(ev, x, nbasis, nstates, np.ascontiguousarray(veff, dtype=float),
                              np.ascontiguousarray(prec, dtype=float))
        return ev, x.reshape((nbasis, nstates), order="F")

    def lobpcg(self, nbasis, nstates, veff, prec, nempty, max_iter=None):
        self.lib.ref_set_nx(self.cell["nx"], nempty)
        self.lib.ref_set_diag(1 if max_iter else 0, max_iter or 0, 0)
        ev = np.zeros(nstates)
        x = np.zeros(nbasis * nstates, dtype=complex)
        self.lib.ref_lobpcg(ev, x, nbasis, nstates, np.ascontiguousarray(veff, dtype=float),
                            np.ascontiguousarray(prec, dtype=float))
        return ev, x.reshape((nbasis, nstates), order="F")

    def set_nx(self, nx, nempty):
        self.lib.ref_set_nx(nx, nempty)
        self.cell["nx"] = nx

    # ---- SCF pieces (EvalEnergy.cpp, xc_PZ.cpp, NormalizeRho.cpp, the mixers)
    def set_local(self, sfac, vps, rhops, esr, eself, nel):
        """sfac, vps, rhops: (NG, NSP) arrays (species fastest in memory)."""
        self.lib.ref_set_local(np.ascontiguousarray(sfac, dtype=complex),
                               np.ascontiguousarray(vps, dtype=float),
                               np.ascontiguousarray(rhops, dtype=float), esr, eself, nel)

    def eval_energy(self, rho, ekin, enl):
        r = np.array(rho, dtype=float, copy=True)
        e = np.zeros(6)
        self.lib.ref_EvalEnergy(r, ekin, enl, e)
        return r, dict(zip(("ETOT", "EKIN", "EHT", "EPSEU", "ENL", "EXC"), e.tolist()))

    def xc_pz(self, rho):
        r = np.array(rho, dtype=float, copy=True)
        v = np.zeros_like(r)
        exc = self.lib.ref_xc_PZ(r, v, len(r))
        return v, exc

    def normalize_rho(self, rho, omega, nel):
        r = np.array(rho, dtype=float, copy=True)
        self.lib.ref_NormalizeRho(r, len(r), omega, nel)
        return r

    def kerker_prec(self, x, beta, q0):
        r = np.array(x, dtype=float, copy=True)
        self.lib.ref_KerkerPrec(r, 1, len(r), beta, q0)
        return r

    def eval_enl(self):
        """EvalENL() on the C0 / FOCC the last eval_rho_psi left; returns ENL."""
        self.lib.ref_EvalENL()
        return self.lib.ref_get_enl()

    def eval_rho_psi(self, eigvec_flat, ld, ngw, nx, focc):
        """Returns (rho increment, EKIN increment, C0)."""
        self.set_nx(nx, 0)
        self.lib.ref_set_focc(np.ascontiguousarray(focc, dtype=float), nx)
        self.lib.ref_alloc_c0()
        self.lib.ref_set_ekin(0.0)
        rho = np.zeros(self.cell["nnr"])
        self.lib.ref_EvalRhoPsi(rho, np.ascontiguousarray(eigvec_flat, dtype=complex), ld, ngw)
        c0 = np.zeros(self.cell["ngwx"] * nx, dtype=complex)
        self.lib.ref_get_c0(c0)
        return rho, self.lib.ref_get_ekin(), c0.reshape((self.cell["ngwx"], nx), order="F")
