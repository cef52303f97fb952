"""Host-side handles over the C ABI: basis generation and the device cell.

``Cell`` mirrors the reference's device API (SetupArrays_ApplyHam_cuda /
CopyRho_ApplyHam_cuda / ApplyHam_block_cuda, common_pspw.h:252-259) with an
explicit handle; arrays use the reference's Fortran layouts.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import PREC_F32, PREC_F64, BasisInfo, check, lib, ptr


def _f(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def _flat(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype).reshape(-1, order="F"))


def basis_gamma(lattice, ecut_ry, nr=None, na=(), tau=()):
    """The reference's Gamma-point basis (Setup/GVectorsGen/GkVectorsGen/
    PhaseFactor) for lattice rows A1, A2, A3 in bohr and ECUT in Rydberg.
    tau: list per species of (na, 3) positions in bohr."""
    L = lib()
    lat = np.ascontiguousarray(np.asarray(lattice, dtype=float).reshape(9))
    nrf = np.asarray(nr if nr is not None else (0, 0, 0), dtype=np.int32)
    info = BasisInfo()
    check(L.pspw_basis_info_gamma(lat.ctypes.data, float(ecut_ry), nrf.ctypes.data, C.byref(info)))
    ngwx, ngx = info.ngwx, info.ngx
    nsp = max(1, len(na))
    na_arr = np.asarray(list(na) if len(na) else [0], dtype=np.int32)
    nax = int(max(1, na_arr.max()))
    taua = np.zeros((nsp, nax, 3))
    for s in range(len(na)):
        taua[s, : na[s]] = np.asarray(tau[s], dtype=float).reshape(na[s], 3)
    out = dict(n123=np.zeros(ngwx, np.uint32), xkg=np.zeros(ngwx), igk=np.zeros(ngwx, np.int32),
               N1=np.zeros(ngx, np.int32), N2=np.zeros(ngx, np.int32), N3=np.zeros(ngx, np.int32),
               IN1=np.zeros(ngx, np.int32), IN2=np.zeros(ngx, np.int32),
               IN3=np.zeros(ngx, np.int32), G=np.zeros(ngx), GG=np.zeros((ngx + 1) * 3),
               eigr=np.zeros(2 * ngwx * nax * nsp))
    check(L.pspw_basis_build_gamma(
        lat.ctypes.data, float(ecut_ry), nrf.ctypes.data, nsp, na_arr.ctypes.data,
        np.ascontiguousarray(taua.reshape(-1)).ctypes.data, C.byref(info),
        *(out[k].ctypes.data for k in ("n123", "xkg", "igk", "N1", "N2", "N3", "IN1", "IN2", "IN3",
                                       "G", "GG", "eigr"))))
    out["eigr"] = out["eigr"].view(np.complex128).reshape((ngwx, nax, nsp), order="F")
    out.update(nr=tuple(info.nr), ngw=info.ngw, ngwx=ngwx, ngx=ngx, ng=info.ng, alat=info.alat,
               omega=info.omega, tpiba=info.tpiba, tpiba2=info.tpiba2, gcut=info.gcut,
               gcutw=info.gcutw, nax=nax, nsp=nsp, na=list(na))
    return out


class Cell:
    """One geometry/k-point on one GPU (pspw_cell)."""

    def __init__(self, nr, ngw, ngwx, n123, xkg, tpiba2, na, lm_end, eigr, pkg_a, wnl, device=0):
        L = lib()
        self._h = C.c_void_p()
        nsp = len(na)
        nax = int(max(na)) if nsp else 0
        nlmax = int(np.asarray(pkg_a).shape[0]) if nsp else 4
        self._keep = dict(
            n123=np.ascontiguousarray(np.asarray(n123, dtype=np.uint32)),
            xkg=np.ascontiguousarray(np.asarray(xkg, dtype=float)),
            na=np.asarray(na, dtype=np.int32), lm_end=np.asarray(lm_end, dtype=np.int32),
            eigr=_flat(eigr, np.complex128).view(np.float64), pkg_a=_flat(pkg_a, float),
            wnl=_flat(wnl, float))
        k = self._keep
        check(L.pspw_cell_create(C.byref(self._h), int(device), int(nr[0]), int(nr[1]), int(nr[2]),
                                 int(ngw), int(ngwx), k["n123"].ctypes.data, k["xkg"].ctypes.data,
                                 float(tpiba2), nsp, k["na"].ctypes.data, nax,
                                 k["lm_end"].ctypes.data, nlmax, k["eigr"].ctypes.data,
                                 k["pkg_a"].ctypes.data, k["wnl"].ctypes.data))
        self.nr = tuple(int(x) for x in nr)
        self.nnr = self.nr[0] * self.nr[1] * self.nr[2]
        self.ngw = int(ngw)
        self.device = device

    @classmethod
    def from_arrays(cls, cell, device=0):
        """From a dict with keys nr, ngw, ngwx, n123, xkg, tpiba2, na, lm_end,
        eigr, pkg_a, wnl (the reference's arrays)."""
        return cls(cell["nr"], cell["ngw"], cell["ngwx"], cell["n123"], cell["xkg"],
                   cell["tpiba2"], cell["na"], cell["lm_end"], cell["eigr"], cell["pkg_a"],
                   cell["wnl"], device=device)

    @classmethod
    def borrow(cls, handle, nr, ngw, device=0, owner=None):
        """A view of a cell owned elsewhere (e.g. by a System): closing it
        does not destroy the handle; `owner` is kept alive."""
        c = cls.__new__(cls)
        c._h = handle
        c._owned = False
        c._owner = owner
        c.nr = tuple(int(x) for x in nr)
        c.nnr = c.nr[0] * c.nr[1] * c.nr[2]
        c.ngw = int(ngw)
        c.device = device
        return c

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h and getattr(self, "_owned", True):
            lib().pspw_cell_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sizes(self):
        o = np.zeros(8, dtype=np.int32)
        check(lib().pspw_cell_sizes(self._h, o.ctypes.data))
        return dict(zip(("n1", "n2", "n3", "ngw", "nsticks", "nxa", "nat", "nproj"), o.tolist()))

    def stream(self):
        s = C.c_void_p()
        check(lib().pspw_cell_get_stream(self._h, C.byref(s)))
        return s.value

    def set_veff(self, veff):
        v = np.ascontiguousarray(np.asarray(veff, dtype=float).reshape(-1))
        check(lib().pspw_cell_set_veff(self._h, v.ctypes.data, v.size))

    def set_band_batch(self, n):
        check(lib().pspw_cell_set_band_batch(self._h, int(n)))

    def set_nl_path(self, path):
        """NL_AUTO / NL_SIMT / NL_TENSOR_CORE kernels for the FP32 projector GEMMs."""
        check(lib().pspw_cell_set_nl_path(self._h, int(path)))

    def set_nl_overlap(self, mode):
        """OVERLAP_AUTO / OVERLAP_ON / OVERLAP_OFF: the projection of H*psi
        concurrent with the FFT passes or after them (same results)."""
        check(lib().pspw_cell_set_nl_overlap(self._h, int(mode)))

    def check_device_wait(self, complete):
        """One bounded device-side barrier wait (the tensor-core kernels'
        kind); raises PspwError(TIMEOUT) when nothing completes it."""
        check(lib().pspw_cell_check_device_wait(self._h, int(complete)))

    # ---- host FP64 (the reference signatures' data)
    def apply_ham_block(self, vin):
        vin = _f(vin, np.complex128)
        if vin.ndim == 1:
            vin = vin[:, None]
        ngw, nb = vin.shape
        out = np.zeros((ngw, nb), dtype=np.complex128, order="F")
        check(lib().pspw_apply_ham_block(self._h, vin.ctypes.data, out.ctypes.data, ngw, nb))
        return out

    def chebyfilt(self, X, degree, lb, ub, prec=PREC_F64):
        X = np.array(_f(X, np.complex128), order="F", copy=True)
        ngw, nb = X.shape
        check(lib().pspw_chebyfilt(self._h, X.ctypes.data, ngw, nb, int(degree), float(lb),
                                   float(ub), int(prec)))
        return X

    # ---- device buffers (torch tensors), enqueued on the cell stream
    def apply_ham_block_dev(self, d_in, d_out, ld, ngw, nb, prec):
        check(lib().pspw_apply_ham_block_dev(self._h, int(prec), ptr(d_in), ptr(d_out), int(ld),
                                             int(ngw), int(nb)))

    def chebyfilt_dev(self, d_x, ld, ngw, nb, degree, lb, ub, prec):
        check(lib().pspw_chebyfilt_dev(self._h, int(prec), ptr(d_x), int(ld), int(ngw), int(nb),
                                       int(degree), float(lb), float(ub)))

    def zgemm_dev(self, opa, m, n, k, alpha, d_a, lda, d_b, ldb, beta, d_c, ldc):
        """C = alpha op(A) B + beta C on device FP64 complex matrices
        (column-major; op 'N' or 'C'), enqueued on the cell stream."""
        al = np.array([complex(alpha).real, complex(alpha).imag])
        be = np.array([complex(beta).real, complex(beta).imag])
        check(lib().pspw_zgemm_dev(self._h, opa.encode() if isinstance(opa, str) else opa,
                                   int(m), int(n), int(k), al.ctypes.data, ptr(d_a), int(lda),
                                   ptr(d_b), int(ldb), be.ctypes.data, ptr(d_c), int(ldc)))

    def eig_zheevd_dev(self, d_a, lda, d_w, n):
        """eig_zheevd on device pointers (upper triangle read; eigenvectors
        into A, ascending eigenvalues into w), enqueued on the cell stream."""
        check(lib().pspw_eig_zheevd_dev(self._h, ptr(d_a), int(lda), ptr(d_w), int(n)))

    def ortho_span_dev(self, d_x, ngw, n):
        """Orthonormal basis of span(X) in place (device, ld ngw): the SCF
        loop's CholeskyQR2 step."""
        check(lib().pspw_ortho_span_dev(self._h, ptr(d_x), int(ngw), int(n)))

    # ---- solvers and dense steps (host buffers; reference semantics)
    def gen_prec(self, nbasis, tau):
        p = np.zeros(nbasis)
        check(lib().pspw_gen_prec(self._h, p.ctypes.data, int(nbasis), float(tau)))
        return p

    def ortho_qr(self, X):
        X = np.array(_f(X, np.complex128), order="F", copy=True)
        check(lib().pspw_ortho_qr(self._h, X.ctypes.data, X.shape[0], X.shape[1]))
        return X

    def eig_zheevd(self, A):
        A = np.array(_f(A, np.complex128), order="F", copy=True)
        n = A.shape[0]
        w = np.zeros(n)
        check(lib().pspw_eig_zheevd(self._h, A.ctypes.data, n, w.ctypes.data, n))
        return w, A

    def eig_zhegv_eval(self, A, B):
        A = np.array(_f(A, np.complex128), order="F", copy=True)
        B = np.array(_f(B, np.complex128), order="F", copy=True)
        n = A.shape[0]
        w = np.zeros(n)
        E = np.zeros((n, n), dtype=np.complex128, order="F")
        check(lib().pspw_eig_zhegv_eval(self._h, A.ctypes.data, n, B.ctypes.data, n, w.ctypes.data,
                                        E.ctypes.data, n, n))
        return w, E

    def _solver(self, name, nbasis, nstates, prec, nempty, max_iter, hprec, X0=None):
        if X0 is None:
            X = np.zeros((nbasis, nstates), dtype=np.complex128, order="F")
        else:
            X = np.array(np.asarray(X0, dtype=np.complex128)[:nbasis, :nstates], order="F")
        ev = np.zeros(nstates)
        res = np.zeros(nstates)
        it = C.c_int()
        p = np.ascontiguousarray(np.asarray(prec, dtype=float)[:nbasis])
        check(getattr(lib(), name)(self._h, ev.ctypes.data, X.ctypes.data, int(nbasis),
                                   int(nstates), p.ctypes.data, int(nempty), int(max_iter or 0),
                                   int(hprec), res.ctypes.data, C.byref(it)))
        return ev, X, res, it.value

    def davidson(self, nbasis, nstates, prec, nempty, max_iter=None, hprec=PREC_F64):
        return self._solver("pspw_davidson", nbasis, nstates, prec, nempty, max_iter, hprec)

    def lobpcg(self, nbasis, nstates, prec, nempty, max_iter=None, hprec=PREC_F64):
        return self._solver("pspw_lobpcg", nbasis, nstates, prec, nempty, max_iter, hprec)

    def lobpcg_ortho(self, nbasis, nstates, prec, nempty, max_iter=None, hprec=PREC_F64,
                     X0=None):
        """LOBPCG with an orthonormal [X W P] basis (opt-in, see pspw_gpu.h),
        from the reference's random start, or from the block X0
        (nbasis x nstates) when given."""
        if X0 is None:
            return self._solver("pspw_lobpcg_ortho", nbasis, nstates, prec, nempty, max_iter,
                                hprec)
        return self._solver("pspw_lobpcg_ortho_from", nbasis, nstates, prec, nempty, max_iter,
                            hprec, X0)

    def lanczos(self, v0, k):
        v = np.array(np.asarray(v0, dtype=np.complex128), copy=True)
        T = np.zeros((k, k), order="F")
        f = np.zeros_like(v)
        check(lib().pspw_lanczos(self._h, v.ctypes.data, v.size, int(k), T.ctypes.data, int(k),
                                 f.ctypes.data))
        return T, f, v

    def eval_rho_psi(self, rhoe, eigvec_flat, ld, ngw, nx, focc, wkpt, omega, ekin=0.0):
        rho = np.array(np.asarray(rhoe, dtype=float), copy=True)
        ev = np.ascontiguousarray(np.asarray(eigvec_flat, dtype=np.complex128))
        fo = np.ascontiguousarray(np.asarray(focc, dtype=float))
        ek = C.c_double(ekin)
        check(lib().pspw_eval_rho_psi(self._h, rho.ctypes.data, ev.ctypes.data, int(ld), int(ngw),
                                      int(nx), fo.ctypes.data, float(wkpt), float(omega),
                                      C.byref(ek)))
        return rho, ek.value

    def eval_enl(self, c0, nx, focc, wkpt):
        """EvalENL for one k-point: (ENL, FNL[nx, nproj]) from C0 (ngw x >= nx)."""
        a = np.asfortranarray(np.asarray(c0, dtype=np.complex128))
        ngw = a.shape[0]
        fo = np.ascontiguousarray(np.asarray(focc, dtype=float))
        nproj = self.sizes()["nproj"]
        fnl = np.zeros((nx, max(1, nproj)), dtype=np.complex128, order="F")
        e = C.c_double(0.0)
        check(lib().pspw_eval_enl(self._h, a.ctypes.data, ngw, ngw, int(nx), fo.ctypes.data,
                                  float(wkpt), C.byref(e), fnl.ctypes.data))
        return e.value, fnl[:, :nproj]

    # ---- timing
    def timing_enable(self, mask):
        check(lib().pspw_timing_enable(self._h, int(mask)))

    def timing_read(self, family):
        ms = C.c_double()
        n = C.c_longlong()
        check(lib().pspw_timing_read(self._h, int(family), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def timing_reset(self):
        check(lib().pspw_timing_reset(self._h))

    def kernel_launches(self):
        n = C.c_longlong()
        check(lib().pspw_kernel_launches(self._h, C.byref(n)))
        return n.value


def random_col(nelem, seed):
    """util_random_cpu.cpp:5-23 start vector (bit-exact)."""
    a = np.zeros(nelem, dtype=np.complex128)
    check(lib().pspw_random_col(a.ctypes.data, int(nelem), int(seed)))
    return a


__all__ = ["Cell", "basis_gamma", "random_col", "PREC_F32", "PREC_F64"]
