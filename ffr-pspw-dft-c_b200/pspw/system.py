"""A system set up from the reference's own input files (pspw_system_*): the
INPUT keyword file and FHI98 pseudopotentials read the way ReadInputFile.cpp
and ReadPseudopotentials.cpp read them, the set-up of Setup.cpp and
PrepareSCF.cpp with its heavy arrays built on the device, and the ChebySCF
loop of the reference's main program on it."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import PREC_F64, check, lib
from .cell import Cell
from .scf import Scf, ScfParams

_DIMS = ("nr1", "nr2", "nr3", "nnr", "ngw", "ngwx", "ng", "ngx", "nx", "nlmax", "nax", "nsp",
         "nempty", "iscf", "nkpt", "idiag")
_SCAL = ("tpiba", "tpiba2", "omega", "alat", "gcut", "gcutw", "nel", "esr", "eself", "ecut",
         "wkpt")
# name -> (PSPW_SYS_* id, dtype, shape from dims, Fortran order)
_ARRAYS = {
    "eigr": (0, np.complex128, lambda d: (d["ngwx"], d["nax"], d["nsp"])),
    "sfac": (1, np.complex128, lambda d: (d["nsp"], d["ng"])),
    "vps": (2, np.float64, lambda d: (d["nsp"], d["ng"])),
    "rhops": (3, np.float64, lambda d: (d["nsp"], d["ng"])),
    "pkg_a": (4, np.float64, lambda d: (d["nlmax"], d["ngwx"], d["nsp"])),
    "rho_start": (5, np.float64, lambda d: (d["nnr"],)),
    "wnl": (6, np.float64, lambda d: (d["nsp"], d["nlmax"])),
    "focc": (7, np.float64, lambda d: (d["nx"],)),
    "n123": (8, np.uint32, lambda d: (d["ngwx"],)),
    "xkg": (9, np.float64, lambda d: (d["ngwx"],)),
    "tau": (10, np.float64, lambda d: (3, d["nax"], d["nsp"])),
    "g": (11, np.float64, lambda d: (d["ng"],)),
}
_TIMES = ("host_input_basis", "phase_structure", "local_ff", "nonlocal_ff", "cell_scf",
          "start_density", "ewald", "total")


class System:
    """pspw_system: INPUT in `directory` read and set up on GPU `device`."""

    def __init__(self, directory, device=0):
        self._h = C.c_void_p()
        check(lib().pspw_system_load(str(directory).encode(), int(device), C.byref(self._h)))
        self.device = device
        d = np.zeros(16, dtype=np.int32)
        v = np.zeros(16)
        check(lib().pspw_system_info(self._h, d.ctypes.data, v.ctypes.data))
        self.dims = {k: int(x) for k, x in zip(_DIMS, d)}
        self.scalars = {k: float(x) for k, x in zip(_SCAL, v)}
        self.dims["nr"] = (self.dims["nr1"], self.dims["nr2"], self.dims["nr3"])

    def close(self):
        if self._h:
            lib().pspw_system_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        p = ScfParams()
        check(lib().pspw_system_params(self._h, C.byref(p)))
        return {name: getattr(p, name) for name, _ in ScfParams._fields_}

    def array(self, name):
        which, dtype, shape = _ARRAYS[name]
        shp = shape(self.dims)
        out = np.zeros(int(np.prod(shp)), dtype=dtype)
        check(lib().pspw_system_array(self._h, which, out.ctypes.data, out.nbytes))
        return out.reshape(shp, order="F")

    def cell(self):
        h = C.c_void_p()
        check(lib().pspw_system_cell(self._h, C.byref(h)))
        return Cell.borrow(h, self.dims["nr"], self.dims["ngw"], self.device, owner=self)

    def scf(self):
        h = C.c_void_p()
        check(lib().pspw_system_scf(self._h, C.byref(h)))
        return Scf.borrow(h, self.cell(), owner=self)

    def timing(self):
        t = np.zeros(8)
        check(lib().pspw_system_timing(self._h, t.ctypes.data))
        return dict(zip(_TIMES, t.tolist()))

    def cheby_scf(self, filter_prec=PREC_F64, outdir=None, **controls):
        """ChebySCFLoop() of the reference's main program on this system.
        `controls` override the INPUT's SCF controls (pspw_scf_params
        fields, e.g. pulay_beta=0.3, mixdim=6, conv=1e-8, max_scf_iter=200).
        Returns eig (NX), energies, iterations, converged and hist
        (iterations x {ETOT, |dETOT|, d, ms since the call began})."""
        nx = self.dims["nx"]
        eig, e6 = np.zeros(nx), np.zeros(6)
        its, cv = C.c_int(0), C.c_int(0)
        p = self.params()
        p.update(controls, filter_prec=int(filter_prec))
        hist = np.zeros(4 * max(1, p["max_scf_iter"]))
        sp = ScfParams(**p)
        check(lib().pspw_system_cheby_scf_with(self._h, C.byref(sp),
                                               None if outdir is None else str(outdir).encode(),
                                               eig.ctypes.data, e6.ctypes.data, C.byref(its),
                                               C.byref(cv), hist.ctypes.data))
        n = its.value
        return dict(eig=eig, iterations=n, converged=bool(cv.value),
                    hist=hist.reshape(-1, 4)[:n],
                    energies=dict(zip(("ETOT", "EKIN", "EHT", "EPSEU", "ENL", "EXC"),
                                      e6.tolist())))


def print_3d_array(a, nr, path):
    """Print3DArray.cpp: one `%18.10f` value per line."""
    x = np.ascontiguousarray(np.asarray(a, dtype=float).reshape(-1))
    check(lib().pspw_print_3d_array(x.ctypes.data, int(nr[0]), int(nr[1]), int(nr[2]),
                                    str(path).encode()))
