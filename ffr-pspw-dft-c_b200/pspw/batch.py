"""Batched block H*psi over many independent cells in one graph launch
(pspw_batch_*), and the uneven synthetic cells it is measured on:
orthorhombic cells with lattice constants uniform in 8-16 bohr, 2-16 atoms
at least 3 bohr apart (minimum image), ecutwfc uniform in 10-25 Ha with the
smallest 5-smooth grid above 2 G_max L / 2 pi + 1 for ecutrho = 4 ecutwfc
on each axis (clipped to 24..72), and 8-256 bands; potentials and
wavefunctions as the Si workloads (pspw.synth)."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import synth
from ._lib import PREC_F32, PREC_F64, check, lib
from .cell import Cell, basis_gamma
from .serve import smooth_grid


def ortho_cell(rng, nat_range=(2, 16), lat_range=(8.0, 16.0), ecut_range=(10.0, 25.0),
               band_range=(8, 256), min_sep=3.0):
    abc = rng.uniform(*lat_range, 3)
    lat = np.diag(abc)
    nat = int(rng.integers(nat_range[0], nat_range[1] + 1))
    pos = []
    while len(pos) < nat:
        p = rng.uniform(0.0, 1.0, 3) * abc
        ok = True
        for q in pos:
            d = p - q
            d -= np.round(d / abc) * abc  # minimum image
            if np.linalg.norm(d) < min_sep:
                ok = False
                break
        if ok:
            pos.append(p)
    pos = np.array(pos)
    ec = float(rng.uniform(*ecut_range))
    gmax = math.sqrt(8.0 * ec)
    nr = tuple(smooth_grid(2.0 * gmax * L / (2.0 * math.pi) + 1.0) for L in abc)
    b = basis_gamma(lat, 2.0 * ec, nr, [nat], [pos])
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=[4], lattice=lat, positions=pos)
    b["veff"] = synth.local_potential(b["nr"], lat, pos)
    nb = int(rng.integers(band_range[0], band_range[1] + 1))
    b["nbands"] = min(nb, b["ngw"])
    b["psi"] = synth.wavefunctions(b, lat, b["nbands"], int(rng.integers(1 << 30)))
    b["ecut_ha"] = ec
    return b


class Batch:
    """pspw_batch over Cell objects (kept alive by the batch)."""

    def __init__(self, cells, nbands, prec=PREC_F32):
        self.cells = list(cells)
        self.nbands = [int(n) for n in nbands]
        self.prec = prec
        arr = (C.c_void_p * len(self.cells))(*[c.handle.value for c in self.cells])
        nb = np.ascontiguousarray(self.nbands, dtype=np.int32)
        self._h = C.c_void_p()
        check(lib().pspw_batch_create(len(self.cells), arr, nb.ctypes.data, int(prec),
                                      C.byref(self._h)))

    @property
    def dtype(self):
        return np.complex128 if self.prec == PREC_F64 else np.complex64

    def upload(self, i, psi):
        a = np.asfortranarray(np.asarray(psi, dtype=self.dtype))
        check(lib().pspw_batch_upload(self._h, int(i), a.ctypes.data))

    def download(self, i):
        out = np.zeros((self.cells[i].ngw, self.nbands[i]), dtype=self.dtype, order="F")
        check(lib().pspw_batch_download(self._h, int(i), out.ctypes.data))
        return out

    def tune(self, reps=3):
        check(lib().pspw_batch_tune(self._h, int(reps)))

    def schedule(self, i):
        bb, path, ms = C.c_int(), C.c_int(), C.c_double()
        check(lib().pspw_batch_schedule(self._h, int(i), C.byref(bb), C.byref(path),
                                        C.byref(ms)))
        return {"band_batch": bb.value, "nl_path": path.value, "ms": ms.value}

    def apply(self):
        check(lib().pspw_batch_apply(self._h))

    def kernels(self):
        """Kernel launches one apply replays."""
        n = C.c_longlong()
        check(lib().pspw_batch_kernels(self._h, C.byref(n)))
        return n.value

    def stream(self):
        s = C.c_void_p()
        check(lib().pspw_batch_stream(self._h, C.byref(s)))
        return s.value

    def synchronize(self):
        check(lib().pspw_batch_synchronize(self._h))

    def close(self):
        if self._h:
            lib().pspw_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Batch", "ortho_cell", "PREC_F32", "PREC_F64", "Cell"]
