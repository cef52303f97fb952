"""SCF serving: synthetic cluster jobs, a seeded Poisson arrival schedule and
the device server of the C ABI (pspw_server_*: continuous batching of
independent ChebySCF jobs on one GPU, admitted by HBM footprint).

A job is a directory with an INPUT and FHI98 pseudopotential files in the
reference's formats: an isolated cluster of atoms of up to four species in a
cubic box, each species a synthetic local + s/p KB pseudopotential with an
attractive Gaussian well, four valence electrons per atom and
ceil(0.6 * valence electrons) + 8 states.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from ._lib import PREC_F64, check, lib
from .inputs import write_input_species, write_synthetic_fhi


class ServerConfig(C.Structure):
    _fields_ = [("slots", C.c_int), ("hbm_budget_bytes", C.c_double),
                ("filter_prec", C.c_int), ("conv_per_atom", C.c_double),
                ("max_scf_iter", C.c_int), ("pulay_beta", C.c_double), ("mixdim", C.c_int)]


class JobResult(C.Structure):
    _fields_ = [("id", C.c_int), ("status", C.c_int), ("natoms", C.c_int), ("nbands", C.c_int),
                ("ngw", C.c_int), ("nnr", C.c_int), ("iterations", C.c_int),
                ("converged", C.c_int), ("etot", C.c_double), ("footprint_bytes", C.c_double),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_scf", C.c_double),
                ("t_done", C.c_double), ("error", C.c_char * 160)]


class Server:
    """pspw_server on GPU `device`: `slots` concurrent SCF jobs."""

    def __init__(self, device=0, slots=4, hbm_budget_bytes=0.0, filter_prec=PREC_F64,
                 conv_per_atom=1e-6, max_scf_iter=100, pulay_beta=0.3, mixdim=6):
        cfg = ServerConfig(int(slots), float(hbm_budget_bytes), int(filter_prec),
                           float(conv_per_atom), int(max_scf_iter), float(pulay_beta),
                           int(mixdim))
        self._h = C.c_void_p()
        check(lib().pspw_server_create(int(device), C.byref(cfg), C.byref(self._h)))

    def submit(self, directory):
        jid = C.c_int()
        check(lib().pspw_server_submit(self._h, str(directory).encode(), C.byref(jid)))
        return jid.value

    def wait(self, job_id, neig=0):
        r = JobResult()
        eig = np.zeros(max(1, neig))
        check(lib().pspw_server_wait(self._h, int(job_id), C.byref(r), eig.ctypes.data,
                                     int(neig)))
        out = {name: getattr(r, name) for name, _ in JobResult._fields_}
        out["error"] = r.error.decode(errors="replace")
        if neig:
            out["eig"] = eig[:neig]
        return out

    def now(self):
        t = C.c_double()
        check(lib().pspw_server_now(self._h, C.byref(t)))
        return t.value

    def close(self):
        if self._h:
            lib().pspw_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def smooth_grid(n, lo=24, hi=128):
    """Smallest 2,3,5-smooth length >= n, clipped to [lo, hi]."""
    m = max(int(math.ceil(n)), lo)
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1 or m >= hi:
            return min(m, hi) if k == 1 else hi
        m += 1


def species_set(rng, nsp=4):
    """(depth Ha, width bohr) of the synthetic Gaussian wells."""
    return [(float(rng.uniform(1.0, 4.0)), float(rng.uniform(0.8, 1.6))) for _ in range(nsp)]


def cluster_job(rng, directory, species, natoms=None, ecut_ha=None, box=None, min_sep=2.2,
                vacuum=6.0, natoms_range=(2, 64), ecut_range=(12.0, 25.0), box_max=24.0,
                ekt=None, imix=3):
    """Write one cluster job into `directory`; returns its description.
    Atoms are placed uniformly (rejection sampling, pairwise distance >=
    min_sep) in the central cube of the box, leaving `vacuum` bohr between
    periodic images; the FFT grid is the smallest 5-smooth length above
    2 G_max L / 2 pi + 1 for ecutrho = 4 ecutwfc, kept within 24..128 (the
    ranges above need at most 120, so the density sphere always fits the
    grid: a smaller grid would alias it).
    ekt (eV): Fermi-Dirac occupations at that temperature (INPUT `tmetal`,
    `ekt`); None keeps the reference's fixed occupations.  imix: the INPUT's
    mixer (3 Pulay, 4 Broyden, ...)."""
    os.makedirs(directory, exist_ok=True)
    nat = int(natoms if natoms is not None else rng.integers(natoms_range[0], natoms_range[1] + 1))
    lo = max(10.0, vacuum + (nat * 12.0) ** (1.0 / 3.0))
    L = float(box if box is not None else rng.uniform(lo, max(lo, box_max)))
    ec = float(ecut_ha if ecut_ha is not None else rng.uniform(*ecut_range))
    inner = L - vacuum
    pos = []
    tries = 0
    while len(pos) < nat:
        p = (L - inner) / 2 + rng.uniform(0.0, inner, 3)
        if all(np.linalg.norm(p - q) >= min_sep for q in pos):
            pos.append(p)
        tries += 1
        if tries > 200000:
            raise RuntimeError("cluster_job: cannot place the atoms; enlarge the box")
    kinds = rng.integers(0, len(species), nat)
    groups = []
    for s, (depth, width) in enumerate(species):
        sel = [pos[i] for i in range(nat) if kinds[i] == s]
        if sel:
            name = f"S{s}.fhi"
            write_synthetic_fhi(os.path.join(directory, name), zv=4.0, well=-depth, width=width)
            groups.append((name, np.array(sel)))
    gmax = math.sqrt(2.0 * 4.0 * ec)
    n = smooth_grid(2.0 * gmax * L / (2.0 * math.pi) + 1.0)
    nval = 4 * nat
    nx = int(math.ceil(0.6 * nval)) + 8
    nempty = nx - (nval + 1) // 2
    write_input_species(os.path.join(directory, "INPUT"), groups, L, 2.0 * ec, nempty,
                        fft_grid=(n, n, n), imix=imix, idiag=-1, max_scf=100, conv=1e-6 * nat,
                        ekt=ekt)
    return {"dir": directory, "natoms": nat, "box": L, "ecut_ha": ec, "grid": n, "nx": nx,
            "species": [int(k) for k in kinds]}


def poisson_arrivals(rng, rate, n):
    """Arrival times (s) of n jobs of a Poisson process of `rate` jobs/s."""
    return np.cumsum(rng.exponential(1.0 / rate, n))


def percentile(values, q):
    v = np.sort(np.asarray(values, dtype=float))
    if not len(v):
        return None
    return float(np.percentile(v, q, method="linear"))
