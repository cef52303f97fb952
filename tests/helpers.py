"""Shared test helpers: golden fixtures, oracle cells and error norms; the
input-file writers live in the package (pspw.inputs)."""
from __future__ import annotations

import os

import numpy as np

from pspw.inputs import write_input, write_synthetic_fhi  # noqa: F401

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


def scf_lines(log):
    """The `! iter ETOT dETOT drho` lines of a reference log."""
    out = []
    for line in log.splitlines():
        parts = line.split()
        if len(parts) == 5 and parts[0] == "!":
            out.append((int(parts[1]), float(parts[2]), float(parts[3]), float(parts[4])))
    return out
