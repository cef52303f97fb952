"""TEST INFRASTRUCTURE -- runs the reference program's own set-up and SCF loop
in a process of its own (the reference keeps its state in globals) and saves
what the device SCF loop needs to start from the same point.

    python ref_program_case.py WORKDIR OUT.npz [setup]

WORKDIR holds INPUT and the pseudopotential files.  The script runs
ReadInputFile, Setup, PrepareSCF (main.cpp), the starting density of
ChebySCFLoop.cpp:157-168 and EwaldEnergy, saves the cell, the local and
nonlocal pseudopotential arrays, the start density and the INPUT controls,
then (unless `setup` is given) runs ChebySCFLoop() with rand() seeded by
srand(1) and saves its final EIG and energies.  The reference's `!` lines go to stdout.
Needs oracle/_ref/libref.so."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))

import numpy as np  # noqa: E402

from ref_lib import RefLib  # noqa: E402


def main(workdir, out, setup_only=False):
    R = RefLib("libref.so")
    b = R.program_setup(workdir)
    ctrl = b.pop("ctrl")
    sys.stdout.flush()
    if setup_only:
        eig, e6 = np.zeros(0), np.zeros(6)
    else:
        eig, e6 = R.program_cheby_scf(workdir)
    arrays = {k: np.asarray(v) for k, v in b.items() if not isinstance(v, (list, tuple, dict))}
    arrays.update(nr=np.asarray(b["nr"]), na=np.asarray(b["na"]), lm_end=np.asarray(b["lm_end"]),
                  eig=eig, e6=e6,
                  ctrl_names=np.asarray(list(ctrl.keys())),
                  ctrl_values=np.asarray([float(v) for v in ctrl.values()]))
    np.savez(out, **arrays)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], len(sys.argv) > 3 and sys.argv[3] == "setup")
