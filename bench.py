#!/usr/bin/env python
"""Benchmark of the block H*psi path (Chebyshev-filter form) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--prec f32|f64]
                    [--workload si64|si216|scf-si8|scf-si64|converge-si64|eig-si216|setup-si64|
                                setup-si216|serve|batch|dense] [--rate R --jobs N --slots S]

One step = one call of the degree-10 Chebyshev filter (chebyfilt.cpp:6-74)
on the Si64 cell (64 atoms, a = 20.52 bohr, ecutwfc 15 Ha, 64^3 grid,
NGW 23847, 144 bands, synthetic local + s/p KB pseudopotential): ten block
H*psi applications with the three-term recurrence fused into the projector
GEMM epilogue.  The metric is H*psi GB/s: the algorithmic bytes of one block
H*psi (every 3D FFT = one grid read + one write, psi in/out once, V and the
projector inputs once per block; FP32 complex 8 B / real 4 B) times the ten
applications, divided by the device time of the step.  The same byte count
is used for every arm, so ratios are ratios of work per second.

Engine arm: inputs resident in HBM; each step restores X from a device copy
(the filter overwrites X) and runs the filter; L2 is flushed between steps
(256 MB write, outside the event-timed interval).  Multi-GPU: one process
per GPU, each filters its own replica of the block (weak scaling, no
collective: bands are independent).  e2e: the same filter through the C ABI
with pinned host FP64 buffers, host->device and device->host copies inside.

Reference arm (--impl reference): the reference's own chebyfilt built from
its sources (oracle/_ref/libref.so; FFT by the oracle's FFTW-API shim,
BLAS by scipy's OpenBLAS) on the host cores, one process per core, each
filtering a slice of bands of the same cell (a bounded sample).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ffr-pspw-dft-c_b200"))

import numpy as np  # noqa: E402

DEGREE = 10
# --nl-overlap values: the cell's PSPW_OVERLAP_* modes
OVERLAP_MODES = {"auto": 0, "on": 1, "off": 2}
LB, UB = 0.5, 16.0  # filter window (Ha) for the Si64 cell's spectrum
METRIC = "Hpsi GB/s (algorithmic, FP32 byte model; Chebyshev filter degree 10)"
WORKLOAD = ("Chebyshev filter (degree 10, chebyfilt.cpp) on Si64: 64 atoms, a=20.52 bohr, "
            "ecutwfc 15 Ha, grid 64^3, NGW 23847, 144 bands, s+p KB projectors")


# tcgen05.mma kind::tf32 dense rate measured on this pool's B200s
# (ffr-pspw-dft-c_b200/microbench/tcgen05_tf32_rate.cu): 4086 flop per cycle
# per SM (M=128, N=256, K=8 in 128.3 cycles), x 148 SMs x 1.965 GHz
TF32_DENSE_TFLOPS = 1188.3


def hpsi_bytes_model(ngw, nnr, nb, nat, fp64=False):
    sc, sr = (16, 8) if fp64 else (8, 4)
    return nb * (2 * ngw + 4 * nnr) * sc + nnr * sr + ngw * (4 + sr) + ngw * (nat * sc + 4 * sr)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ reference arm
def _ref_worker(args):
    """One host process: the reference's chebyfilt on `nbands` bands of the Si64
    cell, `steps` timed calls after `warmup`.  Returns per-step seconds."""
    nbands, steps, warmup, seed = args
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from ref_lib import RefLib
    from pspw import synth
    lat, pos = synth.si_diamond(2)
    R = RefLib()
    b = R.setup(lat, 30.0, (64, 64, 64), [64], [pos], [4.0], [3], [3], 4)
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    R.set_nl(pkg_a, wnl)
    veff = synth.local_potential(b["nr"], lat, pos)
    psi = synth.wavefunctions(b, lat, nbands, seed)
    R.set_nx(nbands - 2, 0)  # chebyfilt's width is NX+2 (chebyfilt.cpp:20)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)  # the reference prints; keep the JSON line clean
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        R.chebyfilt(psi, DEGREE, LB, UB, veff)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    return b["ngw"], times


def reference_sample(steps, warmup, bands_per_proc=4, procs=None):
    """Time the reference filter on all host cores.  Returns a dict with the
    metric value (same byte model as the engine arm) and the sample."""
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from ref_lib import ref_available
    if not ref_available():
        return None, "oracle/_ref/libref.so not built (make -C oracle)"
    procs = procs or len(os.sched_getaffinity(0)) or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(bands_per_proc, steps, warmup, 100 + i) for i in range(procs)])
    ngw = res[0][0]
    per_step = [max(r[1][k] for r in res) for k in range(steps)]
    t = sum(per_step) / len(per_step)
    nb_total = bands_per_proc * procs
    bytes_step = DEGREE * hpsi_bytes_model(ngw, 64 ** 3, nb_total, 64)
    return {"value": bytes_step / t / 1e9, "unit": "GB/s", "cores": procs, "kind": "reference",
            "seconds_per_step": t, "bands": nb_total,
            "sample": (f"reference chebyfilt (degree {DEGREE}) built from its sources, FFT by the "
                       f"oracle's FFTW-API shim (FFTW3 not installed), scipy OpenBLAS; {procs} "
                       f"processes x {bands_per_proc} bands of the Si64 cell = {nb_total} of 144 "
                       f"bands; {steps} timed calls")}, None


# ------------------------------------------------------------------ SCF-loop and set-up rows
# --workload scf-si8 | scf-si64: one step = one ChebySCF iteration
# (ChebySCFLoop.cpp:275-366: filter, QR, Rayleigh-Ritz, EvalRhoPsi, EvalENL,
# Pulay mixing, EvalEnergy, new bounds with a 10-step Lanczos) of the whole
# program run from an INPUT in the reference's format (random start,
# scf_conv_crit 0 so every iteration runs).  --workload setup-si64 |
# setup-si216: one step = the whole set-up before the SCF loop (ReadInputFile,
# ReadPseudopotentials, Setup, PrepareSCF, the starting density, EwaldEnergy).
ROW_WORKLOADS = {
    "scf-si8": dict(kind="scf", nrep=1, grid=(32, 32, 32), nempty=5,
                    text="Si8, a=10.26 bohr, ECUT 30 Ry, grid 32^3, NGW 2945, NX 21 (23 bands)"),
    "scf-si64": dict(kind="scf", nrep=2, grid=(64, 64, 64), nempty=14,
                     text="Si64, a=20.52 bohr, ECUT 30 Ry, grid 64^3, NGW 23847, NX 142 "
                          "(144 bands)"),
    "converge-si64": dict(kind="converge", nrep=2, grid=(64, 64, 64), nempty=14,
                          text="Si64, a=20.52 bohr, ECUT 30 Ry, grid 64^3, NGW 23847, NX 142 "
                               "(144 bands), to |dETOT| <= 1e-6 Ha"),
    "eig-si216": dict(kind="eigsolve", nrep=3, grid=(96, 96, 96), nempty=32,
                      text="Si216, a=30.78 bohr, ECUT 30 Ry, grid 96^3, NGW 80725, 512 states"),
    "setup-si64": dict(kind="setup", nrep=2, grid=(64, 64, 64), nempty=14,
                       text="Si64, a=20.52 bohr, ECUT 30 Ry, grid 64^3, NGW 23847, NX 142"),
    "setup-si216": dict(kind="setup", nrep=3, grid=(96, 96, 96), nempty=32,
                        text="Si216, a=30.78 bohr, ECUT 30 Ry, grid 96^3, NGW 80725, NX 464"),
}


def _write_row_input(d, w, max_scf, conv=0.0, imix=3):
    from pspw import synth
    from pspw.inputs import write_input, write_synthetic_fhi
    os.makedirs(d, exist_ok=True)
    lat, pos = synth.si_diamond(w["nrep"])
    write_synthetic_fhi(os.path.join(d, "X.fhi"))
    write_input(os.path.join(d, "INPUT"), "X.fhi", pos, float(lat[0][0]), ecut_ry=30.0, iscf=1,
                idiag=-1, imix=imix, max_scf=max_scf, nempty=w["nempty"], fft_grid=w["grid"],
                conv=conv)
    return d


def _ref_program_seconds(d, timeout):
    exe = os.path.join(ROOT, "oracle", "_ref", "ffr_pspw_dft.x")
    t0 = time.perf_counter()
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(r.stdout[-500:])
    return time.perf_counter() - t0


def _ref_setup_seconds(d):
    code = ("import sys, time, json; sys.path.insert(0, %r); from ref_lib import RefLib; "
            "R = RefLib(); t = time.perf_counter(); R.program_setup(%r); "
            "sys.stderr.write(json.dumps(time.perf_counter() - t))"
            % (os.path.join(ROOT, "oracle"), d))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-500:])
    return float(r.stderr.strip().splitlines()[-1])


def row_reference(args, w, tmp):
    """The reference on the row's workload, on the host cores (single
    process: the reference's SCF loop and set-up are serial)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from ref_lib import ref_available
    if not (ref_available() and os.path.exists(os.path.join(ROOT, "oracle", "_ref",
                                                             "ffr_pspw_dft.x"))):
        return None, "oracle/_ref not built (make -C oracle)"
    if w["kind"] == "eigsolve":
        return None, ("one reference LOBPCG iteration on Si216 (512 single-band ApplyHam "
                      "calls, 1536^3 LAPACK) takes tens of minutes")
    if w["kind"] == "converge":
        return None, ("one reference ChebySCF iteration on Si64 takes minutes, a converged "
                      "run hours; --workload scf-si64 --impl reference gives its rate")
    if w["kind"] == "setup":
        d = _write_row_input(os.path.join(tmp, "ref_setup"), w, 1)
        ts = [_ref_setup_seconds(d) for _ in range(max(1, args.steps))]
        t = sum(ts) / len(ts)
        return {"value": 1.0 / t, "unit": "set-ups/s", "cores": len(os.sched_getaffinity(0)),
                "kind": "reference",
                "seconds_per_step": t,
                "sample": f"reference ReadInputFile+Setup+PrepareSCF+starting density+"
                          f"EwaldEnergy built from its sources (serial code), {len(ts)} "
                          f"runs"}, None
    if args.workload == "scf-si64":
        # one reference iteration on Si64 takes minutes: its filter (more than
        # 90 % of the iteration) timed on all host cores as a bounded sample
        ref, why = reference_sample(steps=1, warmup=0)
        if ref is None:
            return None, why
        bytes_filter = DEGREE * hpsi_bytes_model(23847, 64 ** 3, 144, 64)
        t = bytes_filter / (ref["value"] * 1e9)
        return {"value": 1.0 / t, "unit": "SCF iterations/s", "cores": ref["cores"],
                "kind": "reference", "seconds_per_step": t,
                "sample": "the reference's chebyfilt of the 144-band Si64 block only (the rest "
                          "of the iteration not counted, so this is an upper bound of the "
                          "reference's iteration rate); " + ref["sample"]}, None
    k = max(1, args.steps)
    t_short = _ref_program_seconds(_write_row_input(os.path.join(tmp, "ref_a"), w, 1), 3600)
    t_long = _ref_program_seconds(_write_row_input(os.path.join(tmp, "ref_b"), w, 1 + k), 3600)
    t = (t_long - t_short) / k
    return {"value": 1.0 / t, "unit": "SCF iterations/s", "cores": len(os.sched_getaffinity(0)),
            "kind": "reference", "seconds_per_step": t,
            "sample": f"the reference program (main.cpp -> ChebySCFLoop) built from its "
                      f"sources on the same INPUT, run with MAX_SCF_ITER 1 and {1 + k}: "
                      f"(difference of wall times) / {k}; serial code, OpenBLAS with its "
                      f"default threads for the dense steps"}, None


def run_row(args, rank, world, local_rank):
    import tempfile

    import torch
    from pspw import PREC_F32, PREC_F64, replica
    from pspw.system import System
    w = ROW_WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    prec = PREC_F64 if args.prec == "f64" else PREC_F32
    tmp = tempfile.mkdtemp(prefix="pspw_row_")
    config = {"workload": f"{args.workload}: {w['text']}", "input": "INPUT + synthetic FHI98 "
              "pseudopotential in the reference's formats", "mixing": "Pulay (IMIX 3)",
              "start": "random (IDIAG -1)", "filter_prec": args.prec,
              "parallelism": f"replica x{world}",
              "l2": "inputs (NNR grids, the NGW x (NX+2) block) larger than L2 at Si64; "
                    "no flush"}
    clocks = ClockSampler(local_rank)
    if w["kind"] == "scf":
        n_it = args.warmup + args.steps
        S = System(_write_row_input(os.path.join(tmp, "engine"), w, n_it), device=local_rank)
        S.cell().set_nl_overlap(OVERLAP_MODES[args.nl_overlap])
        S.cheby_scf(filter_prec=prec)  # warm-up run (allocations, first-touch)
        replica.barrier()
        clocks.start()
        res = S.cheby_scf(filter_prec=prec)
        clocks.stop()
        h = res["hist"]
        assert res["iterations"] == n_it and np.isfinite(h[:, 0]).all()
        t = (h[n_it - 1, 3] - h[args.warmup - 1, 3]) * 1e-3 / args.steps
        # a third run with the phase timers on (CUDA events around each phase
        # on the cell stream), reported as the mean per iteration
        cell = S.cell()
        cell.timing_reset()
        cell.timing_enable(sum(1 << f for f in range(11, 19)))
        S.cheby_scf(filter_prec=prec)
        cell.timing_enable(0)
        names = ("filter", "qr", "rayleigh_ritz_products", "eigendecomposition", "density",
                 "enl", "mixing_energy", "lanczos_bounds")
        parts = {nm: round(cell.timing_read(f)[0] / n_it, 3) for nm, f in zip(names, range(11, 19))}
        S.close()
        unit, metric = "SCF iterations/s", "ChebySCF iterations/s (whole iteration on the device)"
    else:
        d = _write_row_input(os.path.join(tmp, "engine"), w, 1)
        for _ in range(args.warmup):
            System(d, device=local_rank).close()
        replica.barrier()
        clocks.start()
        ts, parts = [], None
        for _ in range(args.steps):
            t0 = time.perf_counter()
            S = System(d, device=local_rank)
            ts.append(time.perf_counter() - t0)
            parts = S.timing()
            S.close()
        clocks.stop()
        t = sum(ts) / len(ts)
        unit, metric = "set-ups/s", "system set-ups/s (INPUT to a ready cell, SCF handle and " \
                                    "starting density)"
    t_max = replica.max_over_ranks(t)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref, why = row_reference(argparse.Namespace(steps=1, workload=args.workload), w, tmp)
        cpu = ({k: (round(v, 6) if isinstance(v, float) else v) for k, v in ref.items()
                if k in ("value", "unit", "cores", "kind", "sample")} if ref else
               {"value": None, "unavailable": why})
    if rank == 0:
        out = {"metric": metric, "value": round(world / t_max, 4), "unit": unit, "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_max * 1e3, 3),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64" if args.prec == "f64" else "c64 filter, f64 rest",
               "data": "synthetic", "config": config, "cpu_baseline": cpu,
               "clocks": clocks.summary(),
               "timing": "host wall clock between iteration ends (the loop synchronises at "
                         "each iteration end)" if w["kind"] == "scf" else
                         "host wall clock around pspw_system_load"}
        if w["kind"] == "setup":
            out["phases_ms"] = {k: round(v, 3) for k, v in parts.items()}
        else:
            out["phases_ms_per_iteration"] = parts
        print(json.dumps(out))


MAX_SCF_CONVERGE = 160
PULAY_CFG1 = dict(pulay_beta=0.3, mixdim=6)  # the Si64 SCF configuration's Pulay mixer


def _time_to_band(hist, e_star, band):
    """(ms, iteration) at which ETOT enters |ETOT - e_star| <= band and stays
    there for the rest of the run; (None, None) if it never does."""
    err = np.abs(hist[:, 0] - e_star)
    inside = err <= band
    if not inside[-1]:
        return None, None
    i = len(inside) - 1
    while i > 0 and inside[i - 1]:
        i -= 1
    return float(hist[i, 3]), i + 1


def run_converge(args, rank, world, local_rank):
    """--workload converge-si64: the Si64 SCF target, time to converged of
    the mixed form (the filter and the H*v of the Lanczos filter bounds in
    FP32; orthonormalisation, Rayleigh-Ritz, density, energies and mixing in
    FP64) against the plain FP64 form.

    Converged means: ETOT within 1e-6 Ha/atom of the fixed point and staying
    there.  The fixed point E* is the FP64 run with Kerker mixing (whose
    |dETOT| falls monotonically) taken to |dETOT| <= 1e-10 Ha.  Each timed run
    (its own freshly loaded system; loading not timed) runs to |dETOT| <= 1e-9
    Ha or MAX_SCF_CONVERGE iterations; its per-iteration host timestamps give
    the time at which ETOT entered the 1e-6 Ha/atom band around E* for good.
    The per-atom stop rule |dETOT| <= 1e-6 Ha/atom is reported beside it
    (where it fires and how far from E* it stops).  Mixers: Pulay with beta
    0.3 and a 6-step history (the configuration's mixer; the reference
    hard-codes beta 0.25 in PulayRhoMix.cpp:10, so the engine's explicit
    controls set it) and Kerker (IMIX 1).  value = the mixed Pulay run's
    time to converged (s)."""
    import tempfile

    import torch
    from pspw import PREC_F32, PREC_F64, replica
    from pspw.system import System
    w = ROW_WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    tmp = tempfile.mkdtemp(prefix="pspw_conv_")
    dirs = {mx: _write_row_input(os.path.join(tmp, mx), w, MAX_SCF_CONVERGE, conv=1e-9,
                                 imix=im) for mx, im in (("pulay", 3), ("kerker", 1))}
    controls = {"pulay": PULAY_CFG1, "kerker": {}}
    nat = 8 * w["nrep"] ** 3
    band = 1e-6 * nat
    nocc = int(round(4 * nat / 2))
    modes = {"fp64": PREC_F64, "mixed": PREC_F32}
    # the fixed point
    S = System(dirs["kerker"], device=local_rank)
    star = S.cheby_scf(filter_prec=PREC_F64, conv=1e-10, max_scf_iter=400)
    S.close()
    e_star = star["energies"]["ETOT"]
    S = System(dirs["pulay"], device=local_rank)
    S.cheby_scf(filter_prec=PREC_F32, max_scf_iter=3)  # warm-up (modules, handles)
    S.close()
    replica.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    report = {}
    for mx, d in dirs.items():
        runs = {m: [] for m in modes}
        last = {}
        for _ in range(max(1, args.steps)):
            for m, prec in modes.items():
                S = System(d, device=local_rank)
                torch.cuda.synchronize()
                res = S.cheby_scf(filter_prec=prec, **controls[mx])
                S.close()
                t_ms, it = _time_to_band(res["hist"], e_star, band)
                runs[m].append(t_ms)
                last[m] = (res, it)
        out = {}
        for m in modes:
            res, it = last[m]
            h = res["hist"]
            ok = all(t is not None for t in runs[m])
            t_conv = replica.max_over_ranks(sum(runs[m]) / len(runs[m]) * 1e-3) if ok else None
            stop = np.nonzero(h[:, 1] <= band)[0]
            de = res["eig"][:nocc] - star["eig"][:nocc]
            out[m] = {
                "seconds_to_converged": round(t_conv, 4) if ok else None,
                "iterations_to_converged": it,
                "ms_per_iteration": round(float(np.diff(h[:, 3]).mean()), 3),
                "final_etot_error_ha_per_atom": abs(res["energies"]["ETOT"] - e_star) / nat,
                "final_eig_max_error_ha_occupied": float(np.abs(de).max()),
                "iterations_run": res["iterations"],
                "per_atom_stop_rule": (
                    {"iteration": int(stop[0]) + 1,
                     "seconds": round(float(h[stop[0], 3]) * 1e-3, 4),
                     "etot_error_ha_per_atom": float(abs(h[stop[0], 0] - e_star) / nat)}
                    if len(stop) else None)}
        sp = (round(out["fp64"]["seconds_to_converged"] / out["mixed"]["seconds_to_converged"], 3)
              if out["fp64"]["seconds_to_converged"] and out["mixed"]["seconds_to_converged"]
              else None)
        report[mx] = {"controls": controls[mx] or "INPUT (rho_mix_fac 0.3)", "modes": out,
                      "speedup_mixed_vs_fp64": sp}
    clocks.stop()
    p32 = report["pulay"]["modes"]["mixed"]
    p64 = report["pulay"]["modes"]["fp64"]
    if rank == 0:
        out = {"metric": "Si64 ChebySCF time to converged (1e-6 Ha/atom of the FP64 fixed point), "
                         "FP32 filter / FP64 Rayleigh-Ritz, Pulay beta 0.3 history 6",
               "value": p32["seconds_to_converged"], "unit": "s", "n_gpus": world,
               "steps": args.steps, "warmup": 1,
               "ms_per_step": (round(p32["seconds_to_converged"] * 1e3, 3)
                               if p32["seconds_to_converged"] else None),
               "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
               "dtype": "c64 filter, f64 rest", "data": "synthetic",
               "config": {"workload": f"{args.workload}: {w['text']}",
                          "input": "INPUT + synthetic FHI98 pseudopotential in the "
                                   "reference's formats",
                          "start": "random (IDIAG -1)", "filter_degree": 10,
                          "criterion": "ETOT within 1e-6 Ha/atom of E* (FP64, Kerker, "
                                       "|dETOT| <= 1e-10) and staying there",
                          "parallelism": f"replica x{world}",
                          "l2": "inputs larger than L2; no flush"},
               "fixed_point": {"etot_ha": e_star, "iterations": star["iterations"],
                               "converged": star["converged"]},
               "pulay": report["pulay"], "kerker": report["kerker"],
               "speedup_mixed_vs_fp64": report["pulay"]["speedup_mixed_vs_fp64"],
               "speedup_per_iteration": round(p64["ms_per_iteration"] / p32["ms_per_iteration"],
                                              3),
               "cpu_baseline": {"value": None,
                                "unavailable": "one reference iteration on Si64 takes minutes "
                                               "(see --workload scf-si64 for its rate)"},
               "clocks": clocks.summary(),
               "timing": "host timestamps at the end of each SCF iteration (ms since the "
                         "call began; the loop synchronises there)"}
        print(json.dumps(out))


def cheby_start(cell, ngw, nb, torch, dev, iters=30, extra=32, degree=10, seed=11):
    """A common start block for the eigensolver comparison: Chebyshev-filtered
    subspace iteration (the SCF loop's eigen-part, ChebySCFLoop.cpp:280-307,
    on the fixed potential) in FP64 on nb + extra columns: filter on
    [largest Ritz value, Lanczos upper bound], span orthonormalisation,
    Rayleigh-Ritz.  Returns the nb lowest Ritz vectors (host, ngw x nb) and
    the largest residual norm among them."""
    from pspw import PREC_F64
    m = nb + extra
    g = torch.Generator(device=dev).manual_seed(seed)
    X = torch.complex(torch.randn(m, ngw, device=dev, dtype=torch.float64, generator=g),
                      torch.randn(m, ngw, device=dev, dtype=torch.float64, generator=g))
    HX = torch.zeros_like(X)
    S = torch.zeros(m, m, dtype=torch.complex128, device=dev)
    w = torch.zeros(m, dtype=torch.float64, device=dev)
    rng = np.random.default_rng(seed)
    # upper bound of the spectrum: largest Ritz value of a 10-step Lanczos
    # plus the residual norm (Zhou and Saad, J. Comput. Phys. 219 (2006))
    T, f, _ = cell.lanczos(rng.standard_normal(ngw) + 1j * rng.standard_normal(ngw), 10)
    ub = float(np.linalg.eigvalsh(0.5 * (T + T.T)).max()) + float(np.linalg.norm(f))

    def rayleigh_ritz():
        nonlocal X
        cell.apply_ham_block_dev(X, HX, ngw, ngw, m, PREC_F64)
        cell.zgemm_dev("C", m, m, ngw, 1.0, X, ngw, HX, ngw, 0.0, S, m)
        cell.eig_zheevd_dev(S, m, w, m)
        Y = torch.zeros_like(X)
        cell.zgemm_dev("N", ngw, m, m, 1.0, X, ngw, S, m, 0.0, Y, ngw)
        X = Y

    cell.ortho_span_dev(X, ngw, m)
    rayleigh_ritz()
    for _ in range(iters):
        torch.cuda.synchronize()
        lb = float(w[-1])
        cell.chebyfilt_dev(X, ngw, ngw, m, degree, lb, ub, PREC_F64)
        cell.ortho_span_dev(X, ngw, m)
        rayleigh_ritz()
    cell.apply_ham_block_dev(X, HX, ngw, ngw, m, PREC_F64)
    torch.cuda.synchronize()
    r = (HX[:nb] - w[:nb, None] * X[:nb]).abs().pow(2).sum(1).sqrt()
    return np.ascontiguousarray(X[:nb].cpu().numpy().T), float(r.max()), ub


def run_eigsolve(args, rank, world, local_rank):
    """--workload eig-si216: the block eigensolvers on the Si216 cell (96^3,
    NGW 80725, 512 bands, fixed V_loc): davidson_cpu (2 x 512 subspace),
    lobpcg_cpu (Q of 3 x 512 columns, 1536 x 1536 Rayleigh-Ritz) and the
    opt-in lobpcg_ortho (orthonormal [X W P] basis) on the device, each run
    for at most `--steps` iterations from the reference's own
    random start (random_col), with H*psi and the preconditioner in FP64 and
    in FP32; orthonormalisation, Gram matrices and the subspace eigensolves
    are FP64 in both.  Eigenvalues of the states both runs resolve
    (residual below 1e-4, 1e-3, 1e-2) are compared between the two.
    --solvers picks the solvers (default both).  value = iterations per
    second of the first solver with FP32 H*psi."""
    import torch
    from pspw import PREC_F32, PREC_F64, replica, workloads
    torch.cuda.set_device(local_rank)
    wl = workloads.si_cell(3, 96)
    cell = workloads.make_cell(wl, device=local_rank)
    ngw, nb, nempty = wl["ngw"], 512, 32
    prec = cell.gen_prec(ngw, -10.0)
    iters = max(1, args.steps)
    out_modes = {}
    clocks = ClockSampler(local_rank)
    cell.lobpcg(ngw, nb, prec, nempty, max_iter=1, hprec=PREC_F32)  # warm-up (allocations)
    cell.davidson(ngw, nb, prec, nempty, max_iter=1, hprec=PREC_F32)
    replica.barrier()
    clocks.start()
    start = None
    if args.warm_start:
        t0 = time.perf_counter()
        X0, r0, ub0 = cheby_start(cell, ngw, nb, torch, torch.device("cuda", local_rank))
        start = {"kind": "Chebyshev-filtered subspace iteration, FP64, 30 passes of degree 10 "
                         "on 544 columns", "seconds": round(time.perf_counter() - t0, 3),
                 "max_residual": r0, "ub": ub0}
    for solver in args.solvers.split(","):
        run = getattr(cell, solver)
        res = {}
        for name, hp in (("fp64", PREC_F64), ("fp32", PREC_F32)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if start is not None:
                ev, _, r, it = run(ngw, nb, prec, nempty, max_iter=iters, hprec=hp, X0=X0)
            else:
                ev, _, r, it = run(ngw, nb, prec, nempty, max_iter=iters, hprec=hp)
            res[name] = (time.perf_counter() - t0, ev, r, it)
        r64 = np.maximum(res["fp64"][2], res["fp32"][2])  # both runs resolve the state
        d = np.abs(res["fp64"][1] - res["fp32"][1])
        out_modes[solver] = {
            m: {"seconds": round(v[0], 3), "iterations": v[3],
                "ms_per_iteration": round(v[0] * 1e3 / max(1, v[3]), 2)}
            for m, v in res.items()}
        out_modes[solver]["residual_min_median_max"] = [float(np.min(r64)),
                                                         float(np.median(r64)),
                                                         float(np.max(r64))]
        for tol in (1e-4, 1e-3, 1e-2):
            ok = r64 < tol
            out_modes[solver][f"states_res_below_{tol:g}"] = int(ok.sum())
            out_modes[solver][f"eig_max_error_ha_res_below_{tol:g}"] = (
                float(d[ok].max()) if ok.any() else None)
        out_modes[solver]["eig_max_error_ha_all"] = float(d.max())
        out_modes[solver]["speedup_fp32_vs_fp64"] = round(res["fp64"][0] / res["fp32"][0], 3)
    clocks.stop()
    cell.close()
    lob = out_modes[args.solvers.split(",")[0]]["fp32"]
    t_it = replica.max_over_ranks(lob["seconds"] / max(1, lob["iterations"]))
    if rank == 0:
        print(json.dumps({
            "metric": f"Si216 {args.solvers.split(',')[0]} iterations/s, FP32 H*psi, FP64 "
                      "subspace steps",
            "value": round(world / t_it, 4), "unit": "iterations/s", "n_gpus": world,
            "steps": iters, "warmup": 1, "ms_per_step": round(t_it * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 H*psi, f64 rest", "data": "synthetic",
            "config": {"workload": "eig-si216: Si216, a=30.78 bohr, ECUT 30 Ry, grid 96^3, "
                                   "NGW 80725, 512 states (32 empty), fixed V_loc",
                       "start": (start if start is not None
                                 else "random_col (the reference's LCG start)"),
                       "preconditioner": "GenPrec tau=-10 (Teter)",
                       "parallelism": f"replica x{world}",
                       "l2": "inputs larger than L2; no flush"},
            "solvers": out_modes,
            "cpu_baseline": {"value": None,
                             "unavailable": "one reference LOBPCG iteration on Si216 "
                                            "(512 single-band ApplyHam calls, 1536^3 "
                                            "LAPACK) takes tens of minutes"},
            "clocks": clocks.summary(),
            "timing": "host wall clock around each solver call"}))


# ------------------------------------------------------------------ dense FP64 steps
DENSE_SHAPES = [  # (name, op, m, n, k)
    ("Gram X^H Y, Si64 SCF (146 x 146 over NGW 23847)", "C", 146, 146, 23847),
    ("rotation X Q, Si64 SCF (23847 x 146, k 146)", "N", 23847, 146, 146),
    ("FP64 projection beta^H psi, Si64 (256 x 144 over NGW 23847)", "C", 256, 144, 23847),
    ("FP64 back-projection beta W, Si64 (23847 x 144, k 256)", "N", 23847, 144, 256),
    ("Gram Q^H HQ, Si216 LOBPCG (1536 x 1536 over NGW 80725)", "C", 1536, 1536, 80725),
]


def run_dense(args, rank, world, local_rank):
    """--workload dense: the FP64 dense steps of the SCF loop and the
    solvers, timed with CUDA events on the cell stream: the engine's DMMA
    complex GEMM at the shapes the Si64 SCF and the Si216 LOBPCG use, beside
    cuBLAS ZGEMM on the same operands (torch.matmul of complex128 tensors,
    the library baseline), and the 146 x 146 Hermitian eigensolve against
    cuSOLVER zheevd (torch.linalg.eigh).  Complex MAC = 8 flops."""
    import torch
    from pspw import workloads
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = workloads.workload("si8")
    cell = workloads.make_cell(w, device=local_rank)
    stream = torch.cuda.ExternalStream(cell.stream(), device=dev)
    g = torch.Generator(device=dev).manual_seed(5)
    reps = max(3, args.steps)

    def crand(rows, cols):
        return torch.complex(torch.randn(rows, cols, device=dev, dtype=torch.float64,
                                         generator=g),
                             torch.randn(rows, cols, device=dev, dtype=torch.float64,
                                         generator=g))

    def timed(fn):
        with torch.cuda.stream(stream):
            for _ in range(2):
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    rows = []
    for name, op, m, n, k in DENSE_SHAPES:
        # column-major operands as torch row-major transposes
        At = crand(m, k) if op == "C" else crand(k, m)   # A^H: A is k x m -> tensor (m, k)
        Bt = crand(n, k)
        Ct = torch.zeros(n, m, dtype=torch.complex128, device=dev)
        lda = k if op == "C" else m
        ms_own = timed(lambda: cell.zgemm_dev(op, m, n, k, 1.0, At, lda, Bt, k, 0.0, Ct, m))
        A_lib = At.conj() if op == "C" else At.T  # (m, k)
        B_lib = Bt.T
        ms_lib = timed(lambda: torch.matmul(A_lib, B_lib))
        ref = torch.matmul(A_lib, B_lib)
        err = float((Ct.T - ref).abs().max() / ref.abs().max())
        fl = 8.0 * m * n * k
        rows.append({"gemm": name, "m": m, "n": n, "k": k, "op": op,
                     "engine_ms": round(ms_own, 4), "engine_tflops": round(fl / ms_own / 1e9, 2),
                     "cublas_ms": round(ms_lib, 4), "cublas_tflops": round(fl / ms_lib / 1e9, 2),
                     "rel_diff": err})
        del At, Bt, Ct, A_lib, B_lib, ref
    # Hermitian eigensolve of order 146 (the Si64 Rayleigh-Ritz matrix)
    n = 146
    M = crand(n, n)
    H = (M + M.conj().T) * 0.5
    Hc = H.clone()
    wv = torch.zeros(n, dtype=torch.float64, device=dev)

    def own_eig():
        Hc.copy_(H)
        cell.eig_zheevd_dev(Hc, n, wv, n)

    ms_eig = timed(own_eig)
    ms_eig_lib = timed(lambda: torch.linalg.eigh(H))
    # the SCF's orthonormalisation of the filtered block (23847 x 146)
    X0 = crand(146, 23847)
    Xs = X0.clone()

    def own_span():
        Xs.copy_(X0)
        cell.ortho_span_dev(Xs, 23847, 146)

    ms_span = timed(own_span)
    ms_qr_lib = timed(lambda: torch.linalg.qr(X0.T))
    wl = torch.linalg.eigvalsh(H)
    eig_err = float((wv - wl).abs().max() / wl.abs().max())
    if rank == 0:
        out = {"metric": "FP64 dense steps: DMMA complex GEMM TFLOP/s at the Si64 SCF shapes",
               "value": rows[0]["engine_tflops"], "unit": "TFLOP/s", "n_gpus": world,
               "steps": reps, "warmup": 2, "ms_per_step": rows[0]["engine_ms"],
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "c128", "data": "synthetic (normal random matrices)",
               "config": {"workload": "dense: the SCF loop's and LOBPCG's FP64 GEMM shapes, "
                                      "the 146 x 146 Hermitian eigensolve"},
               "gemm": rows,
               "eig146": {"engine_ms": round(ms_eig, 4), "cusolver_ms": round(ms_eig_lib, 4),
                          "eigenvalue_rel_diff": eig_err},
               "ortho_span_23847x146": {"engine_ms": round(ms_span, 4),
                                        "cusolver_householder_qr_ms": round(ms_qr_lib, 4)}}
        print(json.dumps(out))


# ------------------------------------------------------------------ batched cells
def run_batch(args, rank, world, local_rank):
    """--workload batch: block H*psi over 32 independent orthorhombic cells
    (lattice constants 8-16 bohr, 2-16 atoms at least 3 bohr apart, ecutwfc
    10-25 Ha with 5-smooth grids 24-72 per axis, 8-256 bands; seeded) in one
    CUDA-graph launch per step, FP32, each cell on the schedule the batch's
    autotuner picked.  value = the summed algorithmic bytes of the cells'
    H*psi (FP32 byte model) / the step's device time."""
    import torch
    from pspw import PREC_F32, Cell, replica
    from pspw.batch import Batch, ortho_cell
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    rng = np.random.default_rng(2026 + rank)
    data = [ortho_cell(rng) for _ in range(args.cells)]
    cells = []
    for d in data:
        c = Cell.from_arrays(d, device=local_rank)
        c.set_veff(d["veff"])
        cells.append(c)
    b = Batch(cells, [d["nbands"] for d in data], PREC_F32)
    for i, d in enumerate(data):
        b.upload(i, d["psi"])
    t0 = time.perf_counter()
    b.tune(reps=3)
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        b.apply()
    b.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    clocks.start()
    replica.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            b.apply()
            evs[k][1].record(stream)
    b.synchronize()
    clocks.stop()
    launches = b.kernels() * args.steps  # graph replays: the captured kernels
    ms = sum(a.elapsed_time(z) for a, z in evs) / args.steps
    ms_max = replica.max_over_ranks(ms, device=dev)
    nbytes = sum(hpsi_bytes_model(d["ngw"], int(np.prod(d["nr"])), d["nbands"],
                                  len(d["positions"])) for d in data)
    gbs = replica.weak_throughput(nbytes, world, ms_max * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    sched = [b.schedule(i) for i in range(len(data))]
    eager_ms = sum(s["ms"] for s in sched)
    b.close()
    if rank == 0:
        print(json.dumps({
            "metric": "batched H*psi GB/s over 32 uneven cells (FP32 byte model), one graph "
                      "launch per step",
            "value": round(gbs, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": f"batch: {len(data)} orthorhombic cells, a,b,c 8-16 bohr, "
                                   "2-16 atoms, ecutwfc 10-25 Ha, grids 24-72, 8-256 bands "
                                   "(seed 2026)",
                       "grids": sorted({tuple(d["nr"]) for d in data}),
                       "bands_total": int(sum(d["nbands"] for d in data)),
                       "parallelism": f"replica x{world}",
                       "l2": "flushed between steps (256 MB write, outside the timed interval)"},
            "roofline": {"kernel": "whole batch (graph)", "bound": "hbm",
                         "achieved": round(gbs / world, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / world / peak, 4),
                         "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                         "bytes_per_launch": int(nbytes), "traffic": None},
            "tuned_eager_ms_sum": round(eager_ms, 4),
            "graph_vs_eager_sum": round(eager_ms / ms_max, 3),
            "tune_seconds": round(tune_s, 2),
            "schedules": {"band_batch": [s["band_batch"] for s in sched],
                          "nl_path": [s["nl_path"] for s in sched]},
            "gpu_launches": launches // args.steps,
            "cpu_baseline": {"value": None,
                             "unavailable": "the reference applies H*psi to one cell per "
                                            "process; see the default workload for its rate"},
            "clocks": clocks.summary(),
            "timing": "CUDA events on the batch stream around each graph launch"}))


# ------------------------------------------------------------------ SCF serving
def run_serve(args, rank, world, local_rank):
    """--workload serve: the SCF serving loop.  Jobs (isolated clusters of
    2-64 atoms of four synthetic species with Gaussian wells of depth 1-4 Ha
    and width 0.8-1.6 bohr, cubic boxes up to 24 bohr, ecutwfc 12-25 Ha,
    ceil(0.6 * 4 * atoms) + 8 states, random start, the reference's Broyden
    mixing (IMIX 4, alpha 0.25; its Pulay mixing converges few of these
    random clusters within 200 iterations), converged at |dETOT| <= 1e-6
    Ha/atom within 200 iterations) arrive by a
    seeded Poisson process at --rate jobs/s and are submitted to the device
    server (continuous batching over --slots concurrent jobs, admission by
    HBM footprint).  Each precision form serves the same job sequence.
    Latency = completion - arrival (queueing included); throughput = jobs /
    (last completion - first arrival).  value = the mixed form's jobs/s."""
    import tempfile

    import torch
    from pspw import PREC_F32, PREC_F64, replica, serve
    torch.cuda.set_device(local_rank)
    rng = np.random.default_rng(2028 + rank)
    species = serve.species_set(rng)
    tmp = tempfile.mkdtemp(prefix="pspw_serve_")
    jobs = [serve.cluster_job(rng, os.path.join(tmp, f"job{k}"), species, imix=4)
            for k in range(args.jobs)]
    arrivals = serve.poisson_arrivals(np.random.default_rng(77), args.rate, args.jobs)
    warm = serve.cluster_job(np.random.default_rng(1), os.path.join(tmp, "warm"), species,
                             natoms=4, ecut_ha=12.0, box=10.5)
    clocks = ClockSampler(local_rank)
    out_modes = {}
    replica.barrier()
    clocks.start()
    for name, prec in (("fp64", PREC_F64), ("mixed", PREC_F32)):
        srv = serve.Server(device=local_rank, slots=args.slots, filter_prec=prec,
                           conv_per_atom=1e-6, max_scf_iter=200, pulay_beta=0.0, mixdim=0)
        srv.wait(srv.submit(warm["dir"]))  # module loading, library handles
        t0 = time.perf_counter()
        ids, t_arr = [], []
        for a, j in zip(arrivals, jobs):
            delay = a - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            t_arr.append(srv.now())
            ids.append(srv.submit(j["dir"]))
        res = [srv.wait(i) for i in ids]
        srv.close()
        lat = [r["t_done"] - ta for r, ta in zip(res, t_arr)]
        ok = [r["status"] == 0 for r in res]
        conv = [bool(r["converged"]) for r in res]
        span = max(r["t_done"] for r in res) - min(t_arr)
        out_modes[name] = {
            "jobs_per_s": round(len(res) / span, 4),
            "latency_p50_s": round(serve.percentile(lat, 50), 4),
            "latency_p99_s": round(serve.percentile(lat, 99), 4),
            "latency_mean_s": round(float(np.mean(lat)), 4),
            "queue_mean_s": round(float(np.mean([r["t_admit"] - ta
                                                 for r, ta in zip(res, t_arr)])), 4),
            "latency_converged_p50_s": (round(serve.percentile(
                [x for x, cv in zip(lat, conv) if cv], 50), 4) if any(conv) else None),
            "latency_converged_p99_s": (round(serve.percentile(
                [x for x, cv in zip(lat, conv) if cv], 99), 4) if any(conv) else None),
            "ok": int(sum(ok)), "converged": int(sum(conv)), "jobs": len(res),
            "errors": sorted({r["error"] for r in res if r["status"] != 0}),
            "iterations_mean": round(float(np.mean([r["iterations"] for r in res])), 2),
            "max_concurrent": int(max(sum(1 for q in res if q["t_admit"] <= r["t_admit"] < q["t_done"])
                                      for r in res)),
            "makespan_s": round(span, 3)}
        out_modes[name]["_etot"] = [r["etot"] for r in res]
    clocks.stop()
    e64, e32 = out_modes["fp64"].pop("_etot"), out_modes["mixed"].pop("_etot")
    nat = np.array([j["natoms"] for j in jobs])
    de = np.abs(np.array(e32) - np.array(e64)) / nat
    m = out_modes["mixed"]
    if rank == 0:
        print(json.dumps({
            "metric": "SCF serving jobs/s (Poisson arrivals, continuous batching), mixed form; "
                      "p50/p99 time-to-converged beside it",
            "value": m["jobs_per_s"], "unit": "jobs/s", "n_gpus": world, "steps": args.jobs,
            "warmup": 1, "ms_per_step": round(1e3 / m["jobs_per_s"], 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 filter, f64 rest", "data": "synthetic",
            "config": {"workload": f"serve: {args.jobs} cluster jobs (2-64 atoms, 4 species, "
                                   f"box 10-24 bohr, ecutwfc 12-25 Ha), Poisson arrivals at "
                                   f"{args.rate} jobs/s (seed 77), {args.slots} slots",
                       "stop": "|dETOT| <= 1e-6 Ha/atom, at most 200 iterations",
                       "mixing": "the reference's Broyden (IMIX 4, alpha 0.25)",
                       "start": "random (IDIAG -1)",
                       "parallelism": f"replica x{world}",
                       "l2": "inputs larger than L2 for the large jobs; no flush"},
            "modes": out_modes,
            "etot_mixed_vs_fp64_ha_per_atom": {"max": float(de.max()),
                                               "median": float(np.median(de))},
            "cpu_baseline": {"value": None,
                             "unavailable": "the reference runs one SCF job per process; one "
                                            "such job of this mix takes minutes on the host"},
            "clocks": clocks.summary(),
            "timing": "server clock (host steady clock) from submission at the arrival time "
                      "to the job's completion"}))


# ------------------------------------------------------------------ engine arm
def run_engine(args, rank, world, local_rank):
    import torch
    from pspw import PREC_F32, PREC_F64, replica, workloads
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = workloads.workload(args.workload)
    cell = workloads.make_cell(w, device=local_rank)
    cell.set_nl_overlap(OVERLAP_MODES[args.nl_overlap])
    sizes = cell.sizes()
    psi = w["psi"]
    ngw, nb = psi.shape
    nnr = int(np.prod(w["nr"]))
    nat = sizes["nat"]
    fp64 = args.prec == "f64"
    prec = PREC_F64 if fp64 else PREC_F32
    cdt = torch.complex128 if fp64 else torch.complex64
    x0 = torch.from_numpy(np.ascontiguousarray(psi.T)).to(cdt).to(dev)  # (nb, ngw) = ngw x nb col-major
    x = torch.empty_like(x0)
    stream = torch.cuda.ExternalStream(cell.stream(), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        x.copy_(x0)
        cell.chebyfilt_dev(x, ngw, ngw, nb, DEGREE, LB, UB, prec)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.5)
    fam_mask = sum(1 << f for f in range(3, 10))
    cell.timing_reset()
    cell.timing_enable(fam_mask)
    l0 = cell.kernel_launches()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    replica.barrier()
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(float(k))  # evict L2 between steps (not timed)
            evs[k][0].record(stream)
            step()
            evs[k][1].record(stream)
    torch.cuda.synchronize()
    replica.barrier()
    t_wall = time.perf_counter() - t_wall
    launches = (cell.kernel_launches() - l0) // args.steps
    cell.timing_enable(0)
    fam = {f: cell.timing_read(f) for f in range(3, 10)}
    clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ms = sum(step_ms) / len(step_ms)
    ms_max = replica.max_over_ranks(ms, device=dev)
    bytes_step = DEGREE * hpsi_bytes_model(ngw, nnr, nb, nat, fp64=False)
    value = replica.weak_throughput(bytes_step, world, ms_max * 1e-3) / 1e9

    # ---- per-kernel roofline (dominant kernel family on the cell stream)
    # Algorithmic bytes of each kernel = its share of the block H*psi byte
    # model B_Hpsi (psi in/out and the maps to the stick kernels, the 3D-FFT
    # grid traffic 4*NNR*s_c per band and V_eff to the plane kernel, the
    # projector inputs to the projector kernels).  The projector GEMMs are
    # reported in flops (F_NL = 8*NGW*nproj*nb per GEMM, complex MAC = 8).
    sc, sr = (16, 8) if fp64 else (8, 4)
    calls = args.steps * DEGREE
    names = {3: "k_sticks_inv", 5: "k_plane", 7: "k_sticks_fwd", 8: "k_proj_tc(+k_proj_tc_wtiles)",
             9: "k_backproj_tc"}
    if fp64:
        names.update({8: "k_proj(+k_proj_reduce)", 9: "k_backproj"})
    fam_ms = {f: fam[f][0] for f in fam if fam[f][1] > 0}
    nproj = sizes["nproj"]
    alg_bytes = {  # per H*psi call
        3: nb * ngw * sc + ngw * 4,
        5: nb * 4 * nnr * sc + nnr * sr,
        7: nb * 2 * ngw * sc + ngw * (4 + sr),
        8: nb * ngw * sc + ngw * (nat * sc + 4 * sr),
        9: 3 * nb * ngw * sc + ngw * (nat * sc + 4 * sr),
    }
    alg_flops = {8: 8.0 * ngw * nproj * nb, 9: 8.0 * ngw * nproj * nb}
    # the dominant family on the critical path: the projection (family 8)
    # runs on the cell's second stream, concurrently with the FFT passes, so
    # its event time spans the plane kernel's and is not serial time (in the
    # serialised ncu launch list it is 21 % of the H*psi, the plane kernel 46 %)
    top = max((f for f in fam_ms if f != 8), key=lambda f: fam_ms[f])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "measured" if "hbm_gbs" in peaks else "fallback"
    n_launch = fam[top][1]
    avg_us = fam_ms[top] / n_launch * 1e3
    if top in (3, 5, 7):
        per_launch = alg_bytes[top] * calls / n_launch
        achieved = per_launch / (avg_us * 1e-6) / 1e9
        roof = {"kernel": names[top], "bound": "hbm", "achieved": round(achieved, 1),
                "peak": hbm_peak, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                "peak_source": hbm_src, "bytes_per_launch": int(per_launch),
                "launches": n_launch, "avg_launch_us": round(avg_us, 2)}
    else:
        per_launch = alg_flops[top] * calls / n_launch
        achieved = per_launch / (avg_us * 1e-6) / 1e12
        roof = {"kernel": names[top], "bound": "tensor", "achieved": round(achieved, 2),
                "peak": TF32_DENSE_TFLOPS, "unit": "TFLOP/s",
                "frac": round(achieved / TF32_DENSE_TFLOPS, 4),
                "peak_source": "measured tcgen05 kind::tf32 MMA rate (4086 flop/cycle/SM at "
                               "1965 MHz); the kernels issue 3 TF32 products per FP32 product",
                "flops_per_launch": int(per_launch), "launches": n_launch,
                "avg_launch_us": round(avg_us, 2)}
    # every family on the same footing, for the launch-share table
    fam_report = {}
    for f, t in fam_ms.items():
        d = {"ms_per_step": round(t / args.steps, 4), "launches_per_step": fam[f][1] // args.steps}
        if f in alg_bytes:
            d["alg_gbs"] = round(alg_bytes[f] * calls / (t * 1e-3) / 1e9, 1)
        if f in alg_flops:
            d["alg_tflops"] = round(alg_flops[f] * calls / (t * 1e-3) / 1e12, 2)
        fam_report[names.get(f, str(f))] = d
    roof["traffic"] = _ncu_traffic(args.workload, roof["kernel"], args.prec)
    roof["traffic_source"] = ("profiles/ncu_traffic.txt: dram__bytes_read.sum + "
                              "dram__bytes_write.sum per launch from an ncu capture of this "
                              "command (not measured in this run)")
    kernels_ms = fam_report
    hpsi_ms = ms_max / DEGREE
    hpsi_roof = {"bytes_per_hpsi": hpsi_bytes_model(ngw, nnr, nb, nat, fp64=fp64),
                 "ms_per_hpsi": round(hpsi_ms, 4),
                 "achieved_gbs": round(hpsi_bytes_model(ngw, nnr, nb, nat, fp64=fp64)
                                       / (hpsi_ms * 1e-3) / 1e9, 1),
                 "frac_of_measured_hbm": None}
    hpsi_roof["frac_of_measured_hbm"] = round(hpsi_roof["achieved_gbs"] / hbm_peak, 4)

    # ---- e2e through the C ABI with pinned host buffers (FP64 host data)
    e2e = None
    if not args.no_e2e:
        host = torch.empty((nb, ngw), dtype=torch.complex128, pin_memory=True)
        host.copy_(torch.from_numpy(np.ascontiguousarray(psi.T)))
        hx = host.numpy()  # pinned, Fortran-ordered ngw x nb when viewed transposed
        from pspw._lib import check, lib
        L = lib()
        for _ in range(2):
            hx[:] = psi.T
            check(L.pspw_chebyfilt(cell.handle, hx.ctypes.data, ngw, nb, DEGREE, LB, UB, prec))
        e_steps = max(3, args.steps // 2)
        tt = []
        for _ in range(e_steps):
            hx[:] = psi.T  # the filter overwrites X; restore (host memcpy, not timed)
            t0 = time.perf_counter()
            check(L.pspw_chebyfilt(cell.handle, hx.ctypes.data, ngw, nb, DEGREE, LB, UB, prec))
            tt.append(time.perf_counter() - t0)
        et = replica.max_over_ranks(sum(tt) / len(tt), device=dev)
        e2e = {"value": round(replica.weak_throughput(bytes_step, world, et) / 1e9, 2),
               "unit": "GB/s",
               "h2d_bytes_per_step": ngw * nb * 16, "d2h_bytes_per_step": ngw * nb * 16,
               "seconds_per_step": round(et, 6),
               "path": "pspw_chebyfilt (C ABI, host FP64 X, FP32 on device)" if not fp64
               else "pspw_chebyfilt (C ABI, host FP64 X, FP64 on device)"}

    # ---- the same filter in FP64 (complex128 throughout, the reference's
    # arithmetic), timed the same way: the like-for-like line against the
    # reference arm, which computes in complex128
    fp64_line = None
    if not fp64 and not args.no_fp64_line:
        fp64_line = _time_fp64_filter(args, cell, psi, dev, stream, flush, ngw, nb, nnr, nat,
                                      bytes_step, world, hbm_peak, hbm_src)

    return dict(value=value, ms=ms_max, wall=t_wall, launches=launches, roof=roof,
                hpsi_roof=hpsi_roof, kernels_ms=kernels_ms, clocks=clocks.summary(), e2e=e2e,
                ngw=ngw, nb=nb, sizes=sizes, fp64=fp64_line)


def _time_fp64_filter(args, cell, psi, dev, stream, flush, ngw, nb, nnr, nat, bytes_step32,
                      world, hbm_peak, hbm_src):
    """The bench step with PREC_F64 on a complex128 block: W warm-up steps,
    K timed steps (CUDA events on the cell stream, L2 flushed between steps
    outside the timed interval).  Reports the line's metric (FP32 byte
    model, so it compares with the complex128 reference arm as work per
    second) and the FP64 byte model's GB/s and fraction of the HBM peak."""
    import torch
    from pspw import PREC_F64, replica
    x0 = torch.from_numpy(np.ascontiguousarray(psi.T)).to(torch.complex128).to(dev)
    x = torch.empty_like(x0)

    def step():
        x.copy_(x0)
        cell.chebyfilt_dev(x, ngw, ngw, nb, DEGREE, LB, UB, PREC_F64)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    fams = (3, 5, 7, 8, 9)
    cell.timing_reset()
    cell.timing_enable(sum(1 << f for f in fams))
    l0 = cell.kernel_launches()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    replica.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            step()
            evs[k][1].record(stream)
    torch.cuda.synchronize()
    cell.timing_enable(0)
    launches = (cell.kernel_launches() - l0) // args.steps
    fam = {f: cell.timing_read(f) for f in fams}
    ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    ms_max = replica.max_over_ranks(ms, device=dev)
    b64 = hpsi_bytes_model(ngw, nnr, nb, nat, fp64=True)
    hpsi_ms = ms_max / DEGREE
    names = {3: "k_sticks_inv", 5: "k_plane", 7: "k_sticks_fwd", 8: "projection",
             9: "back-projection"}
    return {"dtype": "c128", "ms_per_step": round(ms_max, 4),
            "value": round(replica.weak_throughput(bytes_step32, world, ms_max * 1e-3) / 1e9, 2),
            "unit": "GB/s (the line's FP32 byte model)",
            "hpsi": {"bytes_per_hpsi": b64, "ms_per_hpsi": round(hpsi_ms, 4),
                     "achieved_gbs": round(b64 / (hpsi_ms * 1e-3) / 1e9, 1),
                     "frac_of_measured_hbm": round(b64 / (hpsi_ms * 1e-3) / 1e9 / hbm_peak, 4),
                     "peak_source": hbm_src},
            "kernels_ms_per_step": {names[f]: round(fam[f][0] / args.steps, 4)
                                    for f in fams if fam[f][1] > 0},
            "gpu_launches": launches}


def _ncu_traffic(workload, kernel, prec):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu
    summary (lines `workload kernel prec bytes`), or None if not captured."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if (len(parts) >= 4 and parts[0] == workload and parts[1] == kernel
                and parts[2] == prec):
            try:
                return int(float(parts[3]))
            except ValueError:
                return None
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--prec", default="f32", choices=["f32", "f64"])
    ap.add_argument("--workload", default="si64")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--nl-overlap", default="auto", choices=sorted(OVERLAP_MODES),
                    help="projection concurrent with the FFT passes (on), after them (off), "
                         "or the engine's per-precision default (auto)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-line", action="store_true",
                    help="si64/si216: skip the complex128 filter timed beside the FP32 one")
    ap.add_argument("--rate", type=float, default=4.0, help="serve: arrivals per second")
    ap.add_argument("--jobs", type=int, default=24, help="serve: jobs per precision form")
    ap.add_argument("--slots", type=int, default=8, help="serve: concurrent jobs")
    ap.add_argument("--cells", type=int, default=32, help="batch: cells per batch")
    ap.add_argument("--warm-start", action="store_true",
                    help="eig-si216: start the solvers (lobpcg_ortho only) from a "
                         "Chebyshev-filtered block instead of the random start")
    ap.add_argument("--solvers", default="lobpcg,davidson",
                    help="eig-si216: comma-separated solvers (lobpcg, davidson, "
                         "lobpcg_ortho)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    config = {"workload": WORKLOAD, "cell": "Si64 diamond-cubic, synthetic pseudopotential",
              "grid": [64, 64, 64], "ngw": 23847, "bands": 144, "filter_degree": DEGREE,
              "filter_window_ha": [LB, UB], "global_batch": 144 * world,
              "parallelism": f"replica x{world} (bands independent, no collective)",
              "l2": "flushed between steps (256 MB write, outside the timed interval)"}

    if args.workload == "dense":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "a microbenchmark of the engine's dense kernels against "
                                  "cuBLAS/cuSOLVER; no CPU counterpart is timed"}))
            return
        run_dense(args, rank, world, local_rank)
        return

    if args.workload == "batch":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference applies H*psi to one cell per process"}))
            return
        run_batch(args, rank, world, local_rank)
        return

    if args.workload == "serve":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no serving loop; it runs one SCF job per "
                                  "process"}))
            return
        run_serve(args, rank, world, local_rank)
        return

    if args.workload in ROW_WORKLOADS:
        if args.impl == "reference":
            if rank != 0:
                return
            import tempfile
            w = ROW_WORKLOADS[args.workload]
            ref, why = row_reference(args, w, tempfile.mkdtemp(prefix="pspw_row_ref_"))
            if ref is None:
                print(json.dumps({"impl": "reference", "unavailable": why}))
                return
            print(json.dumps({"impl": "reference", "metric": args.workload, "value":
                              round(ref["value"], 6), "unit": ref["unit"], "n_gpus": args.gpus,
                              "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": round(ref["seconds_per_step"] * 1e3, 3),
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "c128", "data": "synthetic",
                              "config": {"workload": f"{args.workload}: {w['text']}"},
                              "cpu_baseline": {k: ref[k] for k in ("value", "unit", "cores",
                                                                   "kind", "sample")},
                              "e2e": {"value": round(ref["value"], 6), "unit": ref["unit"],
                                      "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
            return
        import torch
        if world > 1:
            import datetime
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                                 device_id=torch.device("cuda", local_rank))
        if ROW_WORKLOADS[args.workload]["kind"] == "converge":
            run_converge(args, rank, world, local_rank)
        elif ROW_WORKLOADS[args.workload]["kind"] == "eigsolve":
            run_eigsolve(args, rank, world, local_rank)
        else:
            run_row(args, rank, world, local_rank)
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return

    if args.impl == "reference":
        if rank != 0:
            return
        ref, why = reference_sample(args.steps, args.warmup)
        if ref is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": round(ref["value"], 4), "unit": "GB/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ref["seconds_per_step"] * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": config,
            "cpu_baseline": {k: ref[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": round(ref["value"], 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return

    import torch
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    r = run_engine(args, rank, world, local_rank)
    if args.workload != "si64":  # the line names the cell it ran on
        s = r["sizes"]
        grid = [s["n1"], s["n2"], s["n3"]]
        config = dict(config, grid=grid, ngw=r["ngw"], bands=r["nb"],
                      global_batch=r["nb"] * world,
                      cell=f"{args.workload} diamond-cubic, synthetic pseudopotential",
                      workload=(f"Chebyshev filter (degree {DEGREE}, chebyfilt.cpp) on "
                                f"{args.workload}: {s['nat']} atoms, grid "
                                f"{grid[0]}x{grid[1]}x{grid[2]}, NGW {r['ngw']}, {r['nb']} "
                                f"bands, s+p KB projectors"))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref, why = reference_sample(steps=1, warmup=0)
        cpu = ({k: (round(v, 4) if isinstance(v, float) else v) for k, v in ref.items()
                if k in ("value", "unit", "cores", "kind", "sample")} if ref else
               {"value": None, "unavailable": why})
    if rank == 0:
        out = {
            "metric": METRIC, "value": round(r["value"], 2), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms"], 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128" if args.prec == "f64" else "c64", "data": "synthetic",
            "config": config, "roofline": r["roof"], "hpsi": r["hpsi_roof"],
            "kernels_ms_per_step": r["kernels_ms"], "cpu_baseline": cpu, "e2e": r["e2e"],
            "gpu_launches": r["launches"], "clocks": r["clocks"],
            "wall_s_timed": round(r["wall"], 4),
        }
        if r["fp64"]:
            out["fp64"] = r["fp64"]
        print(json.dumps(out))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
