"""Oracle runs of many shots in parallel worker processes — TEST INFRASTRUCTURE.

Large-grid parity tests need the CPU oracle for several shots of a full
benchmark grid. The reference build (oracle/_ref) is single-threaded, so each
shot runs in its own spawned process (spawned, never forked: the parent may
already hold a CUDA context). A worker runs one shot's forward, residual and
adjoint, and writes the traces, the forward and backward DFT fields and the
residual to .npy files in a scratch directory; the parent then forms the
gradient in the reference's shot order (gradient_F accumulates shot by shot
into one float array, with double intermediates, so per-shot pieces cannot be
summed afterwards and give the same bits).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _paths():
    for p in (os.path.join(ROOT, "ifos3d-dev_b200"), os.path.join(ROOT, "oracle"), HERE):
        if p not in sys.path:
            sys.path.insert(0, p)


def _shot_worker(args):
    """forward (+ residual + adjoint when obs is given) of one shot; arrays to files."""
    kind, threads, p_fields, m, cp, sp, sig, recpos, finv, ntast, obs, out_dir, s = args
    _paths()
    from pyoracle import IfoParams, Oracle
    O = Oracle(kind, threads=threads)
    p = IfoParams(**p_fields)
    nf = 0 if finv is None else len(finv)
    f = O.forward(p, m, cp, sp, sig, recpos, finv if nf else None, ntast, want_dft=nf > 0)
    np.save(os.path.join(out_dir, f"sec{s}.npy"), f["sections"])
    if nf:
        np.save(os.path.join(out_dir, f"fdft{s}.npy"), f["dft"])
    if obs is not None and nf:
        d, l2 = O.residual(p, obs, f["sections"])
        np.save(os.path.join(out_dir, f"diff{s}.npy"), d)
        b = O.adjoint(p, m, cp, recpos, d, finv, ntast)
        np.save(os.path.join(out_dir, f"bdft{s}.npy"), b["dft"])
    return s


def params_dict(ip) -> dict:
    return {name: getattr(ip, name) for name, _ in ip._fields_}


def run_shots(kind, ip, m, cp, shots, recpos, finv, ntast, obs, out_dir, procs, threads=1):
    """Run every shot (index s: shots[s], obs[s] or None) in `procs` spawned
    worker processes; the results are in out_dir (sec{s}, fdft{s}, diff{s}, bdft{s})."""
    jobs = [(kind, threads, params_dict(ip), m, cp, sp, sig, recpos, finv, ntast,
             None if obs is None else obs[s], out_dir, s) for s, (sp, sig) in enumerate(shots)]
    with mp.get_context("spawn").Pool(max(1, min(procs, len(jobs)))) as pool:
        return pool.map(_shot_worker, jobs)


def load(out_dir, name, s):
    return np.load(os.path.join(out_dir, f"{name}{s}.npy"))
