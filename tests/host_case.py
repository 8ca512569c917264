"""Input directories in the reference's own formats for the drop-in host test —
TEST INFRASTRUCTURE.

write_case() lays out what ifos3d reads (src/read_par_json.c, readmod.c,
sources.c, receiver.c, readinv.c): a JSON parameter file, READMOD=1 model files
(float32, loops z outer, x, y inner: readmod.c:98-101), a source file (x y z
tshift fc amp, metres), a receiver file (x y z, metres), the workflow file and the
output folders. The JSON keys are the ones read_par_json looks up; the values
describe a small seeded case the CPU reference runs in seconds.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np


def _model_files(base, vp, vs, rho):
    # array order [ny][nx][nz] -> file order z outer, x, y inner
    for ext, a in (("vp", vp), ("vs", vs), ("rho", rho)):
        np.ascontiguousarray(np.transpose(a, (2, 1, 0)), np.float32).tofile(f"{base}.{ext}")


def models(nx, ny, nz, seed=3):
    """(true, start) velocity models: a smooth depth gradient with a Gaussian
    anomaly (+8 % vp, vs) in the true model."""
    rng = np.random.default_rng(seed)
    depth = np.linspace(2800.0, 3400.0, ny, dtype=np.float64)[:, None, None]
    vp0 = np.broadcast_to(depth, (ny, nx, nz)).astype(np.float64)
    jj, ii, kk = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz), indexing="ij")
    c = [rng.uniform(0.4, 0.6) * n for n in (ny, nx, nz)]
    blob = np.exp(-((jj - c[0]) ** 2 + (ii - c[1]) ** 2 + (kk - c[2]) ** 2) / (2 * 4.0 ** 2))
    vp1 = vp0 * (1 + 0.08 * blob)
    mk = lambda vp: (vp.astype(np.float32), (vp / math.sqrt(3.0)).astype(np.float32),  # noqa: E731
                     (1700.0 + 0.2 * vp).astype(np.float32))
    return mk(vp1), mk(vp0)


def write_case(d, *, method, model, nx=40, ny=40, nz=40, dh=1.0, dt=1e-4, nt=200, free_surf=0, fw=8,
               fdcoeff=2, nshots=2, finv=(400.0, 600.0), filt=0, damptype=2, lbfgs=0, seismo=1,
               seis_file="su/cal", obs_file="su_obs/obs", stype=1, mfile="model/start", nshots_step=None):
    """One run directory. model = (vp, vs, rho) [ny][nx][nz] float32 arrays."""
    for sub in ("in_and_out", "model", "su", "su_obs", "grad"):
        os.makedirs(os.path.join(d, sub), exist_ok=True)
    _model_files(os.path.join(d, mfile), *model)
    # sources: a line of shots at depth 6 cells (metres; sources.c:37-41 subtracts REFSRC)
    xs = np.linspace(12, nx - 12, nshots)
    with open(os.path.join(d, "sources.dat"), "w") as f:
        for x in xs:
            f.write(f"{x * dh:.3f} {6 * dh:.3f} {nz / 2 * dh:.3f} 0.0 500.0 1.0\n")
    # receivers: a 4 x 4 grid at depth 2 cells
    with open(os.path.join(d, "receiver.dat"), "w") as f:
        for x in np.linspace(fw + 3, nx - fw - 3, 4):
            for z in np.linspace(fw + 3, nz - fw - 3, 4):
                f.write(f"{x * dh:.3f} {2 * dh:.3f} {z * dh:.3f}\n")
    # one stage: min/max iterations, (unused columns), nf, frequencies (readinv.c:53)
    with open(os.path.join(d, "workflow.dat"), "w") as f:
        f.write(f"1 1 0.05 1 0.0 0.1 0.0 500.0 {len(finv)} " + " ".join(f"{x:.1f}" for x in finv) + "\n")
    time = (nt - 0.5) * dt  # NT = ceil(TIME/DT) = nt
    par = {
        "NPROCX": "1", "NPROCY": "1", "NPROCZ": "1",
        "NX": str(nx), "NY": str(ny), "NZ": str(nz), "DX": str(dh), "DY": str(dh), "DZ": str(dh),
        "FDORDER": "4", "FDCOEFF": str(fdcoeff),
        "TIME": repr(time), "DT": repr(dt),
        "SOURCE_SHAPE": "4", "SOURCE_TYPE": str(stype), "SRCREC": "1", "SOURCE_FILE": "./sources.dat",
        "RUN_MULTIPLE_SHOTS": "1",
        "READMOD": "1", "MFILE": mfile,
        "L": "0",
        "FREE_SURF": str(free_surf),
        "ABS_TYPE": "1", "FW": str(fw), "VPPML": "3000.0", "FPML": "500.0",
        "SNAP": "0",
        "SEISMO": str(seismo), "READREC": "1", "REC_FILE": "./receiver.dat",
        "REFRECX, REFRECY, REFRECZ": "0.0 , 0.0 , 0.0",
        "NDT": "1", "SEIS_FORMAT": "1", "SEIS_FILE": seis_file,
        "METHOD": str(method),
        "GRAD_FILE": "./grad/g", "MOD_OUT_FILE": "./model/out", "SEIS_OBS_FILE": obs_file, "EXTOBS": "0",
        "INV_FILE": "./workflow.dat",
        "ITMIN, ITMAX": "1 , 1", "FILT": str(filt), "NFMAX": str(len(finv)), "TAST": "100",
        "VP0, VS0, RHO0": "3000.0, 1732.0, 2300.0",
        "WEIGHT_VP,WEIGHT_VS,WEIGHT_RHO": "1.0, 1.0, 0.0",
        "NSHOTS_STEP": str(nshots_step or nshots), "TESTSTEP": "0.02",
        "DAMPTYPE": str(damptype),
        "HESS": "0", "LBFGS": str(lbfgs),
    }
    path = os.path.join(d, "run.json")
    with open(path, "w") as f:
        json.dump(par, f, indent=1)
    return path
