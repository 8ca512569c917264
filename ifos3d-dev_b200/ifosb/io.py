"""The reference's seismogram, model and gradient files (C writers in
csrc/ifosb_io.c) and its file-naming rules.

Naming follows src/saveseis.c:47-64 (synthetic and observed seismograms, per rank
and merged), src/readseis.c:39-47 and src/readseis_split.c:36-38 (observed data
read back), src/outmod.c:44-46 and src/outgrad.c:44-46 (model and gradient
files). Sections are [ntr][ns] float32; receiver positions [ntr][3] grid indices.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import EARG, IfosbError, lib

SEIS_EXT = {0: "su", 1: "su", 2: "txt", 3: "bin"}  # saveseis.c:40-45
COMPONENTS = ("vx", "vy", "vz")


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _check(rc, what):
    if rc != 0:
        raise IfosbError(rc, what)


def seis_rank_file(seisfile, comp, iteration, fmt, ishot, myid, multiple_shots=True):
    """Per-rank seismogram file written by saveseis (saveseis.c:48-63)."""
    ext = SEIS_EXT[fmt]
    if multiple_shots:
        return f"{seisfile}_{comp}_it{iteration}.{ext}.shot{ishot}.{myid}"
    return f"{seisfile}_{comp}_it{iteration}.{ext}.{myid}"


def seis_merged_file(seisfile, comp, iteration, fmt, ishot):
    """File rank 0 merges the ranks' traces into (saveseis.c:86-87)."""
    return f"{seisfile}_{comp}_it{iteration}.{SEIS_EXT[fmt]}.shot{ishot}"


def obs_file(obsfile, comp, ishot, myid, multiple_shots=True):
    """Observed-data file readseis opens (readseis.c:39-47): always SU."""
    if multiple_shots:
        return f"{obsfile}_{comp}_it1.su.shot{ishot}.{myid}"
    return f"{obsfile}_{comp}.su.shot{ishot}.{myid}"


def obs_split_file(obsfile, comp, ishot):
    """External observed-data file readseis_split opens (readseis_split.c:36-38)."""
    return f"{obsfile}_{comp}_ext.su.shot{ishot}"


def write_seis(path, section, rec, *, comp=1, trace_no=None, src=None, dx, dy, dz, ndt, dt, fmt=1,
               littlebig=False):
    """outseis(): one component's [ntr][ns] section to `path` (SU, ASCII or binary)."""
    sec = _f32(section)
    ntr, ns = sec.shape
    r = _i32(rec).reshape(ntr, 3) if ntr else np.zeros((0, 3), np.int32)
    tn = None if trace_no is None else _i32(trace_no)
    s = None if src is None else _f32(src)
    _check(lib().ifosb_write_seis(os.fsencode(path), comp, _p(sec), ntr, ns, _p(r), _p(tn), _p(s), dx, dy, dz,
                                  ndt, dt, fmt, 1 if littlebig else 0), f"write_seis {path}")


def merge_seis(out, inputs, ns):
    """Rank 0's merge of per-rank SU files (saveseis.c:86-229); returns traces written."""
    arr = (C.c_char_p * max(len(inputs), 1))(*[os.fsencode(x) for x in inputs])
    n = C.c_int(0)
    _check(lib().ifosb_merge_seis(os.fsencode(out), len(inputs), arr, ns, C.byref(n)), f"merge_seis {out}")
    return n.value


def read_seis(path, ntr, ns):
    """readseis(): [ntr][ns] traces after their 240-byte headers."""
    out = np.zeros((ntr, ns), np.float32)
    _check(lib().ifosb_read_seis(os.fsencode(path), _p(out), ntr, ns), f"read_seis {path}")
    return out


def read_seis_split(path, keep, ns):
    """readseis_split(): the traces flagged 1 in `keep`, in file order."""
    k = _i32(keep)
    out = np.zeros((int(np.sum(k == 1)), ns), np.float32)
    _check(lib().ifosb_read_seis_split(os.fsencode(path), _p(out), len(k), _p(k), ns), f"read_seis_split {path}")
    return out


# file-name tag of each SEISMO component (saveseis.c:48-63; the curl is "rot")
SEISMO_FILES = {1: ("vx", "vy", "vz"), 2: ("p",), 3: ("div", "rot"), 4: ("vx", "vy", "vz", "p", "div", "rot")}


def save_seis(seisfile, sections, rec, src, *, ishot, iteration, dx, dy, dz, ndt, dt, fmt=1, obs=False,
              method=True, multiple_shots=True, trace_no=None, rank=0, nranks=1, barrier=None, seismo=1):
    """saveseis(): each rank writes its files of the SEISMO components (sections
    [ncomp][ntr][ns] in Engine.forward's order), rank 0 merges the ranks' vx, vy,
    vz files, and those rank files are removed after an inversion iteration
    (iteration > 0, METHOD, not observed data). `barrier` (callable) separates the
    writes from the merge when several ranks share the files."""
    sections = np.asarray(sections)
    ntr, ns = sections.shape[1], sections.shape[2]
    names = SEISMO_FILES[seismo]
    if sections.shape[0] != len(names):
        raise IfosbError(EARG, f"SEISMO {seismo} has {len(names)} components, got {sections.shape[0]}")
    if ntr > 0:
        for c, name in enumerate(names):
            comp = {"vx": 1, "vy": 2, "vz": 3}.get(name, 0)
            write_seis(seis_rank_file(seisfile, name, iteration, fmt, ishot, rank, multiple_shots), sections[c], rec,
                       comp=comp, trace_no=trace_no, src=src, dx=dx, dy=dy, dz=dz, ndt=ndt, dt=dt, fmt=fmt)
    if barrier:
        barrier()
    if rank == 0:
        for name in COMPONENTS:
            ins = [seis_rank_file(seisfile, name, iteration, fmt, ishot, r, True) for r in range(nranks)]
            merge_seis(seis_merged_file(seisfile, name, iteration, fmt, ishot), ins, ns)
    if barrier:
        barrier()
    if iteration > 0 and ntr > 0 and method and not obs:
        for name in COMPONENTS:
            f = seis_rank_file(seisfile, name, iteration, fmt, ishot, rank, True)
            if os.path.exists(f):
                os.remove(f)


def write_model(base, iteration, rho, pi, u, ghosted=False, idx=1, idy=1, idz=1):
    """outmod() + mergemod(): "<base>.vp_it<n>", ".vs_it<n>", ".rho_it<n>" ([z][x][y]).
    rho, pi, u: [ny][nx][nz], or the reference's ghosted [ny+2][nx+2][nz+2] with ghosted=True."""
    arrs = [_f32(a) for a in (rho, pi, u)]
    sh = arrs[0].shape
    if len(sh) != 3 or any(a.shape != sh for a in arrs):
        raise IfosbError(EARG, "rho, pi, u must be 3-D arrays of one shape")
    ny, nx, nz = (sh[0] - 2, sh[1] - 2, sh[2] - 2) if ghosted else sh
    _check(lib().ifosb_write_model(os.fsencode(base), iteration, nx, ny, nz, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]),
                                   1 if ghosted else 0, idx, idy, idz), f"write_model {base}")


def write_gradient(base, finv, iteration, grad, idx=1, idy=1, idz=1):
    """outgrad() + mergemod(): "<base>.vp_<f>Hz_it<n>", ".vs_...", ".rho_..." from [3][ny][nx][nz]."""
    g = _f32(grad)
    if g.ndim != 4 or g.shape[0] != 3:
        raise IfosbError(EARG, f"gradient of shape {g.shape}, expected [3][ny][nx][nz]")
    _, ny, nx, nz = g.shape
    _check(lib().ifosb_write_gradient(os.fsencode(base), finv, iteration, nx, ny, nz, _p(g), 0, idx, idy, idz),
           f"write_gradient {base}")


def read_hessian(base, finv, iteration, ny, nx, nz, vp0, vs0, rho0):
    """readhess(): "<base>.{vp,vs,rho}_<f>Hz_it<n>" into [3][ny][nx][nz], scaled by VP0^2 etc."""
    out = np.zeros((3, ny, nx, nz), np.float32)
    _check(lib().ifosb_read_hessian(os.fsencode(base), finv, iteration, nx, ny, nz, vp0, vs0, rho0, _p(out)),
           f"read_hessian {base}")
    return out
