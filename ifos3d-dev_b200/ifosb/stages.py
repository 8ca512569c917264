"""Multiscale inversion stages: the workflow file (INV_FILE) and the per-stage
Butterworth filter (FILT = 1).

read_inv restates readinv() (src/readinv.c:25-85). Stage g (1-based) skips g-1
lines of the file, reading them as fgets with a 255-byte buffer does (a longer
line counts as several). From there it reads, whitespace-separated:
  itmin itmax abort mute twin0 twin1 owin0 owin1 nf  finv[0] .. finv[nf-1]
The driver uses itmax and the frequencies (src/ifos3d.c:690-701); abort, mute
and the windows are read and unused, as in the reference.

filt_seis (csrc/ifosb_filter.c) is the FILT = 1 low-pass. ifos3d.c:731 applies it
to each shot's source signals and :840-855 to the observed seismograms. The
corner is the stage's highest frequency finv[nf-1].
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import EARG, IfosbError, lib


@dataclass
class WorkflowStage:
    itmin: int
    itmax: int
    abort: float
    mute: int
    twin: tuple
    owin: tuple
    finv: list = field(default_factory=list)


def _fgets_lines(text: bytes):
    """Split as successive fgets(buf, 255, f) calls would: at most 254 bytes or
    up to and including a newline per call."""
    out, i = [], 0
    while i < len(text):
        j = text.find(b"\n", i, i + 254)
        end = j + 1 if j >= 0 else min(i + 254, len(text))
        out.append(text[i:end])
        i = end
    return out


def read_inv(path: str, groupnum: int) -> WorkflowStage:
    """Stage `groupnum` (1-based) of the workflow file, as readinv() reads it."""
    if groupnum < 1:
        raise IfosbError(EARG, "stage numbers start at 1")
    with open(path, "rb") as f:
        text = f.read()
    rest = b"".join(_fgets_lines(text)[groupnum - 1:])
    tok = rest.split()
    if len(tok) < 9:
        raise IfosbError(EARG, f"{path}: stage {groupnum} has fewer than 9 fields")
    nf = int(tok[8])
    if len(tok) < 9 + nf:
        raise IfosbError(EARG, f"{path}: stage {groupnum} lists fewer than {nf} frequencies")
    f32 = lambda t: float(np.float32(float(t)))  # fscanf %f into a float
    return WorkflowStage(itmin=int(tok[0]), itmax=int(tok[1]), abort=f32(tok[2]), mute=int(tok[3]),
                         twin=(f32(tok[4]), f32(tok[5])), owin=(f32(tok[6]), f32(tok[7])),
                         finv=[f32(t) for t in tok[9:9 + nf]])


def read_workflow(path: str, nstages: int) -> list:
    """Stages 1..nstages of a workflow file."""
    return [read_inv(path, g) for g in range(1, nstages + 1)]


def filt_seis(data, finv, dt, order=4, highpass=False):
    """FILT = 1: Butterworth filter of each trace of a [ntr][ns] float32 array
    (returns a filtered copy; the last sample of each trace is kept, as in the
    reference)."""
    a = np.array(data, dtype=np.float32, order="C", copy=True)
    if a.ndim != 2:
        raise IfosbError(EARG, "filt_seis expects [ntr][ns]")
    rc = lib().ifosb_filt_seis(a.ctypes.data_as(C.c_void_p), a.shape[0], a.shape[1], float(finv), float(dt),
                               int(order), 1 if highpass else 0)
    if rc != 0:
        raise IfosbError(rc, "filt_seis")
    return a


def resample(field, spacing, shape, new_spacing):
    """A [ny][nx][nz] field on a grid of spacing (dx, dy, dz) resampled onto a
    grid of `shape` (ny, nx, nz) and spacing new_spacing (ifosb_resample:
    trilinear at the cell positions, constant outside)."""
    a = np.ascontiguousarray(field, np.float32)
    ny, nx, nz = a.shape
    my, mx, mz = shape
    out = np.zeros((my, mx, mz), np.float32)
    rc = lib().ifosb_resample(a.ctypes.data_as(C.c_void_p), nx, ny, nz, *[float(v) for v in spacing],
                              out.ctypes.data_as(C.c_void_p), mx, my, mz, *[float(v) for v in new_spacing])
    if rc != 0:
        raise IfosbError(rc, "resample")
    return out


def resample_model(vp, vs, rho, spacing, shape, new_spacing):
    """vp, vs, rho of one multiscale grid carried to the next (velocities and
    density are interpolated, not the moduli)."""
    return tuple(resample(f, spacing, shape, new_spacing) for f in (vp, vs, rho))
