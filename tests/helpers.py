"""Shared test plumbing: run one case through the CUDA engine and through a CPU oracle."""
import numpy as np

import ifosb
from ifosb import synth
from pyoracle import IfoParams


def ifo_params(c, nmech=None):
    p = c["params"]
    return IfoParams(nx=p.nx, ny=p.ny, nz=p.nz, dx=p.dx, dy=p.dy, dz=p.dz, dt=p.dt, nt=p.nt, time=p.time,
                     fdcoeff=p.fdcoeff, free_surf=p.free_surf, fw=p.fw,
                     nmech=p.nmech if nmech is None else nmech, ndt=p.ndt, ndtshift=p.ndtshift,
                     vppml=c["vppml"], fpml=c["fpml"], alpha=p.alpha, beta=p.beta, source_shape=4)


def oracle_model(c, O, which="start"):
    """Moduli from the oracle's readmod (pins the host's moduli() too)."""
    vp, vs, rho = c[which]
    return O.readmod(ifo_params(c), vp, vs, rho, tau=c["tau"], fl=c["fl"])


def engine_for(c, max_shots=None, which="start", nf=None):
    p = c["params"]
    m, cp, shots = synth.build_inputs(c, which)
    nfv = len(c["finv"]) if nf is None else nf
    e = ifosb.Engine(p, max_shots=max_shots or len(shots), max_nf=nfv)
    e.set_cpml(cp)
    e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
    e.set_receivers(c["recpos"])
    e.set_frequencies(c["finv"][:nfv] if nfv else None, c["ntast"])
    return e, m, cp, shots


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
