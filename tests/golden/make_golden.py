"""Generate the golden fixtures in this directory from the REFERENCE itself.

Every output is produced by the reference's own functions (oracle/_ref, built
from the reference sources by oracle/Makefile and driven in the call order of
src/ifos3d.c): model scaling (readmod), CPML profiles (CPML_coeff), wavelets
(wavelet), the forward loop, residual(), the back-propagation and gradient_F.
The reference ships no tests or golden vectors, so these fixtures are what pins
the C restatement and the CUDA engine when the reference is not available.

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "ifos3d-dev_b200")]

from pyoracle import IfoParams, Oracle  # noqa: E402

CASES = {
    # elastic, free surface, explosive source, receivers incl. one in the CPML frame
    "elastic_fs": dict(nmech=0, free_surf=1, fdcoeff=2, srcs=[[8, 5, 7, 0.0, 600.0, 1.0, 1]]),
    # viscoelastic L=1, CPML on all six faces, Taylor coefficients
    "visco1_cpml": dict(nmech=1, free_surf=0, fdcoeff=1, srcs=[[9, 9, 6, 0.0002, 500.0, 2.0, 1]]),
    # body forces: a single force in x and the custom-angle force next to an explosion
    "forces": dict(nmech=0, free_surf=1, fdcoeff=2, alpha=30.0, beta=60.0,
                   srcs=[[7, 6, 8, 0.0, 550.0, 1.0, 2], [10, 12, 5, 0.0001, 650.0, 1.5, 5],
                         [3, 3, 3, 0.0, 700.0, 0.7, 1]]),
}
NX, NY, NZ, FW, NT = 16, 18, 14, 4, 80
FINV = np.array([350.0, 600.0], np.float32)


def params(c):
    dt = np.float32(1e-4)
    return IfoParams(nx=NX, ny=NY, nz=NZ, dx=1.0, dy=1.0, dz=1.0, dt=dt, nt=NT,
                     time=np.float32(np.float32(NT - 1) * dt), fdcoeff=c["fdcoeff"], free_surf=c["free_surf"],
                     fw=FW, nmech=c["nmech"], ndt=1, ndtshift=0, vppml=3000.0, fpml=500.0,
                     alpha=c.get("alpha", 0.0), beta=c.get("beta", 0.0), source_shape=4)


def checksums(a):
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    return np.stack([a.sum(1), np.abs(a).sum(1), (a * a).sum(1)], 1)


def main():
    R = Oracle("ref")
    rng = np.random.default_rng(20261203)
    for name, c in CASES.items():
        p = params(c)
        shp = (NY, NX, NZ)
        vp = (3000 * (1 + 0.04 * rng.standard_normal(shp))).astype(np.float32)
        vs = (vp / np.float32(1.75)).astype(np.float32)
        rho = (2100 * (1 + 0.04 * rng.standard_normal(shp))).astype(np.float32)
        fl = np.array([300.0], np.float32) if c["nmech"] else None
        tau = 0.04 if c["nmech"] else 0.0
        m = R.readmod(p, vp, vs, rho, tau=tau, fl=fl)
        cp = R.cpml_coeff(p)
        srcpos = np.array(c["srcs"], np.float32)
        sig = R.wavelet(p, srcpos)
        rec = np.array([[4, 1, 4], [8, 1, 7], [12, 1, 10], [6, 9, 5], [2, 15, 12], [14, 16, 2]], np.int32)
        f = R.forward(p, m, cp, srcpos, sig, rec, FINV, 1, True, True)
        obs = (f["sections"] * np.float32(0.85) + np.float32(1e-9)).astype(np.float32)
        diff, l2 = R.residual(p, obs, f["sections"])
        b = R.adjoint(p, m, cp, rec, diff, FINV, 1, True)
        g = R.gradient(p, m, FINV, f["dft"], b["dft"])
        out = dict(vp=vp, vs=vs, rho_in=rho, tau=np.float32(tau), fl=fl if fl is not None else np.zeros(0, np.float32),
                   nmech=c["nmech"], free_surf=c["free_surf"], fdcoeff=c["fdcoeff"], alpha=c.get("alpha", 0.0),
                   beta=c.get("beta", 0.0), nx=NX, ny=NY, nz=NZ, fw=FW, nt=NT, finv=FINV,
                   rho=m["rho"], pi=m["pi"], u=m["u"],
                   taus=m["taus"] if c["nmech"] else np.zeros(0, np.float32),
                   taup=m["taup"] if c["nmech"] else np.zeros(0, np.float32),
                   eta=m["eta"] if c["nmech"] else np.zeros(0, np.float32),
                   cpml=cp, srcpos=srcpos, signals=sig, recpos=rec, obs=obs,
                   sections=f["sections"], diff=diff, l2=np.float32(l2), grad=g,
                   dft_ck=checksums(f["dft"].reshape(12, -1)), bdft_ck=checksums(b["dft"].reshape(12, -1)),
                   state_ck=checksums(f["state"]), bstate_ck=checksums(b["state"]))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "sections max", float(np.abs(f["sections"]).max()), "grad max", float(np.abs(g).max()))


if __name__ == "__main__":
    main()
