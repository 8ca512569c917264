"""Seeded synthetic workloads with the shapes of the engine's benchmark cases.

No field data or checkpoints are available, so models, sources and receivers
are generated here with the sizes and value distributions of each case:

  elastic128  128^3, DH=1 m, DT=1e-4 s, NT=2000, free surface, FW=10 CPML;
              vp=3000, vs=vp/sqrt(3), rho=2000; true model with a 15 m sphere
              (+10 % vp, vs) at the centre; one explosive sin^3 source (fc=100 Hz)
              at x=z=64 m, y=10 m; 25 receivers on a 5x5 x-z grid at j=1;
              DFT at 60 and 100 Hz, ntast=1.
  visco256    256^3, L=3 mechanisms, Q=50 over 20-200 Hz, 8 seeded flat layers
              vp 2500-4500, vs=vp/1.8, rho 1800-2600; sin^3 fc=80 Hz; NT=3000;
              400 surface receivers; forward modelling only.
  elastic192  192x192x160, vp 2000->3500 linear with depth, +-3 % Gaussian random
              field (correlation length 8 cells) on vp, vs, rho; 4 shots; DFT at
              20, 40, 60, 80, 100 Hz.
  visco384    384x384x256, L=3, 3 Gaussian blobs in a layered background, 32 shots
              on an 8x4 surface grid, 1024 receivers, 4 frequencies.

The time step count follows the reference's rounding: NT = ceil(TIME/DT), so
TIME=0.19995 gives NT=2000 (0.2 would give 2001 in float arithmetic).
"""
from __future__ import annotations

import math

import numpy as np

from . import Params, make_params, moduli

PI = 3.141592653589793


def q_tau_fit(q: float, fmin: float, fmax: float, nmech: int):
    """Constant-Q fit with the tau-method (Blanch, Robertsson & Symes 1995):
    relaxation frequencies log-spaced over the band, and the single tau that
    minimises sum_w (Q^-1(w) - 1/q)^2 for the linearised
    Q^-1(w) = tau * sum_l w*t_l / (1 + w^2 t_l^2), t_l = 1/(2 pi f_l).
    Returns (tau, fl[nmech])."""
    fl = np.exp(np.linspace(math.log(fmin), math.log(fmax), nmech)) if nmech > 1 else np.array([math.sqrt(fmin * fmax)])
    w = 2 * PI * np.exp(np.linspace(math.log(fmin), math.log(fmax), 64))
    tl = 1.0 / (2 * PI * fl)
    a = (w[:, None] * tl[None, :] / (1 + (w[:, None] * tl[None, :]) ** 2)).sum(axis=1)
    tau = float((a / q).sum() / (a * a).sum())
    return tau, fl.astype(np.float32)


def tau_of_q(q, fmin, fmax, nmech):
    """The tau method's relaxation time for a Q field: the fit is linear in 1/Q
    (q_tau_fit), so tau = tau(Q=1) / Q, in float64 then rounded to float32.
    Returns (tau[...], fl[nmech])."""
    tau1, fl = q_tau_fit(1.0, fmin, fmax, nmech)
    return (tau1 / np.asarray(q, np.float64)).astype(np.float32), fl


def q_moduli(p, vp, vs, rho, tau, fl):
    """readmod's relaxed moduli (src/readmod.c:48-65, generalised to L mechanisms)
    with a relaxation time per cell (taus = taup = tau), in readmod's arithmetic:
    pts_l = 1 / (2 pi FL_l) and ws = 2 pi FL[1] rounded to float, the sum
    sum_l ws^2 pts_l^2 tau / (1 + ws^2 pts_l^2) with float products and double
    quotients, pi = vp^2 rho / (1 + sum) the same way. Returns dict(rho, pi, u,
    taus, taup, eta) as float32 arrays."""
    L = p.nmech
    fl = np.asarray(fl, np.float32)
    pts = (1.0 / (2.0 * PI * fl.astype(np.float64))).astype(np.float32)
    ws = np.float32(2.0 * PI * float(fl[0]))
    tau = np.asarray(tau, np.float32)
    acc = np.zeros(tau.shape, np.float32)
    for t in pts[:L]:
        w2t2 = np.float32(np.float32(np.float32(ws * ws) * t) * t)
        num = (w2t2 * tau).astype(np.float32)
        acc = (acc.astype(np.float64) + num.astype(np.float64) / (1.0 + np.float64(w2t2))).astype(np.float32)
    den = 1.0 + acc.astype(np.float64)
    vp, vs, rho = (np.asarray(a, np.float32) for a in (vp, vs, rho))
    pi = ((vp * vp * rho).astype(np.float64) / den).astype(np.float32)
    u = ((vs * vs * rho).astype(np.float64) / den).astype(np.float32)
    eta = (np.float32(p.dt) / pts[:L]).astype(np.float32)
    return dict(rho=rho, pi=pi, u=u, taus=tau.copy(), taup=tau.copy(), eta=eta)


def _grid_receivers(nx, nz, n_side, j, margin):
    xs = np.linspace(margin, nx - margin + 1, n_side).round().astype(int)
    zs = np.linspace(margin, nz - margin + 1, n_side).round().astype(int)
    return np.array([[x, j, z] for x in xs for z in zs], np.int32)


def _src(i, j, k, fc, amp=1.0, tshift=0.0, stype=1):
    return np.array([[i, j, k, tshift, fc, amp, stype]], np.float32)


def _gauss_field(shape, corr, rng):
    """Unit-variance Gaussian random field with a Gaussian correlation of `corr` cells."""
    noise = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) for n in shape]
    kk = sum(np.meshgrid(*[ki ** 2 for ki in k], indexing="ij"))
    spec = np.fft.fftn(noise) * np.exp(-2 * (PI * corr) ** 2 * kk / 4)
    f = np.real(np.fft.ifftn(spec))
    return (f / f.std()).astype(np.float32)


def case(name: str, seed: int = 1234, nt: int | None = None, nshots: int | None = None, grid=None):
    """A workload dict: params, true/start velocity models, moduli, shots, receivers, frequencies.
    grid (visco384 only): (NX, NY, NZ) instead of 384 x 256 x 384, for small profiling runs."""
    rng = np.random.default_rng(seed)
    if name == "elastic128":
        n, fw = 128, 10
        nt = nt or 2000
        p = make_params(n, n, n, dh=1.0, dt=1e-4, nt=nt, fdcoeff=2, free_surf=1, fw=fw, nmech=0)
        vp0 = np.full((n, n, n), 3000.0, np.float32)
        vs0 = (vp0 / np.float32(math.sqrt(3.0))).astype(np.float32)
        rho0 = np.full((n, n, n), 2000.0, np.float32)
        jj, ii, kk = np.meshgrid(*(np.arange(1, n + 1),) * 3, indexing="ij")
        c = (n + 1) / 2.0
        sphere = (jj - c) ** 2 + (ii - c) ** 2 + (kk - c) ** 2 <= 15.0 ** 2
        vp1, vs1 = vp0.copy(), vs0.copy()
        vp1[sphere] *= np.float32(1.1)
        vs1[sphere] *= np.float32(1.1)
        shots = [_src(64, 10, 64, 100.0)]
        rec = _grid_receivers(n, n, 5, 1, 24)
        finv, ntast, vppml, fpml, fc = [60.0, 100.0], 1, 3000.0, 100.0, 100.0
        true = (vp1, vs1, rho0)
        start = (vp0, vs0, rho0)
        tau, fl = 0.0, None
    elif name == "visco256":
        n, fw = 256, 10
        nt = nt or 3000
        tau, fl = q_tau_fit(50.0, 20.0, 200.0, 3)
        p = make_params(n, n, n, dh=1.0, dt=1e-4, nt=nt, fdcoeff=2, free_surf=1, fw=fw, nmech=3)
        bounds = np.sort(rng.choice(np.arange(16, n - 16), 7, replace=False))
        vps = rng.permutation(np.linspace(2500, 4500, 8)).astype(np.float32)
        rhos = (1800 + (vps - 2500) / 2000 * 800).astype(np.float32)
        layer = np.searchsorted(bounds, np.arange(1, n + 1), side="right")
        vp = np.broadcast_to(vps[layer][:, None, None], (n, n, n)).astype(np.float32)
        rho = np.broadcast_to(rhos[layer][:, None, None], (n, n, n)).astype(np.float32)
        vs = (vp / np.float32(1.8)).astype(np.float32)
        shots = [_src(128, 10, 128, 80.0)]
        rec = _grid_receivers(n, n, 20, 1, 24)
        finv, ntast, vppml, fpml, fc = [], 1, 4500.0, 80.0, 80.0
        true = start = (vp, vs, rho)
    elif name == "elastic192":
        nx, ny, nz, fw = 192, 192, 160, 10
        nt = nt or 2000
        p = make_params(nx, ny, nz, dh=1.0, dt=1e-4, nt=nt, fdcoeff=2, free_surf=1, fw=fw, nmech=0)
        depth = np.linspace(2000, 3500, ny, dtype=np.float32)[:, None, None]
        bg_vp = np.broadcast_to(depth, (ny, nx, nz)).astype(np.float32)
        pert = 0.03 * _gauss_field((ny, nx, nz), 8.0, rng)
        vp1 = (bg_vp * (1 + pert)).astype(np.float32)
        vs1 = (vp1 / np.float32(math.sqrt(3.0))).astype(np.float32)
        rho1 = ((1700 + 0.2 * bg_vp) * (1 + pert)).astype(np.float32)
        vs0 = (bg_vp / np.float32(math.sqrt(3.0))).astype(np.float32)
        rho0 = (1700 + 0.2 * bg_vp).astype(np.float32)
        nsh = nshots or 4
        xs = np.linspace(40, nx - 40, nsh).round().astype(int)
        shots = [_src(int(x), 10, nz // 2, 100.0) for x in xs]
        rec = _grid_receivers(nx, nz, 8, 1, 20)
        finv, ntast, vppml, fpml, fc = [20.0, 40.0, 60.0, 80.0, 100.0], 1, 3500.0, 100.0, 100.0
        true = (vp1, vs1, rho1)
        start = (bg_vp, vs0, rho0)
        tau, fl = 0.0, None
    elif name == "visco384":
        nx, ny, nz, fw = tuple(grid) + (10,) if grid else (384, 256, 384, 10)
        nt = nt or 2000
        tau, fl = q_tau_fit(50.0, 20.0, 200.0, 3)
        p = make_params(nx, ny, nz, dh=1.0, dt=1e-4, nt=nt, fdcoeff=2, free_surf=1, fw=fw, nmech=3)
        depth = np.linspace(2500, 4000, ny, dtype=np.float32)[:, None, None]
        vp = np.broadcast_to(depth, (ny, nx, nz)).astype(np.float32).copy()
        jj, ii, kk = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz), indexing="ij")
        for _ in range(3):
            cj, ci, ck = rng.uniform(60, ny - 60), rng.uniform(60, nx - 60), rng.uniform(60, nz - 60)
            vp *= 1 + 0.1 * np.exp(-((jj - cj) ** 2 + (ii - ci) ** 2 + (kk - ck) ** 2) / (2 * 20.0 ** 2))
        vp = vp.astype(np.float32)
        vs = (vp / np.float32(1.8)).astype(np.float32)
        rho = (1700 + 0.2 * vp).astype(np.float32)
        nsh = nshots or 32
        gx = np.linspace(60, nx - 60, 8).round().astype(int)
        gz = np.linspace(60, nz - 60, 4).round().astype(int)
        shots = [_src(int(x), 10, int(z), 80.0) for x in gx for z in gz][:nsh]
        rec = _grid_receivers(nx, nz, 32, 1, 24)
        finv, ntast, vppml, fpml, fc = [20.0, 40.0, 60.0, 80.0], 1, 4500.0, 80.0, 80.0
        true = start = (vp, vs, rho)
    else:
        raise KeyError(name)
    return dict(name=name, params=p, true=true, start=start, tau=tau, fl=fl, shots=shots, recpos=rec,
                finv=np.array(finv, np.float32), ntast=ntast, vppml=vppml, fpml=fpml, fc=fc)


def small_case(nx=24, ny=26, nz=22, nt=120, fw=5, free_surf=1, nmech=0, fdcoeff=2, seed=0, nshots=1,
               nsrc=1, ntr=9, stype=1, finv=(300.0, 500.0)):
    """A small heterogeneous case for parity tests (sizes the CPU oracle runs in seconds)."""
    rng = np.random.default_rng(seed)
    p = make_params(nx, ny, nz, dh=1.0, dt=1e-4, nt=nt, fdcoeff=fdcoeff, free_surf=free_surf, fw=fw, nmech=nmech)
    shp = (ny, nx, nz)
    vp = (3000 * (1 + 0.05 * rng.standard_normal(shp))).astype(np.float32)
    vs = (vp / np.float32(math.sqrt(3.0))).astype(np.float32)
    rho = (2000 * (1 + 0.05 * rng.standard_normal(shp))).astype(np.float32)
    tau, fl = (q_tau_fit(50.0, 100.0, 1000.0, nmech) if nmech else (0.0, None))
    shots = []
    for s in range(nshots):
        src = []
        for l in range(nsrc):
            i, j, k = rng.integers(3, nx - 2), rng.integers(2, ny - 2), rng.integers(3, nz - 2)
            src.append([i, j, k, 0.0005 * l, 500.0 + 50 * s, 1.0 + l, stype if l == 0 else 1])
        shots.append(np.array(src, np.float32))
    rec = np.stack([rng.integers(1, nx + 1, ntr), np.ones(ntr, int), rng.integers(1, nz + 1, ntr)], 1).astype(np.int32)
    rec[-1] = [2, ny - 2, 2]  # one receiver inside the CPML frame
    return dict(name="small", params=p, true=(vp, vs, rho), start=(vp, vs, rho), tau=tau, fl=fl, shots=shots,
                recpos=rec, finv=np.array(finv, np.float32), ntast=1, vppml=3000.0, fpml=500.0, fc=500.0)


def build_inputs(c: dict, which: str = "start"):
    """Moduli (readmod arithmetic), CPML profiles and per-shot wavelets of a case."""
    from . import cpml_coeff, wavelet
    p: Params = c["params"]
    vp, vs, rho = c[which]
    m = moduli(p, vp, vs, rho, tau=c["tau"], fl=c["fl"])
    cp = cpml_coeff(p, c["vppml"], c["fpml"])
    shots = [(sp, wavelet(p, 4, sp)) for sp in c["shots"]]
    return m, cp, shots
