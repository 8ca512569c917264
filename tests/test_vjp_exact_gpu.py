"""The exact discrete vector-Jacobian product (ifosb_vjp_exact) against finite
differences.

The reference's gradient (gradient_F over a back-propagation with the forward
operator) only points downhill (test_vjp_fd_gpu.py measures how well). The
exact VJP transposes the discrete time step itself, so the derivative of the
misfit along any model direction d must equal <g, d>:

1. its FP64 forward is the engine's operator: traces within 1e-5 relative L2 of
   the FP32 engine's, and the misfit within 1e-5 of the engine's FP64 misfit;
2. against centred differences of its own FP64 misfit along 4 random
   directions of rho, pi, u (eps = 1e-5 relative, rounded to whole float32 ulps
   so that the perturbation is exactly symmetric): |<g, d> - FD| / |FD| < 1e-6 —
   the transposes are exact to rounding;
3. against centred differences of the GPU's FP32 misfit (the engine's forward
   and ifosb_residual, eps = 1e-3 relative): within 1e-3 along 8 seeded random
   directions.

The same three checks hold for the viscoelastic loop (three relaxation
mechanisms, Q = 20 fitted over 100-600 Hz; the gradient with respect to rho,
pi, u, taus and taup, the random directions mixing all five; taus and taup are
perturbed independently, so the free surface's taus - taup term is exercised).

The case is a small version of the adjoint-check configuration: a 2000-3500 m/s
depth gradient with a +-3 % Gaussian random field as the true model, the smooth
gradient as the start model, free surface, CPML on the other faces, two
explosive shots, 16 surface receivers. The random directions are smooth fields
over the whole grid (CPML frame and surface rows included) mixing vp, vs, rho.
"""
import math

import numpy as np
import pytest

import ifosb
from ifosb import synth

pytestmark = pytest.mark.gpu

NX, NY, NZ, FW, NT, FC, DT = 40, 36, 32, 6, 260, 300.0, 1e-4


def _case():
    rng = np.random.default_rng(17)
    p = ifosb.make_params(NX, NY, NZ, dh=1.0, dt=DT, nt=NT, fdcoeff=2, free_surf=1, fw=FW, nmech=0)
    depth = np.linspace(2000, 3500, NY, dtype=np.float32)[:, None, None]
    bg = np.broadcast_to(depth, (NY, NX, NZ)).astype(np.float32)
    pert = 0.03 * synth._gauss_field((NY, NX, NZ), 4.0, rng)
    true = ((bg * (1 + pert)).astype(np.float32), (bg * (1 + pert) / np.float32(math.sqrt(3))).astype(np.float32),
            ((1700 + 0.2 * bg) * (1 + pert)).astype(np.float32))
    start = (bg.copy(), (bg / np.float32(math.sqrt(3))).astype(np.float32), (1700 + 0.2 * bg).astype(np.float32))
    shots = [(sp, ifosb.wavelet(p, 4, sp)) for sp in (synth._src(x, 6, NZ // 2, FC) for x in (14, 27))]
    e = ifosb.Engine(p, max_shots=len(shots), max_nf=0)
    e.set_cpml(ifosb.cpml_coeff(p, 3500.0, FC))
    e.set_receivers(synth._grid_receivers(NX, NZ, 4, 1, 9))
    e.set_frequencies(None, 1)
    return p, rng, e, shots, true, start


def _moduli(p, vp, vs, rho):
    m = ifosb.moduli(p, vp.ravel(), vs.ravel(), rho.ravel())
    return tuple(m[k].reshape(NY, NX, NZ) for k in ("rho", "pi", "u"))


def _set_moduli(e, mods):
    e.set_model(*mods, None, None, None)


def _directions(rng, count, nfield=3):
    out = []
    for _ in range(count):
        w = rng.uniform(-1, 1, nfield)
        f = synth._gauss_field((NY, NX, NZ), 3.0, rng).astype(np.float64)
        out.append(tuple(wi * f for wi in w))
    return out


def _pm(model, d, eps):
    """model +- h with h ~ eps d model rounded to whole float32 ulps of the model,
    so that m + h and m - h are both exact float32 values (cells where one would
    cross a binade keep h = 0): the perturbation is exactly symmetric and the
    centred difference has no second-order term. Returns m+, m-, h (float64)."""
    plus, minus, half = [], [], []
    for a, dd in zip(model, d):
        a64 = a.astype(np.float64)
        ulp = np.spacing(a).astype(np.float64)
        h = np.round(eps * dd * a64 / ulp) * ulp
        p32, m32 = (a64 + h).astype(np.float32), (a64 - h).astype(np.float32)
        ok = ((p32.astype(np.float64) - a64) == h) & ((a64 - m32.astype(np.float64)) == h)
        h = np.where(ok, h, 0.0)
        plus.append((a64 + h).astype(np.float32))
        minus.append((a64 - h).astype(np.float32))
        half.append(h)
    return tuple(plus), tuple(minus), tuple(half)


def test_exact_vjp_matches_finite_differences():
    p, rng, e, shots, true, start = _case()
    _set_moduli(e, _moduli(p, *true))
    obs = e.forward(shots)
    mods = _moduli(p, *start)
    _set_moduli(e, mods)

    def gpu_misfit(m):
        _set_moduli(e, m)
        e.forward(shots, want_sections=False)
        return float(e.residual(obs).sum())

    def exact_misfit(m):
        _set_moduli(e, m)
        e.forward(shots, want_sections=False)
        e.residual(obs)
        return float(e.vjp_exact(40, want_grad=False)[1][:len(shots)].sum())

    # 1. the FP64 forward is the engine's operator
    e.forward(shots, want_sections=False)
    mis32 = e.residual(obs)
    g, mis64 = e.vjp_exact(40)
    mis64 = mis64[:len(shots)]
    assert np.all(mis32 > 0)
    assert np.allclose(mis64, mis32, rtol=1e-5, atol=0), (mis64, mis32)
    assert np.isfinite(g).all() and np.abs(g).max() > 0
    g2, _ = e.vjp_exact(7)  # the checkpoint interval changes nothing but rounding
    assert np.linalg.norm(g2 - g) <= 1e-12 * np.linalg.norm(g)
    # the same gradient with respect to rho, pi, u (undo pi = rho vp^2, u = rho vs^2)
    rho, pi, u = (a.astype(np.float64) for a in mods)
    vp, vs = np.sqrt(pi / rho), np.sqrt(u / rho)
    g_pi, g_u = g[0] / (2 * rho * vp), g[1] / (2 * rho * vs)
    g_mod = (g[2] - g_pi * vp * vp - g_u * vs * vs, g_pi, g_u)

    # 2. its own FP64 misfit along moduli directions: the transposes, to rounding
    for d in _directions(rng, 4):
        plus, minus, half = _pm(mods, d, 1e-5)
        fd = (exact_misfit(plus) - exact_misfit(minus)) / 2
        dot = sum(float((gq * hq).sum()) for gq, hq in zip(g_mod, half))
        print(f"FP64 misfit: <g,d> {dot:.12e} FD {fd:.12e} rel {abs(dot - fd) / abs(fd):.2e}")
        assert abs(dot - fd) <= 1e-6 * abs(fd)

    # 3. the GPU's FP32 misfit along vp, vs, rho directions, eps = 1e-3
    for d in _directions(rng, 8):
        plus, minus, half = _pm(start, d, 1e-3)
        fd = (gpu_misfit(_moduli(p, *plus)) - gpu_misfit(_moduli(p, *minus))) / 2
        dot = sum(float((gq * hq).sum()) for gq, hq in zip(g, half))
        print(f"FP32 misfit: <g,d> {dot:.6e} FD {fd:.6e} rel {abs(dot - fd) / abs(fd):.2e}")
        assert abs(dot - fd) <= 1e-3 * abs(fd)
    e.close()


def test_exact_vjp_viscoelastic_matches_finite_differences():
    p, rng, e, shots, true, start = _case()
    e.close()
    tau, fl = synth.q_tau_fit(20.0, 100.0, 600.0, 3)
    pv = ifosb.make_params(NX, NY, NZ, dh=1.0, dt=DT, nt=NT, fdcoeff=2, free_surf=1, fw=FW, nmech=3)
    e = ifosb.Engine(pv, max_shots=len(shots), max_nf=0)
    e.set_cpml(ifosb.cpml_coeff(pv, 3500.0, FC))
    e.set_receivers(synth._grid_receivers(NX, NZ, 4, 1, 9))
    e.set_frequencies(None, 1)

    def vmods(vp, vs, rho):
        m = ifosb.moduli(pv, vp.ravel(), vs.ravel(), rho.ravel(), tau=tau, fl=fl)
        return tuple(m[k].reshape(NY, NX, NZ) for k in ("rho", "pi", "u", "taus", "taup")), m["eta"]

    mt, eta = vmods(*true)
    e.set_model(*mt, eta)
    obs = e.forward(shots)
    mods, _ = vmods(*start)

    def gpu_misfit(m):
        e.set_model(*m, eta)
        e.forward(shots, want_sections=False)
        return float(e.residual(obs).sum())

    def exact_misfit(m):
        e.set_model(*m, eta)
        e.forward(shots, want_sections=False)
        e.residual(obs)
        return float(e.vjp_exact(40, want_grad=False, moduli=True)[1][:len(shots)].sum())

    mis32 = np.array([gpu_misfit(mods)])
    g, mis64 = e.vjp_exact(40, moduli=True)
    assert abs(mis64[:len(shots)].sum() / mis32[0] - 1) < 1e-5, (mis64, mis32)
    assert np.isfinite(g).all() and all(np.abs(g[q]).max() > 0 for q in range(5))
    with pytest.raises(ifosb.IfosbError):
        e.vjp_exact(40)  # the (vp, vs, rho) form is elastic
    for d in _directions(rng, 4, 5):
        plus, minus, half = _pm(mods, d, 1e-5)
        fd = (exact_misfit(plus) - exact_misfit(minus)) / 2
        dot = sum(float((gq * hq).sum()) for gq, hq in zip(g, half))
        print(f"L=3 FP64 misfit: <g,d> {dot:.12e} FD {fd:.12e} rel {abs(dot - fd) / abs(fd):.2e}")
        assert abs(dot - fd) <= 1e-6 * abs(fd)
    for d in _directions(rng, 6, 5):
        plus, minus, half = _pm(mods, d, 1e-3)
        fd = (gpu_misfit(plus) - gpu_misfit(minus)) / 2
        dot = sum(float((gq * hq).sum()) for gq, hq in zip(g, half))
        print(f"L=3 FP32 misfit: <g,d> {dot:.6e} FD {fd:.6e} rel {abs(dot - fd) / abs(fd):.2e}")
        assert abs(dot - fd) <= 1e-3 * abs(fd)
    e.close()


def test_exact_vjp_preconditions():
    c = synth.small_case(nx=20, ny=18, nz=20, nt=30, fw=4, nmech=1, nshots=1, seed=3)
    from helpers import engine_for
    e, m, cp, shots = engine_for(c)
    syn = e.forward(shots)
    e.residual(syn * 0.5)
    with pytest.raises(ifosb.IfosbError):
        e.vjp_exact(5)  # viscoelastic: velocities need the reference frequency; the moduli form
    g, mis = e.vjp_exact(5, moduli=True)
    assert g.shape == (5, 18, 20, 20) and np.abs(g[3:]).max() > 0 and mis[0] > 0
    e.close()
    c = synth.small_case(nx=20, ny=18, nz=20, nt=30, fw=4, nmech=0, nshots=1, seed=3)
    e, m, cp, shots = engine_for(c)
    with pytest.raises(ifosb.IfosbError):
        e.vjp_exact(5)  # no forward yet
    syn = e.forward(shots)
    with pytest.raises(ifosb.IfosbError):
        e.vjp_exact(5)  # no residual yet
    e.residual(syn * 0.5)
    with pytest.raises(ifosb.IfosbError):
        e.vjp_exact(0)
    g, mis = e.vjp_exact(4)
    assert np.abs(g).max() > 0 and mis[0] > 0
    gm, mis2 = e.vjp_exact(4, moduli=True)  # the moduli form of the same gradient
    assert np.array_equal(mis, mis2) and not gm[3:].any()
    e.close()


def test_exact_vjp_on_the_adjoint_check_configuration():
    """The adjoint-gradient configuration at its own size: 192 x 192 x 160 cells,
    the Gaussian random-field model (+-3 %, correlation length 8 cells) for the
    observed data, its smooth depth-gradient background as the model, 4 shots, 64
    surface receivers, free surface and CPML; centred differences of the GPU's FP32
    misfit along 8 seeded directions (eps = 1e-3, vp, vs, rho mixed) against the
    exact VJP, within 1e-3 each."""
    c = synth.case("elastic192", nt=600)
    p = c["params"]
    m_true, cp, shots = synth.build_inputs(c, "true")
    e = ifosb.Engine(p, max_shots=len(shots), max_nf=0)
    e.set_cpml(cp)
    e.set_receivers(c["recpos"])
    e.set_frequencies(None, 1)
    shape = (p.ny, p.nx, p.nz)

    def mods_of(vp, vs, rho):
        m = ifosb.moduli(p, vp.ravel(), vs.ravel(), rho.ravel())
        return tuple(m[k].reshape(shape) for k in ("rho", "pi", "u"))

    e.set_model(*mods_of(*c["true"]), None, None, None)
    obs = e.forward(shots)
    start = c["start"]

    def gpu_misfit(model):
        e.set_model(*mods_of(*model), None, None, None)
        e.forward(shots, want_sections=False)
        return float(e.residual(obs).sum())

    j0 = gpu_misfit(start)
    g, mis = e.vjp_exact(40)
    assert abs(mis[:len(shots)].sum() / j0 - 1) < 1e-5
    rng = np.random.default_rng(5)
    worst = 0.0
    for _ in range(8):
        w = rng.uniform(-1, 1, 3)
        f = synth._gauss_field(shape, 8.0, rng).astype(np.float64)
        plus, minus, half = [], [], []
        for a, wi in zip(start, w):
            a64 = a.astype(np.float64)
            plus.append((a64 * (1 + 1e-3 * wi * f)).astype(np.float32))
            minus.append((a64 * (1 - 1e-3 * wi * f)).astype(np.float32))
            half.append((plus[-1].astype(np.float64) - minus[-1].astype(np.float64)) / 2)
        fd = (gpu_misfit(plus) - gpu_misfit(minus)) / 2
        dot = sum(float((gq * hq).sum()) for gq, hq in zip(g, half))
        rel = abs(dot - fd) / abs(fd)
        worst = max(worst, rel)
        print(f"192x192x160 grid: <g,d> {dot:.6e} FD {fd:.6e} rel {rel:.2e}")
        assert rel <= 1e-3
    print(f"192x192x160 grid: worst relative difference {worst:.2e}")
    e.close()
