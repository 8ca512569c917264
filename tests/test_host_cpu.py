"""CPU-side checks of the product library: it loads, exports every entry point
the C header declares, and its host utilities (CPML profiles, wavelets,
relaxed moduli) reproduce the reference's arithmetic bit for bit."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from helpers import ifo_params
from ifosb import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            txt = open(os.path.join(inc, fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(ifosb_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol(ifosb_mod):
    lib = ctypes.CDLL(ifosb_mod.LIB_PATH)
    decl = declared_symbols()
    assert len(decl) >= 20
    for name in sorted(decl):
        assert hasattr(lib, name), name
    assert decl == set(ifosb_mod.exported_symbols())
    out = subprocess.run(["nm", "-D", "--defined-only", ifosb_mod.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (ifosb_\w+)", out))
    assert decl <= exported


def test_library_is_built_for_sm100a(ifosb_mod):
    """The build uses -gencode arch=compute_100a,code=sm_100a only."""
    mk = open(os.path.join(ROOT, "ifos3d-dev_b200", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk and "--fmad=false" in mk


def test_no_gpu_means_enodev_not_fallback(ifosb_mod):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    p = ifosb_mod.make_params(24, 24, 24, fw=5, nt=10)
    with pytest.raises(ifosb_mod.IfosbError) as ei:
        ifosb_mod.Engine(p, 1, 0)
    assert ei.value.code == ifosb_mod.ENODEV


@pytest.mark.parametrize("dh", [(1.0, 1.0, 1.0), (0.8, 1.3, 2.0)])
def test_cpml_profiles_match_reference(dh, ifosb_mod, oracle, request):
    c = synth.small_case(nt=20)
    p = c["params"]
    p.dx, p.dy, p.dz = dh
    ip = ifo_params(c)
    ours = ifosb_mod.cpml_coeff(p, c["vppml"], c["fpml"])
    assert np.array_equal(ours, oracle.cpml_coeff(ip))
    try:
        ref = request.getfixturevalue("ref_oracle")
        assert np.array_equal(ours, ref.cpml_coeff(ip))
    except pytest.skip.Exception:
        pass


@pytest.mark.parametrize("shape", [1, 2, 4, 5])
def test_wavelets_match(shape, ifosb_mod, oracle):
    c = synth.small_case(nt=300)
    ip = ifo_params(c)
    ip.source_shape = shape
    src = np.array([[5, 5, 5, 0.001, 400.0, 2.0, 1], [6, 6, 6, 0.0, 900.0, 0.5, 1]], np.float32)
    assert np.array_equal(ifosb_mod.wavelet(c["params"], shape, src), oracle.wavelet(ip, src))


@pytest.mark.parametrize("nmech", [0, 1, 3])
def test_moduli_match_readmod(nmech, ifosb_mod, oracle):
    c = synth.small_case(nt=20, nmech=nmech)
    vp, vs, rho = c["start"]
    ours = ifosb_mod.moduli(c["params"], vp, vs, rho, tau=c["tau"], fl=c["fl"])
    ref = oracle.readmod(ifo_params(c), vp, vs, rho, tau=c["tau"], fl=c["fl"])
    for k in ("rho", "pi", "u"):
        assert np.array_equal(ours[k], ref[k]), k
    if nmech:
        assert np.array_equal(ours["eta"], ref["eta"])
        assert np.array_equal(ours["taus"], ref["taus"])


def test_ghost_wrap_is_one_rank_matcopy(ifosb_mod, oracle):
    """np.pad(wrap) reproduces matcopy on one rank: av_mat computed from the
    wrapped model equals the reference's (which ran matcopy itself)."""
    c = synth.small_case(nt=10)
    vp, vs, rho = c["start"]
    m = ifosb_mod.moduli(c["params"], vp, vs, rho)
    g = ifosb_mod.ghost_wrap(m["u"])
    assert g.shape == (c["params"].ny + 2, c["params"].nx + 2, c["params"].nz + 2)
    assert np.array_equal(g[0], g[-2]) and np.array_equal(g[:, -1], g[:, 1]) and np.array_equal(g[:, :, 0], g[:, :, -2])
    ip = ifo_params(c)
    avg = oracle.av_mat(ip, m)
    u = g.astype(np.float64)
    uipjp = (4.0 / (1.0 / u[1:-1, 1:-1, 1:-1] + 1.0 / u[1:-1, 2:, 1:-1] + 1.0 / u[2:, 2:, 1:-1] + 1.0 / u[2:, 1:-1, 1:-1])
             ).astype(np.float32)
    assert np.array_equal(uipjp, avg[0])


def test_q_fit_constant_q(ifosb_mod):
    """tau-method fit: the fitted Q stays within a few percent of the target over the band."""
    tau, fl = synth.q_tau_fit(50.0, 20.0, 200.0, 3)
    w = 2 * np.pi * np.exp(np.linspace(np.log(20.0), np.log(200.0), 50))
    tl = 1 / (2 * np.pi * fl)
    a = (w[:, None] * tl / (1 + (w[:, None] * tl) ** 2)).sum(1)
    b = ((w[:, None] * tl) ** 2 / (1 + (w[:, None] * tl) ** 2)).sum(1)
    q = (1 + tau * b) / (tau * a)
    assert np.all(np.abs(q / 50.0 - 1) < 0.25)


def test_q_gradient_chain_rule(ifosb_mod):
    """ifosb.q_gradient: with tau proportional to 1/Q (the tau method), the Q
    gradient is the taup / taus gradients through d tau / dQ = -tau / Q; checked
    by a centred difference of the linear functional <g, tau(Q)> per cell."""
    rng = np.random.default_rng(3)
    gq = rng.standard_normal((2, 4, 5, 6))
    q0 = rng.uniform(20.0, 80.0, (4, 5, 6))
    tau, _ = synth.q_tau_fit(50.0, 20.0, 200.0, 3)
    tp = lambda q: tau * 50.0 / q * 1.1  # noqa: E731  taup and taus with their own constants
    ts = lambda q: tau * 50.0 / q * 0.9  # noqa: E731
    got = ifosb_mod.q_gradient(gq, tp(q0), ts(q0), q0)
    h = 1e-4 * q0
    fd = (gq[0] * (tp(q0 + h) - tp(q0 - h)) + gq[1] * (ts(q0 + h) - ts(q0 - h))) / (2 * h)
    assert np.allclose(got, fd, rtol=1e-6, atol=0)


def test_q_moduli_per_cell_matches_readmod(ifosb_mod):
    """synth.q_moduli (readmod's arithmetic with a relaxation time per cell)
    equals ifosb_moduli (one tau for the model) bit for bit where tau is
    uniform; synth.tau_of_q scales tau as 1/Q."""
    p = ifosb_mod.make_params(10, 9, 8, dh=1.0, dt=1e-4, nt=10, fdcoeff=2, free_surf=0, fw=2, nmech=3)
    rng = np.random.default_rng(4)
    shape = (9, 10, 8)
    vp = rng.uniform(2500, 3500, shape).astype(np.float32)
    vs = (vp / np.float32(np.sqrt(3.0))).astype(np.float32)
    rho = rng.uniform(1800, 2400, shape).astype(np.float32)
    for q in (30.0, 50.0, 100.0):
        tau, fl = synth.q_tau_fit(q, 10.0, 100.0, 3)
        ref = ifosb_mod.moduli(p, vp.ravel(), vs.ravel(), rho.ravel(), tau=tau, fl=fl)
        got = synth.q_moduli(p, vp, vs, rho, np.full(shape, tau, np.float32), fl)
        for k in ("pi", "u", "taus", "taup"):
            assert np.array_equal(got[k].ravel(), ref[k]), (q, k)
        assert np.array_equal(got["eta"], ref["eta"])
    qf = rng.uniform(30, 100, shape).astype(np.float32)
    tq, fl = synth.tau_of_q(qf, 10.0, 100.0, 3)
    t50, _ = synth.q_tau_fit(50.0, 10.0, 100.0, 3)
    np.testing.assert_allclose(tq * qf, np.float32(t50 * 50.0), rtol=1e-6)
