"""Golden fixtures produced by the reference itself (tests/golden/make_golden.py).

CPU: the C restatement and the product's host utilities reproduce them bit for
bit. GPU: the CUDA engine reproduces them bit for bit through the C ABI."""
import glob
import os

import numpy as np
import pytest

import ifosb
from pyoracle import IfoParams

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "*.npz")))


def load(path):
    d = dict(np.load(path))
    return {k: (v.item() if v.ndim == 0 and k not in ("tau", "l2") else v) for k, v in d.items()}


def ifo(d):
    dt = np.float32(1e-4)
    return IfoParams(nx=d["nx"], ny=d["ny"], nz=d["nz"], dx=1.0, dy=1.0, dz=1.0, dt=dt, nt=d["nt"],
                     time=np.float32(np.float32(d["nt"] - 1) * dt), fdcoeff=d["fdcoeff"], free_surf=d["free_surf"],
                     fw=d["fw"], nmech=d["nmech"], ndt=1, ndtshift=0, vppml=3000.0, fpml=500.0,
                     alpha=d["alpha"], beta=d["beta"], source_shape=4)


def prm(d):
    return ifosb.make_params(d["nx"], d["ny"], d["nz"], dh=1.0, dt=1e-4, nt=d["nt"], fdcoeff=d["fdcoeff"],
                             free_surf=d["free_surf"], fw=d["fw"], nmech=d["nmech"], alpha=d["alpha"], beta=d["beta"])


def model(d):
    m = {k: d[k] for k in ("rho", "pi", "u")}
    for k in ("taus", "taup", "eta"):
        m[k] = d[k] if d["nmech"] else None
    return m


def ck(a):
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    return np.stack([a.sum(1), np.abs(a).sum(1), (a * a).sum(1)], 1)


def test_fixtures_present():
    assert len(GOLD) >= 3


@pytest.mark.parametrize("path", GOLD, ids=lambda p: os.path.basename(p)[:-4])
def test_restatement_reproduces_reference_fixture(path, oracle):
    d = load(path)
    p = ifo(d)
    m = oracle.readmod(p, d["vp"], d["vs"], d["rho_in"], tau=float(d["tau"]), fl=d["fl"] if d["nmech"] else None)
    for k in ("rho", "pi", "u"):
        assert np.array_equal(m[k], d[k]), k
    assert np.array_equal(oracle.cpml_coeff(p), d["cpml"])
    assert np.array_equal(oracle.wavelet(p, d["srcpos"]), d["signals"])
    f = oracle.forward(p, model(d), d["cpml"], d["srcpos"], d["signals"], d["recpos"], d["finv"], 1, True, True)
    assert np.array_equal(f["sections"], d["sections"])
    assert np.array_equal(ck(f["dft"].reshape(12, -1)), d["dft_ck"])
    assert np.array_equal(ck(f["state"]), d["state_ck"])
    diff, l2 = oracle.residual(p, d["obs"], f["sections"])
    assert np.array_equal(diff, d["diff"]) and np.float32(l2) == d["l2"]
    b = oracle.adjoint(p, model(d), d["cpml"], d["recpos"], diff, d["finv"], 1, True)
    assert np.array_equal(ck(b["dft"].reshape(12, -1)), d["bdft_ck"])
    assert np.array_equal(ck(b["state"]), d["bstate_ck"])
    assert np.array_equal(oracle.gradient(p, model(d), d["finv"], f["dft"], b["dft"]), d["grad"])


@pytest.mark.parametrize("path", GOLD, ids=lambda p: os.path.basename(p)[:-4])
def test_host_utilities_reproduce_reference_inputs(path, ifosb_mod):
    d = load(path)
    p = prm(d)
    assert np.array_equal(ifosb_mod.cpml_coeff(p, 3000.0, 500.0), d["cpml"])
    assert np.array_equal(ifosb_mod.wavelet(p, 4, d["srcpos"]), d["signals"])
    m = ifosb_mod.moduli(p, d["vp"], d["vs"], d["rho_in"], tau=float(d["tau"]), fl=d["fl"] if d["nmech"] else None)
    for k in ("pi", "u"):
        assert np.array_equal(m[k], d[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLD, ids=lambda p: os.path.basename(p)[:-4])
def test_engine_reproduces_reference_fixture(path):
    d = load(path)
    p = prm(d)
    e = ifosb.Engine(p, max_shots=1, max_nf=len(d["finv"]))
    e.set_cpml(d["cpml"])
    m = model(d)
    e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
    e.set_receivers(d["recpos"])
    e.set_frequencies(d["finv"], 1)
    sec = e.forward([(d["srcpos"], d["signals"])])
    assert np.array_equal(sec[0], d["sections"])
    assert np.array_equal(ck(e.get_dft(0).reshape(12, -1)), d["dft_ck"])
    assert np.array_equal(ck(e.get_state(0)), d["state_ck"])
    mis, l2 = e.residual(d["obs"][None], want_l2_ref=True)
    assert l2[0] == d["l2"]
    e.adjoint()
    assert np.array_equal(ck(e.get_dft(0, back=True).reshape(12, -1)), d["bdft_ck"])
    e.gradient()
    assert np.array_equal(e.get_gradient(), d["grad"])
    e.close()
