"""Approximate Hessian (HESS) on the GPU against the reference itself (oracle/_ref).

Reference side, for each shot in order:
- the forward DFT fields;
- one Hessian wavefield per receiver (ifos3d.c:887-938): adjoint-mode
  propagation of a y-force at that receiver with the backward DFT, run by the
  reference harness's adjoint with that single receiver;
- hess_F over the receivers and frequencies.
Engine side:
- ifosb_hessian_green once, for all receivers, in batches of max_shots;
- one forward batch;
- ifosb_hessian.
The Hessians must be EQUAL. hess_apply is checked against the reference's
hess_apply the same way."""
import numpy as np
import pytest

import ifosb
from helpers import engine_for, ifo_params
from ifosb import synth

pytestmark = pytest.mark.gpu


def step_signal(nt, shift):
    """wavelet.c type 5 (a step at tshift), the reference's Hessian source."""
    s = np.zeros(nt, np.float32)
    s[shift:] = 1.0
    return s


@pytest.mark.parametrize("free_surf", [0, 1])
def test_hessian_matches_reference(ref_oracle, free_surf):
    c = synth.small_case(nx=26, ny=22, nz=24, nt=60, fw=5, nmech=0, nshots=2, seed=31, free_surf=free_surf)
    e, m, cp, shots = engine_for(c, max_shots=2)
    p = ifo_params(c)
    nt = c["params"].nt
    rec = np.asarray(c["recpos"], np.int32)
    ids = [0, 1, 2]
    sigs = np.stack([step_signal(nt, 5 + 4 * q) for q in range(len(ids))])  # one step per receiver
    e.hessian_green(ids, sigs)
    e.zero_hessian()
    e.forward(shots, want_sections=False)
    e.hessian()
    h_eng = e.get_hessian()
    # the reference: Green's functions of the same receivers, then hess_F shot by shot
    ns = ref_oracle.nsamples(p)
    assert ns == nt
    greens = []
    for q, r in enumerate(ids):
        diff = np.zeros((3, 1, ns), np.float32)
        diff[1, 0] = sigs[q]
        greens.append(ref_oracle.adjoint(p, m, cp, rec[r:r + 1], diff, c["finv"], c["ntast"])["dft"])
    greens = np.stack(greens)
    h_ref = np.zeros_like(h_eng)
    for sp, s in shots:
        f = ref_oracle.forward(p, m, cp, sp, s, c["recpos"], c["finv"], c["ntast"], True)
        h_ref = ref_oracle.hessian(p, m, c["finv"], f["dft"], greens, h_ref)
    assert np.isfinite(h_ref).all() and np.abs(h_ref).max() > 0
    assert np.array_equal(h_eng.view(np.uint32), h_ref.view(np.uint32))
    # a second batch accumulates; a forward is needed before each contribution
    with pytest.raises(ifosb.IfosbError):
        e.hessian()
    e.close()


def test_hessian_state_errors():
    c = synth.small_case(nx=20, ny=18, nz=20, nt=30, fw=4, nmech=0, nshots=1, seed=3)
    e, m, cp, shots = engine_for(c)
    with pytest.raises(ifosb.IfosbError):
        e.hessian()  # no Green's functions yet
    with pytest.raises(ifosb.IfosbError):
        e.hessian_green([99], step_signal(c["params"].nt, 2))  # no such receiver
    e.hessian_green([0], step_signal(c["params"].nt, 2))
    e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
    e.forward(shots, want_sections=False)
    with pytest.raises(ifosb.IfosbError):
        e.hessian()  # a new model drops the Green's functions
    e.close()
    cv = synth.small_case(nx=20, ny=18, nz=20, nt=30, fw=4, nmech=1, nshots=1, seed=3)
    ev, _, _, _ = engine_for(cv)
    with pytest.raises(ifosb.IfosbError):
        ev.hessian_green([0], step_signal(cv["params"].nt, 2))  # elastic only
    ev.close()


@pytest.mark.parametrize("lbfgs", [False, True])
def test_hess_apply_matches_reference(ref_oracle, lbfgs):
    import ctypes as C
    from pyoracle import REF_LIB
    lib = C.CDLL(REF_LIB)
    ny, nx, nz = 9, 7, 8
    rng = np.random.default_rng(4)
    g = (rng.standard_normal((3, ny, nx, nz)) * 1e-6).astype(np.float32)
    h = (rng.uniform(0.0, 2.0, (3, ny, nx, nz)) * 1e-9).astype(np.float32)
    h[0, 0, 0, :3] = 0.0
    water = np.array([1e-10, 2e-11, 5e-12], np.float32)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    a = g.copy()
    assert lib.ifo_ref_hess_apply(nx, ny, nz, P(a), P(h), P(water), int(lbfgs), C.c_float(3000.0), C.c_float(1732.0),
                                  C.c_float(2000.0)) == 0
    o = ifosb.Optimizer(nx, ny, nz)
    b = g.copy()
    o.hess_apply(b, h, water, lbfgs=lbfgs, vp0=3000.0, vs0=1732.0, rho0=2000.0)
    o.close()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
