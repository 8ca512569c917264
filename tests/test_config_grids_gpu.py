"""Parity on the benchmark configurations' own grids, against the CPU oracle.

- The adjoint-gradient configuration: 192 x 192 x 160 cells, the Gaussian
  random-field model (+-3 %, correlation length 8 cells) on the 2000-3500 m/s
  depth gradient, 4 shots, 5 frequencies (20-100 Hz). The observed traces come
  from the random-field model, the gradient is taken in the smooth background
  (as the reference's inversion does: forward, residual, adjoint, gradient_F,
  src/ifos3d.c:712-975). Traces, both DFT fields of every shot and the 4-shot
  gradient are compared with the reference build itself (oracle/_ref, every shot
  in its own process), bit for bit, over 50 time steps.
- The batched viscoelastic gradient configuration: 384 x 384 horizontal x 256
  deep cells (NX x NZ x NY), L=3, 4 frequencies, 1024 receivers, two of its
  32 shots in one batch, 12 steps: traces, DFT fields and gradient against the
  C restatement (the reference has no L=3), bit for bit. The wave does not reach
  the receivers in 12 steps, so a seeded residual drives the adjoint.
- The viscoelastic forward-modelling configuration (256^3, L=3, 8 layers, 400
  receivers) for 120 steps: traces and every wavefield against the restatement.

Each grid is the configuration's full size; the full time loops run on the
small grids of the other parity tests, and every step runs the same code."""
import os

import numpy as np
import pytest

from helpers import engine_for, ifo_params, rel_l2
from ifosb import synth
from oracle_pool import load, run_shots
from pyoracle import Oracle, have_ref

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
SEIS_TOL = 1e-5


def _procs():
    return max(1, min(4, os.cpu_count() or 1))


def test_elastic192_full_grid_four_shots_against_the_reference(tmp_path):
    c = synth.case("elastic192", nt=50)
    kind = "ref" if have_ref() else "oracle"
    e, m, cp, shots = engine_for(c)
    mt, _, _ = synth.build_inputs(c, "true")
    e.set_model(mt["rho"], mt["pi"], mt["u"], None, None, None)
    obs = e.forward(shots)  # observed data: the random-field model (bit-identical to the oracle's forward)
    e.set_model(m["rho"], m["pi"], m["u"], None, None, None)
    ip = ifo_params(c)
    out = str(tmp_path)
    run_shots(kind, ip, m, cp, shots, c["recpos"], c["finv"], c["ntast"], obs, out, procs=_procs())

    sec = e.forward(shots)
    for s in range(len(shots)):
        ref = load(out, "sec", s)
        assert np.array_equal(sec[s], ref), f"traces shot {s}"
        assert rel_l2(sec[s], ref) <= SEIS_TOL
        assert np.array_equal(e.get_dft(s), load(out, "fdft", s)), f"forward DFT shot {s}"
    mis = e.residual(obs)
    assert np.all(mis > 0)
    e.adjoint()
    for s in range(len(shots)):
        assert np.array_equal(e.get_dft(s, back=True), load(out, "bdft", s)), f"backward DFT shot {s}"
    e.gradient()
    g = e.get_gradient()
    O = Oracle(kind, threads=0)
    grad = np.zeros((3, ip.ny, ip.nx, ip.nz), np.float32)
    for s in range(len(shots)):  # gradient_F accumulates shot after shot
        grad = O.gradient(ip, m, c["finv"], load(out, "fdft", s), load(out, "bdft", s), grad)
    assert np.abs(grad).max() > 0
    assert np.array_equal(g, grad), "4-shot gradient"
    assert rel_l2(g, grad) <= GRAD_TOL
    e.close()


def test_visco384_full_grid_two_shot_batch_against_the_restatement():
    c = synth.case("visco384", nt=12, nshots=2)
    p = c["params"]
    assert (p.nx, p.ny, p.nz) == (384, 256, 384)
    e, m, cp, shots = engine_for(c)
    sec = e.forward(shots)
    # 12 steps do not carry the wave to the receivers, so the residual of observed
    # traces would be zero: inject a seeded residual instead (the adjoint's input
    # either way), which the near-source forward field then correlates with
    rng = np.random.default_rng(12)
    diff = (1e-9 * rng.standard_normal(sec.shape)).astype(np.float32)
    e.adjoint(diff)
    e.gradient()
    g = e.get_gradient()
    ip = ifo_params(c)
    O = Oracle("oracle", threads=0)
    grad = np.zeros((3, ip.ny, ip.nx, ip.nz), np.float32)
    for s, (sp, sig) in enumerate(shots):
        f = O.forward(ip, m, cp, sp, sig, c["recpos"], c["finv"], c["ntast"], True)
        assert np.array_equal(sec[s], f["sections"]), f"traces shot {s}"
        b = O.adjoint(ip, m, cp, c["recpos"], diff[s], c["finv"], c["ntast"])
        # the engine's DFT fields are those of the last batch: compare before moving on
        assert np.array_equal(e.get_dft(s), f["dft"]), f"forward DFT shot {s}"
        assert np.array_equal(e.get_dft(s, back=True), b["dft"]), f"backward DFT shot {s}"
        grad = O.gradient(ip, m, c["finv"], f["dft"], b["dft"], grad)
        del f, b
    assert np.abs(grad).max() > 0
    assert np.array_equal(g, grad), "2-shot gradient"
    e.close()


def test_visco256_full_grid_120_steps_against_the_restatement():
    c = synth.case("visco256", nt=120)
    e, m, cp, shots = engine_for(c)
    sec = e.forward(shots)
    ip = ifo_params(c)
    O = Oracle("oracle", threads=0)
    sp, sig = shots[0]
    f = O.forward(ip, m, cp, sp, sig, c["recpos"], None, 1, False, True)
    assert np.array_equal(sec[0], f["sections"])
    st = e.get_state(0)
    for q in range(9):
        assert np.array_equal(st[q], f["state"][q]), f"field {q}"
    assert np.abs(st[1][3]).max() > 0  # the wave reached the free surface (j = 1)
    e.close()
