"""Parity at the benchmark configurations' full grid sizes.

The CPU oracle cannot run the full time loops of these workloads in a test, but
it can run their full grids for a few dozen steps. Every time step runs the same
code, so a short run on the full grid together with the long runs on small
grids (test_gpu_parity.py, test_random_cases_gpu.py) covers both the size and
the length. The full-length runs are checked through properties that do not
depend on an oracle:
- elastic128 (128^3, FW=10 CPML, free surface, the sphere-anomaly model, 25
  receivers, 2 frequencies): forward, residual, adjoint and gradient for 40
  steps, bit-identical to the reference (oracle/_ref) or its restatement. The
  wave reaches the free surface and the x/z CPML faces within those steps.
- visco256 (256^3, L=3, 8 layers, 400 receivers): 12 forward steps, every
  wavefield and memory-variable-driven stress bit-identical to the restatement.
- elastic128 at its full NT=2000: a shot gives the same bits alone and in a
  batch of two, and doubling the source doubles the traces to within the
  rounding of the subnormal wavefront (relative L2 < 1e-6).
"""
import numpy as np
import pytest

import ifosb
from helpers import engine_for, rel_l2
from ifosb import synth
from test_gpu_parity import check_case, pick_oracle

pytestmark = pytest.mark.gpu


def test_elastic128_full_grid_gradient_bit_exact(oracle, request):
    c = synth.case("elastic128", nt=40)
    e, ref = check_case(c, pick_oracle(0, oracle, request))
    assert np.abs(ref["grad"]).max() > 0
    # the wavefield reached the free surface and the CPML frame
    st = e.get_state(0)
    fw = c["params"].fw
    assert np.abs(st[1][3]).max() > 0  # plane j = 1 (free surface)
    assert np.abs(st[1][:, 2:fw + 2, :]).max() > 0  # x CPML slab
    e.close()


def test_visco256_full_grid_forward_bit_exact(oracle):
    c = synth.case("visco256", nt=12)
    e, ref = check_case(c, oracle)
    assert np.abs(ref["state"][0][3]).max() > 0
    assert np.abs(e.get_state(0)[1][3]).max() > 0  # the wave reached the free surface (j = 1)
    e.close()


def test_elastic128_full_length_properties():
    c = synth.case("elastic128")
    p = c["params"]
    base = c["shots"][0]
    second = base.copy()
    second[0, 0] = 40
    c["shots"] = [base, second]
    m, cp, shots = synth.build_inputs(c)
    e2 = ifosb.Engine(p, max_shots=2, max_nf=2)
    e1 = ifosb.Engine(p, max_shots=1, max_nf=2)
    for e in (e1, e2):
        e.set_cpml(cp)
        e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
        e.set_receivers(c["recpos"])
        e.set_frequencies(c["finv"], 1)
    both = e2.forward(shots)
    one = e1.forward(shots[:1])
    assert np.array_equal(both[0], one[0])  # batch invariance at full size and length
    dft_one = e1.get_dft(0)
    e2.forward(shots)  # the DFT of shot 0 in the batch
    assert np.array_equal(e2.get_dft(0), dft_one)
    sp, sig = shots[0]
    twice = e1.forward([(sp, (sig * np.float32(2.0)).astype(np.float32))])
    assert np.abs(one[0]).max() > 0
    assert rel_l2(twice[0], 2.0 * one[0].astype(np.float64)) < 1e-6
    e1.close()
    e2.close()
