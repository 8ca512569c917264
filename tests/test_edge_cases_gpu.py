"""Edge cases of the reference's path on the GPU, each against the oracle bit
for bit:
- no receivers on the rank (ntr = 0);
- a batch smaller than the engine's shot capacity;
- DFT accumulation every ntast > 1 steps;
- decimated seismograms (NDT > 1, NDTSHIFT > 0), forward only: the adjoint
  indexes the residual by step and needs NDT = 1;
- the grid's smallest legal size for the CPML frame."""
import numpy as np
import pytest

import ifosb
from helpers import engine_for, ifo_params
from ifosb import synth

pytestmark = pytest.mark.gpu


def oracle_for(oracle, request, nmech=0):
    if nmech <= 1:
        try:
            return request.getfixturevalue("ref_oracle")
        except pytest.skip.Exception:
            return oracle
    return oracle


def forward_pair(c, O, engine_shots=None, max_shots=None):
    e, m, cp, shots = engine_for(c, max_shots=max_shots)
    use = shots if engine_shots is None else [shots[i] for i in engine_shots]
    sec = e.forward(use)
    p = ifo_params(c)
    nf = len(c["finv"])
    for q, (sp, sig) in enumerate(use):
        f = O.forward(p, m, cp, sp, sig, c["recpos"], c["finv"] if nf else None, c["ntast"], True, True)
        st = e.get_state(q)
        for fld in range(9):
            assert np.array_equal(st[fld], f["state"][fld]), f"state field {fld} shot {q}"
        if sec is not None:
            assert np.array_equal(sec[q], f["sections"]), f"sections shot {q}"
        if nf:
            assert np.array_equal(e.get_dft(q), f["dft"]), f"forward DFT shot {q}"
    return e, sec


def test_no_receivers(oracle, request):
    c = synth.small_case(nt=50, seed=41)
    c["recpos"] = np.zeros((0, 3), np.int32)
    e, sec = forward_pair(c, oracle_for(oracle, request))
    assert sec is None or sec.size == 0
    e.close()


def test_partial_batch(oracle, request):
    """Two shots through an engine sized for four: the unused slots stay idle."""
    c = synth.small_case(nt=50, nshots=4, seed=43)
    e, _ = forward_pair(c, oracle_for(oracle, request), engine_shots=[2, 0], max_shots=4)
    e.close()


@pytest.mark.parametrize("ntast", [3, 7])
def test_dft_every_ntast_steps(ntast, oracle, request):
    c = synth.small_case(nt=60, seed=47)
    c["ntast"] = ntast
    e, _ = forward_pair(c, oracle_for(oracle, request))
    e.close()


def test_decimated_seismograms(oracle, request):
    c = synth.small_case(nt=61, seed=53, finv=())
    p = c["params"]
    c["params"] = ifosb.make_params(p.nx, p.ny, p.nz, dh=1.0, dt=1e-4, nt=p.nt, fdcoeff=p.fdcoeff,
                                    free_surf=p.free_surf, fw=p.fw, nmech=0, ndt=3, ndtshift=2)
    e, sec = forward_pair(c, oracle_for(oracle, request))
    assert sec.shape[-1] == ifosb.nsamples(c["params"]) < c["params"].nt
    e.close()


def test_smallest_grid(oracle, request):
    """Every tile touches the CPML frame and the grid is one partial tile wide."""
    c = synth.small_case(nx=13, ny=12, nz=14, nt=40, fw=4, seed=59, ntr=4)
    e, _ = forward_pair(c, oracle_for(oracle, request))
    e.close()
