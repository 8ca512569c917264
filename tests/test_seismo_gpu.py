"""SEISMO 2-4 (pressure, divergence, curl at the receivers, seismo_ssg.c) on
the GPU against the reference's own seismo() in its forward loop, bit for bit.
Both kernel families are covered, for elastic and L=1 models, with receivers
on the free surface, inside the CPML frame and in the interior."""
import numpy as np
import pytest

import ifosb
from helpers import engine_for, ifo_params
from ifosb import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seismo", [2, 3, 4])
@pytest.mark.parametrize("nmech,tma", [(0, "1"), (1, "1"), (0, "0")])
def test_seismo_components_match_reference(seismo, nmech, tma, ref_oracle, monkeypatch):
    monkeypatch.setenv("IFOSB_TMA", tma)
    c = synth.small_case(nt=60, nmech=nmech, seed=61 + seismo, finv=(), ntr=9)
    rec = np.asarray(c["recpos"], np.int32).copy()
    rec[0] = [7, 1, 9]    # on the free surface
    rec[1] = [12, 10, 11]  # interior
    c["recpos"] = rec
    e, m, cp, shots = engine_for(c)
    e.set_seismo(seismo)
    sec = e.forward(shots)
    comps = ifosb.Engine.SEISMO_COMPONENTS[seismo]
    assert sec.shape[1] == len(comps)
    p = ifo_params(c)
    for s, (sp, sig) in enumerate(shots):
        v, pdc = ref_oracle.forward_seismo(p, m, cp, sp, sig, rec, seismo)
        ref = {"vx": v[0], "vy": v[1], "vz": v[2], "p": pdc[0], "div": pdc[1], "curl": pdc[2]}
        for q, name in enumerate(comps):
            assert np.array_equal(sec[s, q].view(np.uint32), ref[name].view(np.uint32)), (name, s)
        assert np.abs(sec[s]).max() > 0
    e.close()


def test_seismo_argument_checks():
    c = synth.small_case(nt=20, seed=5, finv=())
    e, m, cp, shots = engine_for(c)
    with pytest.raises(ifosb.IfosbError):
        e.set_seismo(5)
    e.set_seismo(1)
    assert e.forward(shots).shape[1] == 3
    e.close()
