"""The bounded mbarrier waits of the TMA time-step kernels, made to run out
without a GPU fault.

The reference stops on any failure with err() (src/util.c:30-40, e.g. the NaN
probe of src/ifos3d.c:761). The engine's counterpart for a TMA stage that never
lands is a wait limit: each mbarrier wait gives up after the limit, sets an
error flag, and the call returns IFOSB_ECUDA with the engine still usable.

ifosb_set_wait_test lowers the limit to 1 ms and makes one kernel's producer
warp stop issuing loads part-way through each y chunk (after the boxes it did
issue have landed), so the consumers wait on planes that never arrive: a flag
that nothing sets. The test checks the status, and that the next forward on the
same engine gives the same bits as before."""
import numpy as np
import pytest

import ifosb
from helpers import engine_for
from ifosb import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nmech", [0, 3])
@pytest.mark.parametrize("mode", [0, 1])  # graph replay, plain launches
def test_expired_wait_returns_ecuda_and_engine_recovers(nmech, mode):
    c = synth.small_case(nx=40, ny=34, nz=36, nt=30, nmech=nmech, seed=3, nshots=2)
    e, m, cp, shots = engine_for(c)
    e.set_launch_mode(mode)
    # chunks of 8 planes: a producer that stops at iteration 1 leaves planes unissued
    e.set_launch_shape(len(shots), [8, 1, 8, 1])
    ref = e.forward(shots)
    ref_state = e.get_state(1)
    for kernel in (1, 2):
        e.set_wait_test(wait_ns=1_000_000, kernel=kernel, stop_plane=1)
        with pytest.raises(ifosb.IfosbError) as ei:
            e.forward(shots)
        assert ei.value.code == ifosb.ECUDA
        assert "timed out" in str(ei.value)
        e.set_wait_test()  # back to the 1 s limit and full issue
        again = e.forward(shots)
        assert np.array_equal(again, ref), f"kernel {kernel}: traces differ after the timeout"
        assert np.array_equal(e.get_state(1), ref_state), f"kernel {kernel}: state differs after the timeout"
    e.close()


def test_wait_test_arguments(ifosb_mod):
    c = synth.small_case(nt=10)
    p = c["params"]
    try:
        e = ifosb.Engine(p)
    except ifosb.IfosbError as err:  # no GPU here: the argument checks need an engine
        pytest.skip(str(err))
    for bad in ((10, 1, 1), (2_000_000_000, 1, 1), (1_000_000, 3, 1), (1_000_000, 1, -2)):
        with pytest.raises(ifosb.IfosbError):
            e.set_wait_test(*bad)
    e.set_wait_test()
    e.close()
