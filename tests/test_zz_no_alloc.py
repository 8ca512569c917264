"""ifosb_residual_noalloc — the residual and FP64 misfit on caller-owned device
buffers with a fixed device scratch array — against the engine's ifosb_residual
(same kernels, so the same bits) and against the oracle's residual().

The file is named to be collected last, so that in a full run the entry point is
also exercised after every other test has used the library in this process."""
import numpy as np
import pytest

import ifosb
from helpers import engine_for, ifo_params
from ifosb import synth

FAKE = 4096  # a non-null address; these calls must return before touching it


def test_argument_and_size_checks_launch_nothing(ifosb_mod):
    n_over = ifosb.NOALLOC_MAX_TRACES // 3 + 1
    assert ifosb.residual_noalloc(1, n_over, 8, 1e-4, FAKE, FAKE, FAKE, FAKE) == ifosb.ETOOBIG
    assert ifosb.residual_noalloc(2, ifosb.NOALLOC_MAX_TRACES // 6 + 1, 8, 1e-4, FAKE, FAKE, FAKE, FAKE) == ifosb.ETOOBIG
    assert ifosb.residual_noalloc(0, 4, 8, 1e-4, FAKE, FAKE, FAKE, FAKE) == ifosb.EARG
    assert ifosb.residual_noalloc(1, 4, 0, 1e-4, FAKE, FAKE, FAKE, FAKE) == ifosb.EARG
    assert ifosb.residual_noalloc(1, 4, 8, 1e-4, FAKE, 0, FAKE, FAKE) == ifosb.EARG
    # the residual may not overlap the traces it is formed from (written reversed while they are read)
    n = 3 * 4 * 8 * 4  # bytes of one shot's traces
    assert ifosb.residual_noalloc(1, 4, 8, 1e-4, FAKE, FAKE + 2 * n, FAKE, FAKE) == ifosb.EARG
    assert ifosb.residual_noalloc(1, 4, 8, 1e-4, FAKE, FAKE + 2 * n, FAKE + 2 * n + n - 4, FAKE) == ifosb.EARG


def _np_residual(syn, obs, dt):
    """residual.c:35-60 in numpy: float32 running sum, float32 scaling, reversed."""
    v = np.add.accumulate((syn - obs).astype(np.float32), axis=-1, dtype=np.float32)
    d = (np.float32(dt) * v).astype(np.float32)[..., ::-1]
    mis = (d.astype(np.float64) ** 2).reshape(d.shape[0], -1).sum(axis=1)
    return np.ascontiguousarray(d), mis


@pytest.mark.gpu
def test_two_calls_in_a_row_match_ifosb_residual(oracle):
    import torch

    c = synth.small_case(nshots=2, ntr=9, nt=120, seed=11)
    e, m, cp, shots = engine_for(c, nf=0)
    p = c["params"]
    sec = e.forward(shots)
    rng = np.random.default_rng(5)
    obs1 = (sec * np.float32(0.9) + np.float32(1e-9) * rng.standard_normal(sec.shape)).astype(np.float32)
    obs2 = (sec * np.float32(1.1)).astype(np.float32)
    mis_ref1 = e.residual(obs1)
    mis_ref2 = e.residual(obs2)

    nsh, _, ntr, ns = sec.shape
    dev = torch.device("cuda", 0)
    syn_d = torch.from_numpy(sec).to(dev)
    obs_d = [torch.from_numpy(o).to(dev) for o in (obs1, obs2)]
    diff_d = [torch.full_like(syn_d, float("nan")) for _ in range(2)]
    mis_d = [torch.full((nsh,), float("nan"), dtype=torch.float64, device=dev) for _ in range(2)]
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    for r in range(2):  # back to back on one stream, no wait in between
        rc = ifosb.residual_noalloc(nsh, ntr, ns, p.dt, syn_d.data_ptr(), obs_d[r].data_ptr(), diff_d[r].data_ptr(),
                                    mis_d[r].data_ptr(), stream.cuda_stream)
        assert rc == ifosb.OK
    torch.cuda.synchronize(dev)

    for r, (obs, mis_ref) in enumerate(((obs1, mis_ref1), (obs2, mis_ref2))):
        mis = mis_d[r].cpu().numpy()
        assert np.array_equal(mis, mis_ref), (r, mis, mis_ref)
        diff = diff_d[r].cpu().numpy()
        P = ifo_params(c)
        for s in range(nsh):
            d_or, _ = oracle.residual(P, obs[s], sec[s])
            assert np.array_equal(diff[s], d_or)

    # a smaller call after the larger ones: only shot 1, nothing left over from before
    one_d = torch.full_like(syn_d[:1], float("nan"))
    mis1 = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    rc = ifosb.residual_noalloc(1, ntr, ns, p.dt, syn_d[1:].data_ptr(), obs_d[0][1:].data_ptr(), one_d.data_ptr(),
                                mis1.data_ptr(), stream.cuda_stream)
    assert rc == ifosb.OK
    torch.cuda.synchronize(dev)
    assert mis1.cpu().numpy()[0] == mis_ref1[1]
    assert np.array_equal(one_d.cpu().numpy()[0], diff_d[0].cpu().numpy()[1])


@pytest.mark.gpu
def test_largest_accepted_size_and_rejection_leave_outputs_right(ifosb_mod):
    import torch

    nsh, ntr, ns, dt = 2, ifosb.NOALLOC_MAX_TRACES // 6, 16, 1e-4
    assert nsh * 3 * ntr <= ifosb.NOALLOC_MAX_TRACES
    rng = np.random.default_rng(9)
    syn = rng.standard_normal((nsh, 3, ntr, ns)).astype(np.float32)
    obs = rng.standard_normal((nsh, 3, ntr, ns)).astype(np.float32)
    dev = torch.device("cuda", 0)
    syn_d, obs_d = torch.from_numpy(syn).to(dev), torch.from_numpy(obs).to(dev)
    diff_d = torch.full_like(syn_d, float("nan"))
    mis_d = torch.full((nsh,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    rc = ifosb.residual_noalloc(nsh, ntr, ns, dt, syn_d.data_ptr(), obs_d.data_ptr(), diff_d.data_ptr(),
                                mis_d.data_ptr(), 0)
    assert rc == ifosb.OK
    torch.cuda.synchronize(dev)
    d_np, mis_np = _np_residual(syn, obs, dt)
    assert np.array_equal(diff_d.cpu().numpy(), d_np)
    np.testing.assert_allclose(mis_d.cpu().numpy(), mis_np, rtol=1e-12)

    # one trace more than the scratch holds: rejected, outputs untouched
    before = diff_d.clone()
    rc = ifosb.residual_noalloc(nsh, ntr + 1, ns, dt, syn_d.data_ptr(), obs_d.data_ptr(), diff_d.data_ptr(),
                                mis_d.data_ptr(), 0)
    assert rc == ifosb.ETOOBIG
    torch.cuda.synchronize(dev)
    assert torch.equal(diff_d, before)
