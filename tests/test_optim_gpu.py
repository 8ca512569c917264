"""FP64 optimiser kernels (ifosb_conjugate, ifosb_lbfgs_savegrad, ifosb_lbfgs,
ifosb_modelupdate) against the FP64 CPU oracle and the reference.

Stated errors, asserted below:
  * against the FP64 oracle (oracle/optim_oracle.py, prec="fp64", exactly
    rounded sums): CG betas and the L-BFGS scalars within 1e-12 relative (the
    only difference is the order of the FP64 sums); float32 directions within
    1 ulp; the model update bit-identical (the same float/double expressions);
    the recorded L-BFGS model differences bit-identical (FP64, same expression).
  * against the reference's float arithmetic (prec="ref", pinned to the
    reference build): betas within 1e-4 relative and directions within 1e-4
    relative L2 at these sizes (the reference sums 10^5 float terms in order)."""
import numpy as np
import pytest

import ifosb
import optim_oracle as oo
from helpers import rel_l2

pytestmark = pytest.mark.gpu

SHAPE = (48, 64, 40)  # ny, nx, nz: 122,880 cells, several grid-stride passes


def _grads(rng, scale=1.0):
    return (scale * rng.standard_normal((3,) + SHAPE)).astype(np.float32)


def test_conjugate_sequence_fp64():
    rng = np.random.default_rng(11)
    opt = ifosb.Optimizer(SHAPE[1], SHAPE[0], SHAPE[2])
    pr64 = np.zeros((6,) + SHAPE, np.float32)
    pr32 = pr64.copy()
    g0 = _grads(rng)
    seq = [(g0, 1), (_grads(rng), 0), ((0.5 * g0).astype(np.float32), 0), (_grads(rng, 3.0), 0)]
    for g, cdf in seq:
        gg, go, gr = g.copy(), g.copy(), g.copy()
        beta = opt.conjugate(gg, cdf)
        beta_o = oo.conjugate(go, pr64, cdf, "fp64")
        beta_r = oo.conjugate(gr, pr32, cdf, "ref")
        np.testing.assert_allclose(beta, beta_o, rtol=1e-12, atol=0)
        np.testing.assert_array_max_ulp(gg, go, maxulp=1)
        np.testing.assert_allclose(beta, beta_r, rtol=1e-4, atol=1e-12)
        assert rel_l2(gg, gr) < 1e-4
        pr64[3:6] = gg  # the device keeps its own direction as prior4..6: start the next step alike


@pytest.mark.parametrize("numpar,bfgsnum", [(1, 3), (2, 4)])
def test_lbfgs_iterations_fp64(numpar, bfgsnum):
    """Each call is checked from identical inputs: the oracle's history is set
    to the device's before every step, so 1-ulp differences cannot build up."""
    rng = np.random.default_rng(20 + numpar)
    n = int(np.prod(SHAPE))
    opt = ifosb.Optimizer(SHAPE[1], SHAPE[0], SHAPE[2], numpar=numpar, bfgsnum=bfgsnum)
    st = oo.LBFGSState(n, numpar, bfgsnum, "fp64")
    mshape = tuple(s + 2 for s in SHAPE)
    vp = (3000 + 50 * rng.standard_normal(mshape)).astype(np.float32)
    rho = (2000 + 20 * rng.standard_normal(mshape)).astype(np.float32)
    m_gpu = [rho.copy(), (vp * vp * rho).astype(np.float32), (vp * vp * rho / 3).astype(np.float32)]
    base = _grads(rng, 1e-3)
    for it in range(1, 8):  # wraps the history ring (bfgsnum < 7)
        g = (base + _grads(rng, 2e-4)).astype(np.float32)
        st.s[...], st.y[...], st.scale[...] = opt.history()
        gg, go = g.copy(), g.copy()
        if it == 1:
            opt.lbfgs_savegrad(gg)
            oo.lbfgs_savegrad(st, go)
        else:
            opt.lbfgs(gg, it)
            oo.lbfgs(st, go, it)
            np.testing.assert_array_max_ulp(gg, go, maxulp=1)
            assert not np.array_equal(gg, g)
        s, y, sc = opt.history()
        np.testing.assert_array_equal(y, st.y)
        np.testing.assert_allclose(sc, st.scale, rtol=1e-12, atol=0)
        # model update from the device's direction on both sides: bit-identical
        m_orc = [m.copy() for m in m_gpu]
        go = gg.copy()
        step = 1.0 if it > 1 else 0.05
        opt.modelupdate(gg, *m_gpu, step, (1.0, 1.0, 0.0), 3000.0, 1732.0, 2000.0, lbfgs=True, it_group=it)
        oo.modelupdate(go, *m_orc, step, (1.0, 1.0, 0.0), 3000.0, 1732.0, 2000.0, True, st, it)
        for a, b in zip(m_gpu, m_orc):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(opt.history()[0], st.s)


def test_modelupdate_cg_bit_identical_to_reference_arithmetic():
    rng = np.random.default_rng(31)
    opt = ifosb.Optimizer(SHAPE[1], SHAPE[0], SHAPE[2])
    mshape = tuple(s + 2 for s in SHAPE)
    vp = (2500 + 1000 * rng.random(mshape)).astype(np.float32)
    rho = (1800 + 800 * rng.random(mshape)).astype(np.float32)
    for zero_rho in (False, True):
        m_gpu = [rho.copy(), (vp * vp * rho).astype(np.float32), (vp * vp * rho / 3).astype(np.float32)]
        m_orc = [m.copy() for m in m_gpu]
        g = _grads(rng, 1e-2)
        if zero_rho:
            g[2] = 0.0
        gg, go = g.copy(), g.copy()
        opt.modelupdate(gg, *m_gpu, 0.02, (1.0, 0.8, 0.5), 3000.0, 1700.0, 2000.0)
        oo.modelupdate(go, *m_orc, 0.02, (1.0, 0.8, 0.5), 3000.0, 1700.0, 2000.0)
        np.testing.assert_array_equal(gg, go)
        for a, b in zip(m_gpu, m_orc):
            np.testing.assert_array_equal(a, b)


def test_optimizer_state_errors():
    opt = ifosb.Optimizer(4, 5, 6)
    g = np.zeros((3, 5, 4, 6), np.float32)
    with pytest.raises(ifosb.IfosbError) as ei:
        opt.lbfgs(g, 2)
    assert ei.value.code == ifosb.ESTATE
    with pytest.raises(ValueError):
        opt.conjugate(np.zeros((3, 4, 4, 4), np.float32), 0)
