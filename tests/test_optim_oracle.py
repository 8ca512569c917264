"""The optimiser oracle (oracle/optim_oracle.py) pinned to the reference.

In its "ref" precision the numpy restatement of conjugate, lbfgs_savegrad,
lbfgs, modelupdate and steplength must equal the reference's own functions
(built from the reference sources into oracle/_ref) bit for bit, over whole
iteration sequences that reach the clamps and branches. The library's FP64
steplength (host code, no GPU) must equal the "fp64" restatement exactly."""
import numpy as np
import pytest

import ifosb
import optim_oracle as oo

SHAPE = (7, 6, 5)  # ny, nx, nz


@pytest.fixture(scope="module")
def ref(ref_oracle):
    return oo.RefOptim()


def _grads(rng, scale=1.0):
    return (scale * rng.standard_normal((3,) + SHAPE)).astype(np.float32)


def test_conjugate_sequence_matches_reference(ref):
    rng = np.random.default_rng(1)
    g0 = _grads(rng)
    grads = [g0, _grads(rng), (2.0 * g0).astype(np.float32), _grads(rng, 0.01)]
    cdfs = [1, 0, 0, 0]
    pr_ref = np.zeros((6,) + SHAPE, np.float32)
    pr_orc = pr_ref.copy()
    seen = set()
    for g, cdf in zip(grads, cdfs):
        a, b = g.copy(), g.copy()
        beta_ref = ref.conjugate(a, pr_ref, cdf)
        beta_orc = oo.conjugate(b, pr_orc, cdf, "ref")
        assert np.array_equal(a, b)
        assert np.array_equal(pr_ref, pr_orc)
        assert np.array_equal(beta_ref.astype(np.float64), beta_orc)
        seen.add((beta_orc[0] == 0.0, beta_orc[0] == 0.5))
    assert (False, True) in seen  # beta[0] clamped to 0.5


def test_conjugate_clamps_only_beta0(ref):
    rng = np.random.default_rng(2)
    g = _grads(rng)
    pr_ref = np.zeros((6,) + SHAPE, np.float32)
    pr_orc = pr_ref.copy()
    ref.conjugate(g.copy(), pr_ref, 1)
    oo.conjugate(g.copy(), pr_orc, 1, "ref")
    g2 = g.copy()
    g2[0] *= np.float32(0.5)   # g.(g - p) < 0 -> beta[0] < 0 -> clamped to 0
    g2[1] *= np.float32(0.25)  # beta[1] < 0 too, and stays negative
    g2[2] *= np.float32(3.0)   # beta[2] = 6 > 0.5, not clamped
    a, b = g2.copy(), g2.copy()
    beta_ref = ref.conjugate(a, pr_ref, 0)
    beta_orc = oo.conjugate(b, pr_orc, 0, "ref")
    assert np.array_equal(beta_ref.astype(np.float64), beta_orc)
    assert beta_orc[0] == 0.0 and beta_orc[1] < 0.0 and beta_orc[2] > 0.5
    assert np.array_equal(a, b)


@pytest.mark.parametrize("numpar,bfgsnum", [(1, 3), (2, 2)])
def test_lbfgs_iterations_match_reference(ref, numpar, bfgsnum):
    rng = np.random.default_rng(3 + numpar)
    n = int(np.prod(SHAPE))
    st_ref = oo.LBFGSState(n, numpar, bfgsnum, "ref")
    st_orc = oo.LBFGSState(n, numpar, bfgsnum, "ref")
    vp = (3000 + 100 * rng.standard_normal((SHAPE[0] + 2, SHAPE[1] + 2, SHAPE[2] + 2))).astype(np.float32)
    rho = np.full_like(vp, 2000.0)
    model_ref = [rho.copy(), (vp * vp * rho).astype(np.float32), (vp * vp * rho / 3).astype(np.float32)]
    model_orc = [m.copy() for m in model_ref]
    for it in range(1, 6):
        g = _grads(rng, 1e-3)
        a, b = g.copy(), g.copy()
        ref.lbfgs(a, st_ref, it)
        if it == 1:
            oo.lbfgs_savegrad(st_orc, b)
        else:
            oo.lbfgs(st_orc, b, it)
        assert np.array_equal(a, b), it
        assert np.array_equal(st_ref.y, st_orc.y) and np.array_equal(st_ref.scale, st_orc.scale), it
        step = 0.5 if it > 1 else 0.01
        ref.modelupdate(a, *model_ref, step, (1.0, 1.0, 0.0), 3000.0, 1732.0, 2000.0, True, st_ref, it)
        oo.modelupdate(b, *model_orc, step, (1.0, 1.0, 0.0), 3000.0, 1732.0, 2000.0, True, st_orc, it)
        for x, y in zip(model_ref, model_orc):
            assert np.array_equal(x, y), it
        assert np.array_equal(st_ref.s, st_orc.s), it


@pytest.mark.parametrize("zero_rho_grad", [False, True])
def test_modelupdate_cg_matches_reference(ref, zero_rho_grad):
    rng = np.random.default_rng(7)
    vp = (2500 + 500 * rng.random((SHAPE[0] + 2, SHAPE[1] + 2, SHAPE[2] + 2))).astype(np.float32)
    rho = (1800 + 400 * rng.random(vp.shape)).astype(np.float32)
    m_ref = [rho.copy(), (vp * vp * rho).astype(np.float32), (vp * vp * rho / 3).astype(np.float32)]
    m_orc = [m.copy() for m in m_ref]
    g = _grads(rng, 1e-2)
    if zero_rho_grad:
        g[2] = 0.0
    a, b = g.copy(), g.copy()
    ref.modelupdate(a, *m_ref, 0.03, (1.0, 0.7, 0.5), 3000.0, 1700.0, 2000.0)
    oo.modelupdate(b, *m_orc, 0.03, (1.0, 0.7, 0.5), 3000.0, 1700.0, 2000.0)
    assert np.array_equal(a, b)
    for x, y in zip(m_ref, m_orc):
        assert np.array_equal(x, y)


STEP_CASES = [
    # L2[0..2] at step 0, s, 2s; step[4]; lbfgs; it_group; teststep
    ((1.0, 0.8, 0.75), 0.01, False, 1, 0.01),    # a > 0, minimum inside
    ((1.0, 0.9, 0.8), 0.01, False, 2, 0.01),     # a = 0 or tiny: limits
    ((1.0, 0.99, 0.5), 0.02, False, 3, 0.02),    # a < 0, L2[2] smallest
    ((1.0, 0.7, 0.9), 0.02, False, 3, 0.05),     # a > 0 near step[1]
    ((0.5, 0.9, 1.3), 0.01, False, 1, 0.01),     # a < 0 or linear, L2[0] smallest
    ((1.0, 0.2, 0.1), 0.8, True, 3, 0.5),        # lbfgs cap at 1.0
    ((1.0, 0.5, 0.45), 0.3, True, 1, 0.5),       # lbfgs, first group iteration
    ((2.0, 1.99, 1.985), 1e-4, False, 4, 0.03),  # new test step floored at 0.2*teststep
]


@pytest.mark.parametrize("case", STEP_CASES)
def test_steplength_matches_reference_and_fp64_library(ref, case):
    L, s4, lb, itg, ts = case
    st = np.array([0.0, s4, 2 * s4, 0.0, s4], np.float32)
    L2 = np.array(list(L) + [0.0], np.float32)
    a_ref, b_ref = L2.copy(), st.copy()
    ref.steplength(a_ref, b_ref, lb, itg, ts)
    a_orc, b_orc = L2.copy(), st.copy()
    oo.steplength(a_orc, b_orc, lb, itg, ts, "ref")
    assert np.array_equal(a_ref, a_orc) and np.array_equal(b_ref, b_orc)
    # FP64: the library (host code) and the fp64 restatement do the same double ops
    L64, s64 = L2.astype(np.float64), st.astype(np.float64)
    abc = ifosb.steplength(L64, s64, lb, itg, ts)
    L64o, s64o = L2.astype(np.float64), st.astype(np.float64)
    abco = oo.steplength(L64o, s64o, lb, itg, ts, "fp64")
    assert np.array_equal(L64, L64o) and np.array_equal(s64, s64o)
    assert tuple(abc) == tuple(abco)
    # FP64 against the reference's float result: the same branch, within float rounding
    assert abs(s64[3] - b_ref[3]) <= 1e-5 * max(abs(float(b_ref[3])), 1e-30)
