"""The C restatement (oracle/ifos_oracle.c) against the reference's own functions
(oracle/_ref, compiled from the reference sources) — both on the CPU.

The reference ships no tests or golden vectors, so the restatement is pinned by
running the reference itself on the same seeded inputs: results must be
bit-identical (integer/float equality, not a tolerance)."""
import numpy as np
import pytest

from helpers import ifo_params
from ifosb import synth


CASES = [
    dict(nmech=0, free_surf=1),
    dict(nmech=0, free_surf=0),
    dict(nmech=1, free_surf=1),
    dict(nmech=1, free_surf=0, fdcoeff=1),
    dict(nmech=0, free_surf=1, nsrc=3, stype=2),
    dict(nmech=0, free_surf=1, nsrc=2, stype=5),
]


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "-".join(f"{a}{b}" for a, b in k.items()))
def test_restatement_matches_reference(kw, oracle, ref_oracle):
    c = synth.small_case(nt=60, **kw)
    p = ifo_params(c)
    if kw.get("stype") == 5:
        p.alpha, p.beta = 30.0, 60.0
    vp, vs, rho = c["start"]
    mr = ref_oracle.readmod(p, vp, vs, rho, tau=c["tau"], fl=c["fl"])
    mo = oracle.readmod(p, vp, vs, rho, tau=c["tau"], fl=c["fl"])
    for k in ("rho", "pi", "u"):
        assert np.array_equal(mr[k], mo[k]), k
    cr, co = ref_oracle.cpml_coeff(p), oracle.cpml_coeff(p)
    assert np.array_equal(cr, co)
    assert np.array_equal(ref_oracle.av_mat(p, mr), oracle.av_mat(p, mo))
    sp = c["shots"][0]
    sr, so = ref_oracle.wavelet(p, sp), oracle.wavelet(p, sp)
    assert np.array_equal(sr, so)
    fr = ref_oracle.forward(p, mr, cr, sp, sr, c["recpos"], c["finv"], 1, True, True)
    fo = oracle.forward(p, mo, co, sp, so, c["recpos"], c["finv"], 1, True, True)
    for k in ("sections", "dft", "state"):
        assert np.array_equal(fr[k], fo[k]), k
    assert np.abs(fr["sections"]).max() > 0
    obs = (fr["sections"] * np.float32(0.93)).astype(np.float32)
    dr, l2r = ref_oracle.residual(p, obs, fr["sections"])
    do, l2o = oracle.residual(p, obs, fo["sections"])
    assert np.array_equal(dr, do) and l2r == l2o
    br = ref_oracle.adjoint(p, mr, cr, c["recpos"], dr, c["finv"], 1, True)
    bo = oracle.adjoint(p, mo, co, c["recpos"], do, c["finv"], 1, True)
    for k in ("dft", "state"):
        assert np.array_equal(br[k], bo[k]), k
    gr = ref_oracle.gradient(p, mr, c["finv"], fr["dft"], br["dft"])
    go = oracle.gradient(p, mo, c["finv"], fo["dft"], bo["dft"])
    assert np.array_equal(gr, go)
    assert np.abs(gr).max() > 0


def test_reference_limits_mechanisms(ref_oracle):
    """The reference has one relaxation mechanism at most (src/update_s_ssg.c:75-76)."""
    c = synth.small_case(nt=10, nmech=3)
    p = ifo_params(c)
    m = {"rho": c["start"][2], "pi": c["start"][0], "u": c["start"][1], "taus": c["start"][1],
         "taup": c["start"][1], "eta": np.ones(3, np.float32)}
    with pytest.raises(RuntimeError):
        ref_oracle.forward(p, m, np.zeros((18, 2 * p.fw), np.float32), c["shots"][0],
                           np.zeros((1, p.nt), np.float32), c["recpos"])


def test_nsamples_rounding(oracle):
    """NT/ns rounding of src/ifos3d.c:176-179: TIME=0.19995, DT=1e-4 -> NT=2000."""
    import math
    dt = np.float32(1e-4)
    assert math.ceil(np.float32(0.19995) / dt) == 2000
    assert math.ceil(np.float32(0.2) / dt) == 2001
    c = synth.small_case(nt=2000)
    p = ifo_params(c)
    p.ndt, p.ndtshift = 3, 5
    assert oracle.nsamples(p) == math.ceil((2000 - 5) / 3)


@pytest.mark.parametrize("seed", range(6))
def test_restatement_matches_reference_random(seed, oracle, ref_oracle):
    """Seeded random cases: grid, CPML width, free surface, FD coefficients,
    mechanisms (the reference has L <= 1), sources and their kind, receivers,
    frequencies and DFT interval; forward, residual, adjoint and gradient must
    be bit-identical between the restatement and the reference."""
    rng = np.random.default_rng(100 + seed)
    fw = int(rng.integers(3, 7))
    n = [int(rng.integers(2 * fw + 6, 2 * fw + 16)) for _ in range(3)]
    nf = int(rng.integers(1, 4))
    c = synth.small_case(nx=n[0], ny=n[1], nz=n[2], nt=int(rng.integers(20, 50)), fw=fw,
                         free_surf=int(rng.integers(0, 2)), nmech=int(rng.integers(0, 2)),
                         fdcoeff=int(rng.integers(1, 3)), seed=seed, nsrc=int(rng.integers(1, 3)),
                         ntr=int(rng.integers(2, 10)), stype=int(rng.choice([1, 2, 3, 4])),
                         finv=tuple(float(f) for f in rng.uniform(100.0, 900.0, nf)))
    ntast = int(rng.integers(1, 4))
    p = ifo_params(c)
    vp, vs, rho = c["start"]
    mr = ref_oracle.readmod(p, vp, vs, rho, tau=c["tau"], fl=c["fl"])
    mo = oracle.readmod(p, vp, vs, rho, tau=c["tau"], fl=c["fl"])
    cr, co = ref_oracle.cpml_coeff(p), oracle.cpml_coeff(p)
    sp = c["shots"][0]
    sr, so = ref_oracle.wavelet(p, sp), oracle.wavelet(p, sp)
    fr = ref_oracle.forward(p, mr, cr, sp, sr, c["recpos"], c["finv"], ntast, True, True)
    fo = oracle.forward(p, mo, co, sp, so, c["recpos"], c["finv"], ntast, True, True)
    for k in ("sections", "dft", "state"):
        assert np.array_equal(fr[k], fo[k]), k
    assert np.abs(fr["state"]).max() > 0 and np.abs(fr["dft"]).max() > 0
    obs = (fr["sections"] * np.float32(0.9)).astype(np.float32)
    dr, l2r = ref_oracle.residual(p, obs, fr["sections"])
    do, l2o = oracle.residual(p, obs, fo["sections"])
    assert np.array_equal(dr, do) and l2r == l2o
    br = ref_oracle.adjoint(p, mr, cr, c["recpos"], dr, c["finv"], ntast, True)
    bo = oracle.adjoint(p, mo, co, c["recpos"], do, c["finv"], ntast, True)
    for k in ("dft", "state"):
        assert np.array_equal(br[k], bo[k]), k
    gr = ref_oracle.gradient(p, mr, c["finv"], fr["dft"], br["dft"])
    go = oracle.gradient(p, mo, c["finv"], fo["dft"], bo["dft"])
    assert np.array_equal(gr, go)
