"""GPU engine (through the C ABI) against the CPU oracle, on seeded small cases.

The engine keeps the reference's operand order and promotions and is built
without FMA contraction, so the bar is bit-identity: seismograms, wavefields,
DFT accumulators, residuals and gradients must be EQUAL to the oracle's, not
merely within the 1e-5 / 1e-4 relative-L2 tolerances the project states for
seismograms and gradients (those tolerances are asserted too, as a floor).
For L<=1 the oracle is the reference itself (oracle/_ref) when it is built,
for L>1 the C restatement, which the CPU tests pin to the reference at L<=1."""
import numpy as np
import pytest

import ifosb
from helpers import engine_for, ifo_params, rel_l2
from ifosb import synth

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-5
GRAD_TOL = 1e-4


def pick_oracle(nmech, oracle, request):
    if nmech <= 1:
        try:
            return request.getfixturevalue("ref_oracle")
        except pytest.skip.Exception:
            return oracle
    return oracle


def run_oracle(O, c, m, cp, shots, obs_scale=0.9):
    p = ifo_params(c)
    nf = len(c["finv"])
    out = dict(sections=[], dft=[], state=[], diff=[], l2=[], bdft=[], bstate=[])
    grad = np.zeros((3, p.ny, p.nx, p.nz), np.float32)
    for sp, sig in shots:
        f = O.forward(p, m, cp, sp, sig, c["recpos"], c["finv"] if nf else None, c["ntast"], True, True)
        out["sections"].append(f["sections"])
        out["dft"].append(f["dft"])
        out["state"].append(f["state"])
        if nf:
            obs = (f["sections"] * np.float32(obs_scale)).astype(np.float32)
            d, l2 = O.residual(p, obs, f["sections"])
            out["diff"].append(d)
            out["l2"].append(l2)
            b = O.adjoint(p, m, cp, c["recpos"], d, c["finv"], c["ntast"], True)
            out["bdft"].append(b["dft"])
            out["bstate"].append(b["state"])
            grad = O.gradient(p, m, c["finv"], f["dft"], b["dft"], grad)
    out["grad"] = grad
    return out


def check_case(c, O, obs_scale=0.9, launch_mode=0):
    e, m, cp, shots = engine_for(c)
    e.set_launch_mode(launch_mode)
    ref = run_oracle(O, c, m, cp, shots, obs_scale)
    sec = e.forward(shots)
    nf = len(c["finv"])
    for s in range(len(shots)):
        assert np.array_equal(sec[s], ref["sections"][s]), f"sections shot {s}"
        assert rel_l2(sec[s], ref["sections"][s]) <= SEIS_TOL
        st = e.get_state(s)
        for f in range(9):
            assert np.array_equal(st[f], ref["state"][s][f]), f"state field {f} shot {s}"
        if nf:
            assert np.array_equal(e.get_dft(s), ref["dft"][s]), f"forward DFT shot {s}"
    if not nf:
        return e, ref
    obs = np.stack([(ref["sections"][s] * np.float32(obs_scale)).astype(np.float32) for s in range(len(shots))])
    mis, l2 = e.residual(obs, want_l2_ref=True)
    for s in range(len(shots)):
        d64 = np.asarray(ref["diff"][s], np.float64)
        assert l2[s] == np.float32(ref["l2"][s]), "reference-order float L2"
        assert abs(mis[s] - float((d64 * d64).sum())) <= 1e-12 * float((d64 * d64).sum()) + 1e-300
    e.adjoint()
    for s in range(len(shots)):
        assert np.array_equal(e.get_dft(s, back=True), ref["bdft"][s]), f"backward DFT shot {s}"
        st = e.get_state(s)
        for f in range(9):
            assert np.array_equal(st[f], ref["bstate"][s][f]), f"adjoint state field {f} shot {s}"
    e.gradient()
    g = e.get_gradient()
    assert np.array_equal(g, ref["grad"]), "gradient"
    assert rel_l2(g, ref["grad"]) <= GRAD_TOL
    g64 = e.get_gradient(fp64=True)
    assert rel_l2(g64, ref["grad"]) < 1e-5
    return e, ref


CASES = [
    dict(nmech=0, free_surf=1),
    dict(nmech=0, free_surf=0),
    dict(nmech=0, free_surf=1, fdcoeff=1),
    dict(nmech=1, free_surf=1),
    dict(nmech=1, free_surf=0),
    dict(nmech=3, free_surf=1),
    dict(nmech=2, free_surf=0),
]


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "-".join(f"{a}{b}" for a, b in k.items()))
def test_shot_gradient_bit_exact(kw, oracle, request):
    c = synth.small_case(nt=80, **kw)
    check_case(c, pick_oracle(kw["nmech"], oracle, request))


def test_batched_shots_match_sequential_oracle(oracle, request):
    """Three shots in one launch == three sequential reference shots, and the
    gradient accumulates in the reference's shot order."""
    c = synth.small_case(nt=70, nshots=3, nsrc=2, seed=5)
    check_case(c, pick_oracle(0, oracle, request))


def test_plain_launch_mode_matches(oracle, request):
    c = synth.small_case(nt=40, nmech=1, seed=7)
    check_case(c, pick_oracle(1, oracle, request), launch_mode=1)


@pytest.mark.parametrize("nmech", [0, 3])
def test_untiled_kernels_match(nmech, oracle, request, monkeypatch):
    """The kernels without TMA staging (IFOSB_TMA=0) give the same bits."""
    monkeypatch.setenv("IFOSB_TMA", "0")
    c = synth.small_case(nt=50, nmech=nmech, seed=13, nshots=2)
    check_case(c, pick_oracle(nmech, oracle, request))


def test_tile_edges_and_long_chunks(oracle, request):
    """Grid sizes that are not multiples of the 32x8 tile, several shots, and a y
    extent long enough for multi-plane chunks with ring reuse."""
    c = synth.small_case(nx=37, ny=70, nz=45, nt=30, fw=6, nshots=3, seed=17)
    check_case(c, pick_oracle(0, oracle, request))


@pytest.mark.parametrize("stype", [2, 3, 4, 5])
def test_body_force_sources(stype, oracle, request):
    """Single forces (update_v_ssg.c:474-510), including the reference's rjp/rkp
    pairing for types 3 and 4 and the custom-angle type 5."""
    c = synth.small_case(nt=50, nsrc=3, stype=stype, seed=11, finv=())
    p = c["params"]
    if stype == 5:
        p.alpha, p.beta = 30.0, 60.0
    check_case(c, pick_oracle(0, oracle, request))


def test_edges_points_in_frame_and_shared_cells(oracle, request):
    """Receivers and sources inside the CPML frame, at the surface row j=1, and
    two receivers in one cell (both inject twice, in list order)."""
    c = synth.small_case(nt=60, ntr=6, seed=3)
    c["recpos"] = np.array([[1, 1, 1], [c["params"].nx, c["params"].ny, c["params"].nz], [5, 2, 7],
                            [5, 2, 7], [12, 1, 11], [3, 20, 20]], np.int32)
    c["shots"][0][0, :3] = [2, 1, 2]
    check_case(c, pick_oracle(0, oracle, request))


def test_forward_only_method0(oracle, request):
    c = synth.small_case(nt=60, finv=(), nmech=1)
    check_case(c, pick_oracle(1, oracle, request))


def test_unstable_run_reports_error():
    """A CFL-violating time step trips the NaN probe (ifos3d.c:761) and comes back
    as IFOSB_EUNSTABLE; the engine stays usable afterwards."""
    c = synth.small_case(nt=400, finv=())
    p = c["params"]
    p.dt = np.float32(1e-3)  # vp*DT/DH = 3 >> CFL limit
    e, m, cp, shots = engine_for(c)
    with pytest.raises(ifosb.IfosbError) as ei:
        e.forward(shots)
    assert ei.value.code == ifosb.EUNSTABLE
    e2, _, _, shots2 = engine_for(synth.small_case(nt=20, finv=()))
    assert np.isfinite(e2.forward(shots2)).all()


def test_call_order_errors():
    c = synth.small_case(nt=20)
    e, m, cp, shots = engine_for(c)
    with pytest.raises(ifosb.IfosbError) as ei:
        e.adjoint()
    assert ei.value.code == ifosb.ESTATE
    with pytest.raises(ifosb.IfosbError) as ei:
        e.gradient()
    assert ei.value.code == ifosb.ESTATE
    bad = [(np.array([[0, 1, 1, 0, 100, 1, 1]], np.float32), shots[0][1])]
    with pytest.raises(ifosb.IfosbError) as ei:
        e.forward(bad)
    assert ei.value.code == ifosb.EARG


def test_autotuned_launch_shape_gives_the_same_bits():
    """ifosb_autotune picks a launch shape (y planes per CTA chunk, L2 prefetch
    distance); forward traces and the shot gradient are the same bits as with
    the built-in shape."""
    c = synth.small_case(nx=37, ny=70, nz=45, nt=40, fw=6, nshots=3, seed=17)
    e1, m, cp, shots = engine_for(c)
    e2, _, _, _ = engine_for(c)
    shape = e2.autotune(shots, steps=4)
    for k in ("velocity", "stress"):
        assert 2 <= shape[k]["y_planes_per_cta"] <= 64
        assert shape[k]["l2_prefetch_planes"] in (0, 1, 2, 3)
    out = []
    for e in (e1, e2):
        sec = e.forward(shots)
        obs = (sec * np.float32(0.9)).astype(np.float32)
        mis = e.shot_gradient(shots, obs)
        out.append((sec, mis, e.get_gradient()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_set_launch_shape_reuses_a_tuned_shape():
    """A shape set directly (as a caller that saved an autotuned shape would)
    gives the same bits as the default shape, including odd chunk lengths and
    prefetch off; out-of-range shapes are rejected with a message."""
    import ifosb
    c = synth.small_case(nx=37, ny=70, nz=45, nt=40, fw=6, nshots=3, seed=19)
    e1, m, cp, shots = engine_for(c)
    e2, _, _, _ = engine_for(c)
    e2.set_launch_shape(len(shots), [5, 0, 7, 2])
    out = []
    for e in (e1, e2):
        sec = e.forward(shots)
        obs = (sec * np.float32(0.9)).astype(np.float32)
        mis = e.shot_gradient(shots, obs)
        out.append((sec, mis, e.get_gradient()))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    for bad in ([0, 1, 4, 1], [4, 9, 4, 1], [4, 1, 71, 1], [4, 1, 4, -1]):
        with pytest.raises(ifosb.IfosbError):
            e2.set_launch_shape(len(shots), bad)


@pytest.mark.parametrize("rows", [7, 8])
@pytest.mark.parametrize("nmech", [0, 3])
def test_tile_heights_match(rows, nmech, oracle, request, monkeypatch):
    """Both tile heights of both TMA kernels (by default the velocity kernel
    uses 8-row tiles, the stress kernel 7-row tiles with memory variables and
    8-row tiles without) give the reference's bits for either model kind, on a
    grid that is not a multiple of either."""
    monkeypatch.setenv("IFOSB_TILE_ROWS", str(rows))
    monkeypatch.setenv("IFOSB_VEL_TILE_ROWS", str(rows))
    c = synth.small_case(nx=37, ny=30, nz=35, nt=40, fw=5, nmech=nmech, nshots=2, seed=23)
    check_case(c, pick_oracle(nmech, oracle, request))


def test_time_loop_graph_is_reused():
    """Repeated shot gradients with the same batch shape replay the captured
    forward and adjoint graphs, also across model changes: no new capture once
    the first shot gradient after a model change has run."""
    c = synth.small_case(nt=30, nshots=2, seed=29)
    e, m, cp, shots = engine_for(c)
    sec = e.forward(shots)
    obs = (sec * np.float32(0.9)).astype(np.float32)
    e.shot_gradient(shots, obs)
    e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
    e.shot_gradient(shots, obs)
    steady = e.graph_captures
    assert 2 <= steady <= 4
    for _ in range(3):
        e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
        e.shot_gradient(shots, obs)
    assert e.graph_captures == steady


def test_alternating_batch_shapes_keep_their_graphs():
    """Full batches and a shorter last batch alternate in a multi-batch gradient;
    each shape keeps its own captured graph, so alternating captures nothing new."""
    c = synth.small_case(nt=30, nshots=3, seed=31)
    e, m, cp, shots = engine_for(c)
    full = e.forward(shots[:2])
    part = e.forward(shots[2:])
    steady = e.graph_captures
    for _ in range(3):
        assert np.array_equal(e.forward(shots[:2]), full)
        assert np.array_equal(e.forward(shots[2:]), part)
    assert e.graph_captures == steady
    e.close()
