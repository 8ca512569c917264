"""Multiscale stages: the FILT Butterworth filter (csrc/ifosb_filter.c) and the
workflow reader (ifosb.stages.read_inv) against the reference's filt_seis and
readinv and libcseife's seife_lpb / seife_hpb. All are built from the reference
sources into oracle/_ref. The filter must give the reference's bits."""
import ctypes as C

import numpy as np
import pytest

import ifosb
from ifosb import stages


@pytest.fixture(scope="module")
def ref(ref_oracle):
    from pyoracle import REF_LIB
    lib = C.CDLL(REF_LIB)
    lib.ifo_ref_filt_seis.restype = C.c_int
    lib.ifo_ref_readinv.restype = C.c_int
    for n in ("seife_lpb", "seife_hpb"):
        getattr(lib, n).restype = None
        getattr(lib, n).argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int]
    return lib


def P(a):
    return a.ctypes.data_as(C.c_void_p)


def traces(seed, ntr, ns, dt):
    rng = np.random.default_rng(seed)
    t = np.arange(ns) * dt
    x = rng.standard_normal((ntr, ns)) * 0.1
    x += np.sin(2 * np.pi * 20.0 * t) + 0.5 * np.sin(2 * np.pi * 180.0 * t + 0.3)
    x *= 10.0 ** rng.integers(-9, 2, size=(ntr, 1))
    return x.astype(np.float32)


@pytest.mark.parametrize("finv,dt", [(30.0, 1e-3), (450.0, 1e-4), (7.5, 2e-3)])
def test_filt_seis_matches_reference(ref, finv, dt):
    data = traces(1, 6, 777, dt)
    a = data.copy()
    assert ref.ifo_ref_filt_seis(P(a), a.shape[0], a.shape[1], C.c_float(finv), C.c_float(dt)) == 0
    b = stages.filt_seis(data, finv, dt)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(b[:, -1], data[:, -1])  # the reference leaves the last sample unfiltered
    assert not np.array_equal(b[:, :-1], data[:, :-1])


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5, 8])
@pytest.mark.parametrize("highpass", [False, True])
def test_butterworth_cascade_matches_cseife(ref, order, highpass):
    """Every order and both kinds against libcseife itself. ifosb_filt_seis
    filters (0, s_1..s_{ns-1}), as filt_seis does, so cseife gets that vector."""
    dt, finv = 1e-3, 40.0
    data = traces(2, 3, 500, dt)
    ours = data.copy()
    rc = ifosb.lib().ifosb_filt_seis(P(ours), 3, 500, C.c_float(finv), C.c_float(dt), order, 1 if highpass else 0)
    assert rc == 0
    T0 = 1.0 / np.float64(np.float32(finv))
    for t in range(3):
        x = np.concatenate([[0.0], data[t, :-1].astype(np.float64)])
        fn = ref.seife_hpb if highpass else ref.seife_lpb
        fn(P(x), len(x), float(np.float32(dt)), T0, order)
        assert np.array_equal(ours[t, :-1], x[1:].astype(np.float32))


def test_lowpass_properties():
    dt, ns = 1e-3, 4000
    t = np.arange(ns) * dt
    dc = np.ones((1, ns), np.float32)
    y = stages.filt_seis(dc, 25.0, dt)
    assert abs(y[0, -2] - 1.0) < 1e-5  # unit gain at zero frequency
    hi = np.sin(2 * np.pi * 300.0 * t)[None].astype(np.float32)
    y = stages.filt_seis(hi, 25.0, dt)
    assert np.abs(y[0, 2000:-1]).max() < 1e-3  # 12 octave-dB/octave x 3.6 octaves


WORKFLOW = """1 3 0.01 0 0.0 0.0 0.0 0.0 2 300.0 450.0
1 2 0.01 0 0.0 0.0 0.0 0.0 3 300.0 450.0 600.5
2 5 0.02 1 0.1 0.2 0.3 0.4 1 750.25
"""


def test_read_inv_matches_readinv(ref, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)  # the reference keeps INV_FILE in a char[74]
    open("workflow.txt", "w").write(WORKFLOW)
    for g in (1, 2, 3):
        finv = np.zeros(8, np.float32)
        nf, it = C.c_int(0), np.zeros(2, np.int32)
        assert ref.ifo_ref_readinv(b"workflow.txt", g, P(finv), C.byref(nf), P(it), 8) == g
        st = stages.read_inv("workflow.txt", g)
        assert (st.itmin, st.itmax) == (it[0], it[1])
        assert len(st.finv) == nf.value
        assert np.array_equal(np.float32(st.finv), finv[:nf.value])
    st = stages.read_inv("workflow.txt", 3)
    assert st.mute == 1 and st.owin == (float(np.float32(0.3)), float(np.float32(0.4)))
    assert [s.itmax for s in stages.read_workflow("workflow.txt", 3)] == [3, 2, 5]
    with pytest.raises(ifosb.IfosbError):
        stages.read_inv("workflow.txt", 4)
