"""On-disk formats: ifosb.io (csrc/ifosb_io.c) against the reference's own writers
and readers (outseis, saveseis, outmod + mergemod, outgrad, readseis,
readseis_split), built from the reference sources into oracle/_ref and driven
by oracle/ref_io.c on one rank.

Files must match byte for byte. The exceptions are the SU header bytes that
outseis.c never assigns (cdp, selev, swdep and the trailing pad: stack garbage
in the reference, zeros here). Those are masked in both files before comparing.

The reference builds file names in char[74] buffers (fd.h STRING_SIZE), so every
test works in its temporary directory with short relative names. The library
has no such limit.
"""
import ctypes as C
import os

import numpy as np
import pytest

import ifosb
from ifosb import io as fio

# byte ranges of each 240-byte SU header that outseis() leaves unassigned
UNASSIGNED = [(20, 24), (44, 48), (60, 64), (210, 240)]
GEOM = dict(dx=0.8, dy=1.25, dz=0.7, ndt=2, dt=3.3e-4)


@pytest.fixture(scope="module")
def ref(ref_oracle):
    from pyoracle import REF_LIB
    lib = C.CDLL(REF_LIB)
    for n in ("ifo_ref_outseis", "ifo_ref_saveseis", "ifo_ref_readseis", "ifo_ref_readseis_split",
              "ifo_ref_outmod", "ifo_ref_outgrad", "ifo_ref_readhess"):
        getattr(lib, n).restype = C.c_int
    return lib


@pytest.fixture
def wd(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    import pathlib
    return pathlib.Path(".")


def P(a):
    return a.ctypes.data_as(C.c_void_p)


def f(x):
    return C.c_float(x)


def case(seed, ntr=7, ns=53):
    rng = np.random.default_rng(seed)
    sec = (rng.standard_normal((ntr, ns)) * 10.0 ** rng.integers(-12, 3, size=(ntr, 1))).astype(np.float32)
    sec[0, :5] = 0.0
    sec[1, 3] = -0.0
    rec = np.stack([rng.integers(1, 60, ntr), rng.integers(1, 40, ntr), rng.integers(1, 50, ntr)], 1).astype(np.int32)
    tn = np.sort(rng.choice(np.arange(1, 4 * ntr + 1), ntr, replace=False)).astype(np.int32)
    src = np.array([21.3, 3.7, 17.9], np.float32)
    return sec, np.ascontiguousarray(rec), tn, src


def masked(path, ntr, ns):
    """File bytes with the unassigned header bytes zeroed. A merged file may hold
    no traces: without RUN_MULTIPLE_SHOTS saveseis.c writes rank files without
    the shot number but merges the ones with it (saveseis.c:49-63 vs :92), so
    its merged files are empty, and so are ours."""
    b = bytearray(open(path, "rb").read())
    rec = 240 + 4 * ns
    assert len(b) % rec == 0 and len(b) // rec in (0, ntr)
    for t in range(len(b) // rec):
        for a, e in UNASSIGNED:
            b[t * rec + a:t * rec + e] = bytes(e - a)
    return bytes(b)


def ref_outseis(ref, path, sec, rec, tn, src, fmt, littlebig=0, comp=2):
    ntr, ns = sec.shape
    g = GEOM
    assert ref.ifo_ref_outseis(os.fsencode(path), comp, P(sec), ntr, ns, P(rec), P(tn), P(src), f(g["dx"]),
                               f(g["dy"]), f(g["dz"]), g["ndt"], f(g["dt"]), fmt, littlebig) == 0


@pytest.mark.parametrize("fmt", [0, 1])
def test_su_writer_matches_outseis(ref, wd, fmt):
    sec, rec, tn, src = case(1)
    ntr, ns = sec.shape
    a, b = str(wd / "ref.su"), str(wd / "ours.su")
    ref_outseis(ref, a, sec, rec, tn, src, fmt)
    fio.write_seis(b, sec, rec, comp=2, trace_no=tn, src=src, fmt=fmt, **GEOM)
    assert masked(a, ntr, ns) == masked(b, ntr, ns)
    # spot checks of the header we write
    h = open(b, "rb").read(240)
    assert int.from_bytes(h[0:4], "little", signed=True) == tn[0]
    assert int.from_bytes(h[114:116], "little") == ns
    assert int.from_bytes(h[116:118], "little") == round(GEOM["ndt"] * GEOM["dt"] * 1e6)
    assert int.from_bytes(h[68:70], "little", signed=True) == -3


def test_ascii_and_binary_writers_match_outseis(ref, wd):
    sec, rec, tn, src = case(2, ntr=4, ns=11)
    for fmt, lb in ((2, 0), (3, 0), (3, 1)):
        a, b = str(wd / f"ref{fmt}{lb}"), str(wd / f"ours{fmt}{lb}")
        ref_outseis(ref, a, sec, rec, tn, src, fmt, lb)
        fio.write_seis(b, sec, rec, trace_no=tn, src=src, fmt=fmt, littlebig=bool(lb), **GEOM)
        assert open(a, "rb").read() == open(b, "rb").read(), (fmt, lb)
    sw = np.fromfile(str(wd / "ours31"), np.float32).byteswap().reshape(sec.shape)
    assert np.array_equal(sw.view(np.uint32), sec.view(np.uint32))


@pytest.mark.parametrize("obs,iteration,multiple", [(0, 3, 1), (1, 1, 1), (0, 0, 0)])
def test_save_seis_matches_saveseis(ref, wd, obs, iteration, multiple):
    ntr, ns = 5, 37
    rng = np.random.default_rng(3)
    secs = rng.standard_normal((3, ntr, ns)).astype(np.float32)
    _, rec, tn, _ = case(3, ntr, ns)
    srcpos = np.array([[11.0, 2.0, 9.5], [30.25, 4.5, 12.0]], np.float32)
    ishot = 2
    rdir, odir = wd / "ref", wd / "ours"
    rdir.mkdir()
    odir.mkdir()
    g = GEOM
    base = "seis"
    r_seis, r_obs = str(rdir / base), str(rdir / "obs")
    assert ref.ifo_ref_saveseis(os.fsencode(r_seis), os.fsencode(r_obs), P(secs), ntr, ns, P(rec), P(tn), P(srcpos),
                                2, ishot, obs, iteration, 1, multiple, 1, f(g["dx"]), f(g["dy"]), f(g["dz"]),
                                g["ndt"], f(g["dt"])) == 0
    o_base = str(odir / ("obs" if obs else base))
    fio.save_seis(o_base, secs, rec, srcpos[ishot - 1], ishot=ishot, iteration=iteration, fmt=1, obs=bool(obs),
                  method=True, multiple_shots=bool(multiple), trace_no=tn, **g)
    rf, of = sorted(os.listdir(rdir)), sorted(os.listdir(odir))
    assert rf == of and len(rf) >= 3
    for name in rf:
        assert masked(rdir / name, ntr, ns) == masked(odir / name, ntr, ns), name


def test_read_seis_matches_readseis(ref, wd):
    sec, rec, tn, src = case(4, ntr=6, ns=29)
    ntr, ns = sec.shape
    obs = str(wd / "obs")
    ishot, comp = 3, 2
    for multiple in (1, 0):
        path = fio.obs_file(obs, fio.COMPONENTS[comp - 1], ishot, 0, bool(multiple))
        fio.write_seis(path, sec, rec, trace_no=tn, src=src, **GEOM)
        out_ref = np.full((ntr, ns), 7.0, np.float32)
        assert ref.ifo_ref_readseis(os.fsencode(obs), ishot, P(out_ref), ntr, ns, comp, multiple) == 0
        ours = fio.read_seis(path, ntr, ns)
        assert np.array_equal(out_ref.view(np.uint32), ours.view(np.uint32))
        assert np.array_equal(ours, sec)
    # a file that ends early: the missing samples read as 0 in both
    path = fio.obs_file(obs, "vy", ishot, 0, True)
    data = open(path, "rb").read()
    open(path, "wb").write(data[: 2 * (240 + 4 * ns) + 240 + 4 * 10])
    out_ref = np.zeros((ntr, ns), np.float32)
    assert ref.ifo_ref_readseis(os.fsencode(obs), ishot, P(out_ref), ntr, ns, 2, 1) == 0
    ours = fio.read_seis(path, ntr, ns)
    assert np.array_equal(out_ref, ours)
    assert np.array_equal(ours[2, :10], sec[2, :10]) and not ours[2, 10:].any() and not ours[3:].any()


def test_read_seis_split_matches_readseis_split(ref, wd):
    sec, rec, tn, src = case(5, ntr=9, ns=17)
    ntr, ns = sec.shape
    obs = str(wd / "ext")
    ishot = 1
    path = fio.obs_split_file(obs, "vz", ishot)
    fio.write_seis(path, sec, rec, trace_no=tn, src=src, **GEOM)
    keep = np.array([1, 0, 0, 1, 1, 0, 1, 0, 1], np.int32)
    out_ref = np.zeros((ntr, ns), np.float32)
    k = ref.ifo_ref_readseis_split(os.fsencode(obs), ishot, P(out_ref), ntr, P(keep), ns, 3)
    ours = fio.read_seis_split(path, keep, ns)
    assert k == ours.shape[0] == 5
    assert np.array_equal(out_ref[:k], ours)
    assert np.array_equal(ours, sec[keep == 1])


def ghost_models(seed, ny, nx, nz):
    rng = np.random.default_rng(seed)
    rho = rng.uniform(1500, 2600, (ny + 2, nx + 2, nz + 2)).astype(np.float32)
    vp = rng.uniform(2000, 4500, rho.shape).astype(np.float32)
    vs = (vp / np.float32(1.8)).astype(np.float32)
    pi = (rho * vp * vp).astype(np.float32)
    u = (rho * vs * vs).astype(np.float32)
    return rho, pi, u


@pytest.mark.parametrize("ids", [(1, 1, 1), (2, 1, 3)])
def test_write_model_matches_outmod(ref, wd, ids):
    ny, nx, nz = 6, 5, 7
    rho, pi, u = ghost_models(6, ny, nx, nz)
    a, b, c = str(wd / "ref_mod"), str(wd / "ours_mod"), str(wd / "dense_mod")
    assert ref.ifo_ref_outmod(os.fsencode(a), 4, nx, ny, nz, P(rho), P(pi), P(u), *ids) == 0
    fio.write_model(b, 4, rho, pi, u, ghosted=True, idx=ids[0], idy=ids[1], idz=ids[2])
    inner = [np.ascontiguousarray(x[1:-1, 1:-1, 1:-1]) for x in (rho, pi, u)]
    fio.write_model(c, 4, *inner, idx=ids[0], idy=ids[1], idz=ids[2])
    for q in ("vp", "vs", "rho"):
        ra = open(f"{a}.{q}_it4", "rb").read()
        assert ra == open(f"{b}.{q}_it4", "rb").read() == open(f"{c}.{q}_it4", "rb").read(), q
    assert sorted(p for p in os.listdir(wd) if p.startswith("ref_mod")) == \
        ["ref_mod.rho_it4", "ref_mod.vp_it4", "ref_mod.vs_it4"]  # the rank files are removed
    if ids == (1, 1, 1):
        vp = np.fromfile(f"{b}.vp_it4", np.float32).reshape(nz, nx, ny)
        want = np.sqrt((inner[1] / inner[0]).astype(np.float64)).astype(np.float32).transpose(2, 1, 0)
        assert np.array_equal(vp, want)


@pytest.mark.parametrize("ids", [(1, 1, 1), (1, 2, 2)])
def test_write_gradient_matches_outgrad(ref, wd, ids):
    ny, nx, nz = 5, 4, 6
    rng = np.random.default_rng(7)
    g = (rng.standard_normal((3, ny, nx, nz)) * 1e-9).astype(np.float32)
    a, b = str(wd / "ref_grad"), str(wd / "ours_grad")
    assert ref.ifo_ref_outgrad(os.fsencode(a), f(12.5), 1003, nx, ny, nz, P(g), *ids) == 0
    fio.write_gradient(b, 12.5, 1003, g, idx=ids[0], idy=ids[1], idz=ids[2])
    for q in ("vp", "vs", "rho"):
        assert open(f"{a}.{q}_12.50Hz_it1003", "rb").read() == open(f"{b}.{q}_12.50Hz_it1003", "rb").read()


def test_io_errors(wd):
    with pytest.raises(ifosb.IfosbError) as e:
        fio.read_seis(str(wd / "missing.su"), 3, 10)
    assert e.value.code == ifosb.EIO
    sec, rec, tn, src = case(8, ntr=2, ns=5)
    with pytest.raises(ifosb.IfosbError) as e:
        fio.write_seis(str(wd / "x"), sec, rec, fmt=7, **GEOM)
    assert e.value.code == ifosb.EARG
    with pytest.raises(ifosb.IfosbError):
        fio.write_seis(str(wd / "no_dir" / "x.su"), sec, rec, **GEOM)
    assert fio.merge_seis(str(wd / "m.su"), [str(wd / "none")], 5) == 0


def test_read_hessian_matches_readhess(ref, wd):
    """Hessian files as outgrad writes them (HESS_FILE), read back as readhess
    does: scaled by VP0^2, VS0^2, RHO0^2."""
    ny, nx, nz = 5, 6, 4
    rng = np.random.default_rng(9)
    h = (rng.uniform(0.0, 1.0, (3, ny, nx, nz)) * 1e-12).astype(np.float32)
    fio.write_gradient("hess", 7.25, 1, h)
    out_ref = np.zeros_like(h)
    assert ref.ifo_ref_readhess(b"hess", f(7.25), 1, nx, ny, nz, f(3100.0), f(1790.0), f(2250.0), P(out_ref)) == 0
    ours = fio.read_hessian("hess", 7.25, 1, ny, nx, nz, 3100.0, 1790.0, 2250.0)
    assert np.array_equal(out_ref.view(np.uint32), ours.view(np.uint32))
    assert np.allclose(ours[0], h[0] * 3100.0 ** 2, rtol=1e-6)
    with pytest.raises(ifosb.IfosbError):
        fio.read_hessian("nohess", 7.25, 1, ny, nx, nz, 1.0, 1.0, 1.0)
