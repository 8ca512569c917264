"""The drop-in host: the reference program ifos3d, reading its own JSON
parameter file and writing its own files, with its time loops on the B200
engine (ifos3d-dev_b200/host: the reference's src/ifos3d.c compiled with its
time-loop calls sent through the C ABI), against the unmodified reference
program built from the same sources on one rank (oracle/_ref/ifos3d_ref).

Both run the same input directory (READMOD=1 model files, sources, receivers,
workflow, observed SU data written by the reference's own METHOD=0 run):
- METHOD=0: the SU seismograms of every shot;
- METHOD=1, one iteration: the SU seismograms, the raw, preconditioned and
  conjugated gradient files (GRAD_FILE _it1, _it1001, _it2001; src/ifos3d.c:1000,
  1006, 1016), the model files (MOD_OUT_FILE _it0, _it1) after the step-length
  search, and the driver's misfit log (in_and_out/ifos3D_invers.out)
must be equal byte for byte. The free-surface case also covers the step-length
forwards' use of the current model's moduli at the surface (src/ifos3d.c:1087-1090).
"""
import filecmp
import os
import shutil
import subprocess

import pytest

from host_case import models, write_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ifos3d_ref")
HOST_BIN = os.path.join(ROOT, "ifos3d-dev_b200", "host", "_build", "ifos3d_b200")


def _need_binaries():
    for b in (REF_BIN, HOST_BIN):
        if not os.path.exists(b):
            pytest.skip(f"{b} not built (make -C oracle ref; make -C ifos3d-dev_b200/host)")


def _run(binary, d):
    r = subprocess.run([binary, "run.json"], cwd=d, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"{binary} in {d}: rc={r.returncode}\n{r.stdout[-3000:]}\n{r.stderr[-2000:]}"
    return r.stdout


def _compare_trees(a, b, subdirs):
    n = 0
    for sub in subdirs:
        fa = sorted(os.listdir(os.path.join(a, sub)))
        fb = sorted(os.listdir(os.path.join(b, sub)))
        assert fa == fb, (sub, fa, fb)
        for f in fa:
            pa, pb = os.path.join(a, sub, f), os.path.join(b, sub, f)
            assert filecmp.cmp(pa, pb, shallow=False), f"{sub}/{f} differs"
            n += 1
    return n


CASES = [
    dict(name="toy-like", free_surf=0, damptype=2, seismo=1),
    dict(name="free-surface", free_surf=1, damptype=4, seismo=4),  # DAMPTYPE 4: no damping
]


@pytest.mark.parametrize("kw", CASES, ids=lambda k: k["name"])
def test_dropin_host_matches_the_reference_program(kw, tmp_path):
    _need_binaries()
    kw = {k: v for k, v in kw.items() if k != "name"}
    true, start = models(40, 40, 40)
    # observed data: the reference's own forward in the true model (METHOD=0), and
    # the drop-in host's on the same input: the SU files must agree
    obs = {}
    for who, binary in (("ref", REF_BIN), ("b200", HOST_BIN)):
        d = str(tmp_path / f"obs_{who}")
        write_case(d, method=0, model=true, seis_file="su_obs/obs", mfile="model/true", **kw)
        _run(binary, d)
        obs[who] = d
    assert _compare_trees(obs["ref"], obs["b200"], ["su_obs"]) >= 6
    # one inversion iteration from the start model with the reference's observed data
    inv = {}
    for who, binary in (("ref", REF_BIN), ("b200", HOST_BIN)):
        d = str(tmp_path / f"inv_{who}")
        write_case(d, method=1, model=start, **kw)
        for f in os.listdir(os.path.join(obs["ref"], "su_obs")):
            shutil.copy(os.path.join(obs["ref"], "su_obs", f), os.path.join(d, "su_obs", f))
        _run(binary, d)
        inv[who] = d
    n = _compare_trees(inv["ref"], inv["b200"], ["su", "grad", "model"])
    assert n >= 6 + 9 + 6
    assert filecmp.cmp(os.path.join(inv["ref"], "in_and_out", "ifos3D_invers.out"),
                       os.path.join(inv["b200"], "in_and_out", "ifos3D_invers.out"), shallow=False)
    # the run did something: the raw gradient is not zero and the model moved
    raw = open(os.path.join(inv["ref"], "grad", "g.vp_400.00Hz_it1"), "rb").read()
    assert any(raw)
    assert not filecmp.cmp(os.path.join(inv["ref"], "model", "out.vp_it0"),
                           os.path.join(inv["ref"], "model", "out.vp_it1"), shallow=False)
