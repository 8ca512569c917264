"""bench.py on the CPU: the reference arm's JSON line (the CPU implementation of
the path, timed on this host's cores) and the algorithmic-byte model that the
roofline fractions divide by."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _last_json(out):
    return json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])


@pytest.mark.parametrize("workload,kind", [("visco384", "port"), ("visco256", "port"), ("elastic128", None)])
def test_reference_arm_prints_the_contract_line(workload, kind):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", workload,
                        "--steps", "1", "--warmup", "0", "--cpu-procs", "1", "--cpu-nt", "3"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    d = _last_json(r.stdout)
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["value"] > 0 and d["unit"] == "Gcell-updates/s" and d["higher_is_better"] is True
    assert d["config"]["workload"].startswith(workload)
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] == 1 and cb["kind"] in ("reference", "port") and cb["sample"]
    assert cb["cpu_model"]
    if kind:
        assert cb["kind"] == kind  # L=3 has no reference implementation: the restatement runs
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_algorithmic_bytes_per_cell_step():
    """The per-cell byte model of the roofline: visco256 (L=3, FW=10 CPML, free
    surface, no DFT) 245.38 B; elastic128 with two DFT frequencies 198.75 B; the
    batched visco384 gradient (L=3, four DFT frequencies) 434.875 B."""
    import bench
    sys.path.insert(0, os.path.join(ROOT, "ifos3d-dev_b200"))
    from ifosb import synth
    for name, nf, want in (("visco256", 0, 245.38), ("elastic128", 2, 198.75), ("visco384", 4, 434.88)):
        p = synth.case(name, nt=4)["params"]
        b = bench.alg_bytes_per_cell_step(p, nf, 1)
        assert round(b["total"], 2) == want, (name, b)
        assert abs(b["vel"] + b["stress"] - b["total"]) < 1e-9
