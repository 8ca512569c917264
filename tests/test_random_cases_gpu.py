"""Seeded random cases through the whole shot gradient (forward, residual,
adjoint, DFT gradient) against the oracle, bit for bit. The parameters are
drawn at random: grid sizes that are not tile multiples, CPML width, free
surface, Taylor or Holberg coefficients, 0-3 relaxation mechanisms, 1-3 shots
of 1-2 sources, 1-12 receivers, 0-2 frequencies and the DFT interval. The
reference build is the oracle for L <= 1, the C restatement above."""
import numpy as np
import pytest

from test_gpu_parity import check_case, pick_oracle
from ifosb import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", range(24))
def test_random_case(seed, oracle, request):
    rng = np.random.default_rng(1000 + seed)
    fw = int(rng.integers(3, 7))
    nx, ny, nz = (int(rng.integers(2 * fw + 6, 2 * fw + 30)) for _ in range(3))
    nmech = int(rng.choice([0, 0, 1, 1, 2, 3]))
    nf = int(rng.integers(0, 3))
    finv = tuple(float(f) for f in rng.choice([250.0, 300.0, 420.0, 600.0], nf, replace=False))
    c = synth.small_case(nx=nx, ny=ny, nz=nz, nt=int(rng.integers(30, 70)), fw=fw,
                         free_surf=int(rng.integers(0, 2)), nmech=nmech, fdcoeff=int(rng.integers(1, 3)),
                         seed=seed, nshots=int(rng.integers(1, 4)), nsrc=int(rng.integers(1, 3)),
                         ntr=int(rng.integers(1, 13)), finv=finv)
    c["ntast"] = int(rng.integers(1, 4))
    check_case(c, pick_oracle(nmech, oracle, request))
