"""ifosb_precon_grad against the reference's precon_grad (oracle/_ref, the
reference's own precongrad.c): bit-identical for every DAMPTYPE, with and without
the free surface, sources and receivers in the grid and near its edges."""
import numpy as np
import pytest

import ifosb
from optim_oracle import RefOptim

pytestmark = pytest.mark.gpu

SHAPE = (40, 44, 36)  # ny, nx, nz


def _ref_precon(ref, grad, damptype, free_surf, fw, dh, src, rec):
    import ctypes as C
    lib = ref.lib
    lib.ifo_ref_precon_grad.restype = C.c_int
    ny, nx, nz = SHAPE
    s = np.ascontiguousarray(src, np.float32)
    r = np.ascontiguousarray(rec, np.int32)
    assert lib.ifo_ref_precon_grad(nx, ny, nz, grad.ctypes.data_as(C.c_void_p), damptype, free_surf, fw,
                                   C.c_float(dh[0]), C.c_float(dh[1]), C.c_float(dh[2]), s.shape[0],
                                   s.ctypes.data_as(C.c_void_p), r.shape[0], r.ctypes.data_as(C.c_void_p)) == 0


@pytest.mark.parametrize("damptype", [0, 1, 2, 3])
@pytest.mark.parametrize("free_surf", [0, 1])
def test_precon_grad_matches_reference(ref_oracle, damptype, free_surf):
    ref = RefOptim()
    rng = np.random.default_rng(10 * damptype + free_surf)
    ny, nx, nz = SHAPE
    dh = (1.0, 1.0, 1.0)
    src = np.array([[12.0, 5.0, 18.0], [30.4, 8.6, 10.0], [1.0, 1.0, 1.0]], np.float32)  # metres
    rec = np.stack([rng.integers(1, nx + 1, 30), np.ones(30, int), rng.integers(1, nz + 1, 30)], 1).astype(np.int32)
    rec[0] = [3, 2, 34]
    g = (1e-3 * rng.standard_normal((3,) + SHAPE)).astype(np.float32)
    a, b = g.copy(), g.copy()
    opt = ifosb.Optimizer(nx, ny, nz)
    opt.precon_grad(a, damptype, free_surf, 10, dh, src, rec)
    _ref_precon(ref, b, damptype, free_surf, 10, dh, src, rec)
    assert np.array_equal(a, b)
    if free_surf and damptype in (0, 1, 2):
        assert not a.any()  # the reference's zero top factor with the free surface
    elif damptype in (1, 2):
        assert np.count_nonzero(a != g) > 0


@pytest.mark.parametrize("fw", [3, 10])
def test_constant_boundary_matches_reference(ref_oracle, fw):
    import ctypes as C
    ref = RefOptim()
    lib = ref.lib
    lib.ifo_ref_constant_boundary.restype = C.c_int
    ny, nx, nz = SHAPE
    rng = np.random.default_rng(fw)
    mshape = (ny + 2, nx + 2, nz + 2)
    m = [(2000 + 500 * rng.random(mshape)).astype(np.float32) for _ in range(3)]
    a = [x.copy() for x in m]
    b = [x.copy() for x in m]
    opt = ifosb.Optimizer(nx, ny, nz)
    opt.constant_boundary(*a, fw)
    p = [x.ctypes.data_as(C.c_void_p) for x in b]
    assert lib.ifo_ref_constant_boundary(nx, ny, nz, fw, *p) == 0
    for x, y, z in zip(a, b, m):
        assert np.array_equal(x, y)
        assert not np.array_equal(x, z)  # the frame was rewritten
