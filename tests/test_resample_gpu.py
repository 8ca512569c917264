"""Model resampling between multiscale grids (ifosb_resample): against an FP64
numpy restatement of the same rule (bit for bit), and its properties: a
coarse cell's value reappears at the fine cell at the same position, linear
fields are reproduced inside the grid, and values are held constant outside."""
import numpy as np
import pytest

import ifosb
from ifosb import stages

pytestmark = pytest.mark.gpu


def numpy_resample(a, spacing, shape, new_spacing):
    ny, nx, nz = a.shape
    my, mx, mz = shape

    def weights(m, r, n):
        u = np.arange(1, m + 1, dtype=np.float64) * r
        i0 = np.clip(np.floor(u), 1, n).astype(int)
        w = u - i0
        lo, hi = u <= 1.0, u >= n
        i0[lo], w[lo] = 1, 0.0
        i0[hi], w[hi] = n, 0.0
        i1 = np.where(lo | hi, i0, i0 + 1)
        return i0 - 1, i1 - 1, w

    x0, x1, wx = weights(mx, new_spacing[0] / spacing[0], nx)
    y0, y1, wy = weights(my, new_spacing[1] / spacing[1], ny)
    z0, z1, wz = weights(mz, new_spacing[2] / spacing[2], nz)
    A = a.astype(np.float64)
    wz3, wx3, wy3 = wz[None, None, :], wx[None, :, None], wy[:, None, None]

    def S(jj, ii, kk):
        return A[np.ix_(jj, ii, kk)]

    c00 = S(y0, x0, z0) * (1.0 - wz3) + S(y0, x0, z1) * wz3
    c01 = S(y0, x1, z0) * (1.0 - wz3) + S(y0, x1, z1) * wz3
    c10 = S(y1, x0, z0) * (1.0 - wz3) + S(y1, x0, z1) * wz3
    c11 = S(y1, x1, z0) * (1.0 - wz3) + S(y1, x1, z1) * wz3
    c0 = c00 * (1.0 - wx3) + c01 * wx3
    c1 = c10 * (1.0 - wx3) + c11 * wx3
    return (c0 * (1.0 - wy3) + c1 * wy3).astype(np.float32)


def test_resample_matches_numpy_and_keeps_coarse_values():
    rng = np.random.default_rng(2)
    a = rng.uniform(2000, 4500, (10, 12, 8)).astype(np.float32)
    out = stages.resample(a, (2.0, 2.0, 2.0), (20, 24, 16), (1.0, 1.0, 1.0))
    assert np.array_equal(out, numpy_resample(a, (2.0, 2.0, 2.0), (20, 24, 16), (1.0, 1.0, 1.0)))
    # fine cell 2i sits on coarse cell i
    assert np.array_equal(out[1::2, 1::2, 1::2], a)
    # odd spacings and a shrinking grid
    out2 = stages.resample(a, (2.0, 1.5, 3.0), (7, 9, 11), (2.5, 2.0, 2.25))
    assert np.array_equal(out2, numpy_resample(a, (2.0, 1.5, 3.0), (7, 9, 11), (2.5, 2.0, 2.25)))


def test_resample_reproduces_linear_fields():
    ny, nx, nz = 9, 11, 7
    j, i, k = np.meshgrid(np.arange(1, ny + 1), np.arange(1, nx + 1), np.arange(1, nz + 1), indexing="ij")
    a = (3000.0 + 7.0 * i * 2.0 + 3.0 * j * 2.0 - 5.0 * k * 2.0).astype(np.float32)  # linear in position (2 m)
    out = stages.resample(a, (2.0, 2.0, 2.0), (18, 22, 14), (1.0, 1.0, 1.0))
    J, I, K = np.meshgrid(np.arange(1, 19), np.arange(1, 23), np.arange(1, 15), indexing="ij")
    want = 3000.0 + 7.0 * I + 3.0 * J - 5.0 * K
    inside = (I >= 2) & (J >= 2) & (K >= 2) & (I <= 22) & (J <= 18) & (K <= 14)
    assert np.allclose(out[inside], want[inside], rtol=2e-7, atol=0)
    # outside the source grid (position < 2 m) the first cell's value is held
    assert np.array_equal(out[0, 0, 0], a[0, 0, 0])


def test_resample_model_and_errors():
    vp = np.full((4, 5, 6), 3000.0, np.float32)
    vs, rho = vp / np.float32(1.8), np.full_like(vp, 2000.0)
    r = stages.resample_model(vp, vs, rho, (2.0, 2.0, 2.0), (8, 10, 12), (1.0, 1.0, 1.0))
    assert all(x.shape == (8, 10, 12) for x in r) and np.all(r[0] == 3000.0) and np.all(r[2] == 2000.0)
    with pytest.raises(ifosb.IfosbError):
        stages.resample(vp, (0.0, 1.0, 1.0), (2, 2, 2), (1.0, 1.0, 1.0))
