"""CPU oracle of the inversion-loop updates — TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's optimiser functions in two precisions:
  * ``prec="ref"``  : the reference's own float arithmetic — float32 storage,
    float products, and dot products summed one term at a time in float, in the
    reference's loop order. Pinned bit for bit against the reference build
    (oracle/_ref, functions driven by oracle/ref_optim.c).
  * ``prec="fp64"`` : what the engine computes — the same steps with every dot
    product, scalar and the L-BFGS work vector in float64, sums exactly rounded
    (math.fsum), float32 gradients and models in and out. The GPU results are
    compared with this, and their error against it is stated in the tests.

Sources restated:
  conjugate      src/conjugategrad.c:27-110
  lbfgs_savegrad src/lbfgs_save.c:25-56
  lbfgs          src/lbfgs.c:26-181
  steplength     src/steplength.c:26-91
  modelupdate    src/modelupdate.c:26-160
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def _sum(terms, prec):
    """The reference: `acc += term` in float from 0 (loop order); fp64: exactly rounded."""
    if prec == "ref":
        t = np.ascontiguousarray(terms, np.float32).ravel()
        return f32(np.add.accumulate(t, dtype=np.float32)[-1]) if t.size else f32(0.0)
    return math.fsum(np.asarray(terms, np.float64).ravel())


def conjugate(grad, prior, cdf, prec="ref"):
    """conjugategrad.c:27-110. grad [3][n], prior [6][n] (float32, updated in
    place). Returns beta[3]. Only beta[0] is clamped (the clamps all test
    beta[0], :86-91)."""
    assert grad.shape[0] == 3 and prior.shape[0] == 6
    beta = [0.0, 0.0, 0.0]
    if cdf == 1:  # :43-56
        prior[0:3] = grad
        prior[3:6] = grad
        return np.array(beta, np.float64)
    sums = []
    for c in range(3):  # :59-74
        g, p = grad[c], prior[c]
        if prec == "ref":
            sums.append(_sum(g * (g - p), prec))
            sums.append(_sum(p * p, prec))
        else:
            gd, pd = g.astype(np.float64), p.astype(np.float64)
            sums.append(_sum(gd * (gd - pd), prec))
            sums.append(_sum(pd * pd, prec))
        prior[c] = g
    if cdf == 0:  # :80-84
        for c in range(3):
            if abs(sums[2 * c + 1]) > 0.0:
                beta[c] = (f32(sums[2 * c]) / f32(sums[2 * c + 1])) if prec == "ref" else sums[2 * c] / sums[2 * c + 1]
    if beta[0] < 0:
        beta[0] = 0.0
    if beta[0] > 0.5:
        beta[0] = 0.5
    for c in range(3):  # :94-107
        if prec == "ref":
            d = (prior[3 + c] * f32(beta[c]) + grad[c]).astype(np.float32)
        else:
            d = (prior[3 + c].astype(np.float64) * beta[c] + grad[c].astype(np.float64)).astype(np.float32)
        grad[c] = d
        prior[3 + c] = d
    return np.array([float(b) for b in beta], np.float64)


class LBFGSState:
    """bfgsmod (s), bfgsgrad (y) [bfgsnum][numpar*n], bfgsscale [bfgsnum];
    row w-1 is the reference's row w. float32 for "ref", float64 for "fp64"."""

    def __init__(self, n, numpar, bfgsnum, prec="ref"):
        dt = np.float32 if prec == "ref" else np.float64
        self.prec, self.numpar, self.B, self.n = prec, numpar, bfgsnum, n
        self.s = np.zeros((bfgsnum, numpar * n), dt)
        self.y = np.zeros((bfgsnum, numpar * n), dt)
        self.scale = np.zeros(bfgsnum, dt)


def _slot(v, B):
    w = v % B
    return B if w == 0 else w


def lbfgs_savegrad(st: LBFGSState, grad):
    """lbfgs_save.c:25-56: row 1 of bfgsgrad = the gradient (vp[, vs])."""
    st.y[0] = grad[: st.numpar].reshape(-1)


def lbfgs(st: LBFGSState, grad, it_group):
    """lbfgs.c:26-181 for it_group >= 2; grad[0:numpar] replaced by the direction."""
    B, prec = st.B, st.prec
    g = grad[: st.numpar].reshape(-1)
    m = max(it_group - B, 1)
    w = _slot(it_group - 1, B) - 1
    if prec == "ref":
        st.y[w] = st.y[w] + (-g)
        q = g.astype(np.float32).copy()
        d0 = _sum(st.y[w] * st.s[w], prec)
        d1 = _sum(st.y[w] * st.y[w], prec)
        st.scale[w] = f32(1) / d0
        h0 = f32(d0 / d1)
    else:
        st.y[w] = st.y[w] - g.astype(np.float64)
        q = g.astype(np.float64)
        d0 = _sum(st.y[w] * st.s[w], prec)
        d1 = _sum(st.y[w] * st.y[w], prec)
        st.scale[w] = 1.0 / d0
        h0 = d0 / d1
    alpha = {}
    for v in range(it_group - 1, m - 1, -1):  # :96-115
        w = _slot(v, B) - 1
        if prec == "ref":
            alpha[w] = _sum(st.scale[w] * st.s[w] * q, prec)
            q = (q + (-alpha[w]) * st.y[w]).astype(np.float32)
        else:
            alpha[w] = st.scale[w] * _sum(st.s[w] * q, prec)
            q = q + (-alpha[w]) * st.y[w]
    q = (q * h0).astype(q.dtype)  # :118-121
    for v in range(m, it_group):  # :137-159
        w = _slot(v, B) - 1
        if prec == "ref":
            b = _sum(st.scale[w] * st.y[w] * q, prec)
            q = (q + st.s[w] * f32(alpha[w] - b)).astype(np.float32)
        else:
            coef = alpha[w] - st.scale[w] * _sum(st.y[w] * q, prec)
            q = q + coef * st.s[w]
    w = _slot(it_group, B) - 1  # :161-181
    st.y[w] = g
    grad[: st.numpar] = q.astype(np.float32).reshape(grad[: st.numpar].shape)


def modelupdate(grad, rho, pi, u, step, weight, vp0, vs0, rho0, lbfgs_on=False, st: LBFGSState | None = None,
                it_group=1):
    """modelupdate.c:26-160 on grad [3][ny][nx][nz] and ghosted models (float32,
    in place). The model arithmetic is the reference's in both precisions; with
    L-BFGS the model difference goes to st.s (float32 "ref", float64 "fp64")."""
    step, s1, s2, s3 = f32(step), f32(weight[0]), f32(weight[1]), f32(weight[2])
    vp0, vs0, rho0 = f32(vp0), f32(vs0), f32(rho0)
    if not lbfgs_on:  # :82-117
        mx = [f32(np.abs(grad[c]).max()) for c in range(3)]
        if mx[2] == 0.0:
            mx[2] = f32(1.0)
        if mx[0] > 0.0 and mx[1] > 0.0:
            for c in range(3):
                grad[c] = (grad[c] / mx[c]).astype(np.float32)
    R, P, U = rho[1:-1, 1:-1, 1:-1], pi[1:-1, 1:-1, 1:-1], u[1:-1, 1:-1, 1:-1]
    vp_old = np.sqrt((P / R).astype(np.float32).astype(np.float64))
    vs_old = np.sqrt((U / R).astype(np.float32).astype(np.float64))
    vpnew = (vp_old + (step * s1 * grad[0] * vp0).astype(np.float32).astype(np.float64)).astype(np.float32)
    vsnew = (vs_old + (step * s2 * grad[1] * vs0).astype(np.float32).astype(np.float64)).astype(np.float32)
    rhonew = (R + (s3 * step * grad[2] * rho0).astype(np.float32)).astype(np.float32)
    if lbfgs_on:
        n = vpnew.size
        w = _slot(it_group, st.B) - 1
        st.s[w, :n] = ((vpnew.astype(np.float64) - vp_old) / np.float64(vp0)).ravel()
        if st.numpar > 1:
            st.s[w, n:] = ((vsnew.astype(np.float64) - vs_old) / np.float64(vs0)).ravel()
    U[...] = rhonew * vsnew * vsnew
    P[...] = rhonew * vpnew * vpnew
    R[...] = rhonew


def steplength(L2, step, lbfgs_on, it_group, teststep, prec="ref"):
    """steplength.c:26-91. L2[4], step[5] updated in place; returns (a, b, c).
    "ref": float variables, with the double constants 0.1, 2.5, 0.2 of the C
    (comparisons against them in double); "fp64": everything in double."""
    T = f32 if prec == "ref" else float
    dbl = float
    s0, s1, s2 = T(step[0]), T(step[1]), T(step[2])
    l0, l1, l2 = T(L2[0]), T(L2[1]), T(L2[2])
    a = ((s0 - s1) * (l0 - l2) - (s0 - s2) * (l0 - l1)) / (s0 * s2 * (s0 - s2) + s0 * s1 * (s1 - s0) + s1 * s2 * (s2 - s1))
    b = (l0 - l1) / (s0 - s1)
    b = b - a * (s0 + s1)
    c = l0 - a * s0 * s0 - b * s0
    s3 = T(0.0)
    s4 = T(step[4])
    if a > 0:
        s3 = -b / (T(2) * a)
    if a < 0:
        if l0 < l1 and l0 < l2:
            s3 = T(0.1 * dbl(s1))
        if l1 < l0 and l1 < l2:
            s3 = s1
        if l2 < l0 and l2 < l1:
            s3 = s2
    if dbl(s3) > 2.5 * dbl(s4):
        s3 = T(2.5 * dbl(s4))
    if lbfgs_on and it_group > 1 and dbl(s3) > 1.0:
        s3 = T(1.0)
    if s3 <= 0:
        s3 = T(0.1 * dbl(s1))
    if dbl(s3) < 0.1 * dbl(s1):
        s3 = T(0.1 * dbl(s1))
    L2[3] = a * s3 * s3 + b * s3 + c
    s4 = s3 / T(2)
    tst = dbl(T(teststep))
    if dbl(s4) < 0.2 * tst:
        s4 = T(0.2 * tst)
    if dbl(s4) > tst:
        s4 = T(teststep)
    if lbfgs_on and it_group > 1:
        s4 = T(0.5)
    step[3] = s3
    step[4] = s4
    return a, b, c


class RefOptim:
    """The reference's own optimiser functions (oracle/_ref/libifos_ref.so,
    driven by oracle/ref_optim.c) on flat float32 arrays, updated in place."""

    def __init__(self):
        import ctypes as C

        from pyoracle import REF_LIB

        self.C = C
        self.lib = C.CDLL(REF_LIB)
        for name in ("ifo_ref_conjugate", "ifo_ref_lbfgs", "ifo_ref_steplength", "ifo_ref_modelupdate"):
            getattr(self.lib, name).restype = C.c_int

    def _p(self, a):
        if a is None:
            return None
        assert a.dtype == np.float32 and a.flags.c_contiguous
        return a.ctypes.data_as(self.C.c_void_p)

    def conjugate(self, grad, prior, cdf):
        _, ny, nx, nz = grad.shape
        beta = np.zeros(3, np.float32)
        assert self.lib.ifo_ref_conjugate(nx, ny, nz, self._p(grad), self._p(prior), cdf, self._p(beta)) == 0
        return beta

    def lbfgs(self, grad, st: LBFGSState, it_group):
        """it_group == 1: lbfgs_savegrad; else lbfgs (src/ifos3d.c:1007-1014)."""
        _, ny, nx, nz = grad.shape
        assert self.lib.ifo_ref_lbfgs(nx, ny, nz, st.numpar, st.B, self._p(grad), self._p(st.scale), self._p(st.s),
                                      self._p(st.y), it_group) == 0

    def steplength(self, L2, step, lbfgs_on, it_group, teststep):
        C = self.C
        assert self.lib.ifo_ref_steplength(self._p(L2), self._p(step), int(lbfgs_on), it_group,
                                           C.c_float(teststep)) == 0

    def modelupdate(self, grad, rho, pi, u, step, weight, vp0, vs0, rho0, lbfgs_on=False, st=None, it_group=1):
        C = self.C
        _, ny, nx, nz = grad.shape
        w = np.ascontiguousarray(weight, np.float32)
        numpar, B = (st.numpar, st.B) if st is not None else (1, 0)
        assert self.lib.ifo_ref_modelupdate(nx, ny, nz, self._p(grad), self._p(rho), self._p(pi), self._p(u),
                                            self._p(st.s) if (st is not None and lbfgs_on) else None, numpar, B,
                                            C.c_float(step), self._p(w), C.c_float(vp0), C.c_float(vs0),
                                            C.c_float(rho0), int(lbfgs_on), it_group) == 0
