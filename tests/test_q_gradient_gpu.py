"""Viscoelastic Q gradient (ifosb_get_gradient_q): the gradients with respect to
the model's taup and taus that ifosb_gradient accumulates next to gradient_F's.

The reference has no Q gradient. Its memory-variable update
(src/update_s_ssg.c:108-122) makes a modulus M act, in discfourier's frequency
domain (e^{+i w t}), as M (1 + tau Phi(w)) with Phi = sum_l s t_l / (1 + s t_l),
s = -i w, t_l = DT / eta_l. With gradient_F's lambda and mu correlations taken
complex (C = F conj(B); gradlam and gradmu are their real parts):
    d/dtaup = pi sum_f Re[Phi C_lambda],   d/dtaus = u sum_f Re[Phi (C_mu - 2 C_lambda)].

1. The kernel against a numpy restatement of that formula over the engine's own
   DFT fields, in the kernel's arithmetic order.
2. Against centred finite differences of the FP64 misfit along 12 seeded random
   directions of taup or taus (interior, away from the CPML frame and the free
   surface), with a dense frequency grid (48 frequencies at 1/(NT DT) spacing).
   gradient_F's sign makes the vectors anti-parallel. Measured: cos = -0.981
   over all 12 (taup alone -0.995, taus alone -0.949), the same at eps = 0.03,
   0.1 and 0.2 (the misfit is linear in tau over that range), against cos = -0.93
   without the imaginary part of Phi C and -0.55 with its sign flipped. The
   ratio <g, d> / FD is about -33 on most directions: the reference's frequency
   sum carries no 2 df factor.
"""
import math

import numpy as np
import pytest

import ifosb
from ifosb import synth

pytestmark = pytest.mark.gpu


def stencils(X, Y, Z, ny, nx, nz, b1, b2, dx):
    """gradient_F's nine derivative stencils (gradient_F.c:80-88) at the interior
    of padded [NY+5][NX+4][NZ+4] fields, in float32 as the engine forms them."""

    def sh(A, dj=0, di=0, dk=0):
        return A[3 + dj:ny + 3 + dj, 2 + di:nx + 2 + di, 2 + dk:nz + 2 + dk]

    return [
        (b1 * (sh(X) - sh(X, di=-1)) + b2 * (sh(X, di=1) - sh(X, di=-2))) / dx,
        (b1 * (sh(X, dj=1) - sh(X)) + b2 * (sh(X, dj=2) - sh(X, dj=-1))) / dx,
        (b1 * (sh(X, dk=1) - sh(X)) + b2 * (sh(X, dk=2) - sh(X, dk=-1))) / dx,
        (b1 * (sh(Y, di=1) - sh(Y)) + b2 * (sh(Y, di=2) - sh(Y, di=-1))) / dx,
        (b1 * (sh(Y) - sh(Y, dj=-1)) + b2 * (sh(Y, dj=1) - sh(Y, dj=-2))) / dx,
        (b1 * (sh(Y, dk=1) - sh(Y)) + b2 * (sh(Y, dk=2) - sh(Y, dk=-1))) / dx,
        (b1 * (sh(Z, di=1) - sh(Z)) + b2 * (sh(Z, di=2) - sh(Z, di=-1))) / dx,
        (b1 * (sh(Z, dj=1) - sh(Z)) + b2 * (sh(Z, dj=2) - sh(Z, dj=-1))) / dx,
        (b1 * (sh(Z) - sh(Z, dk=-1)) + b2 * (sh(Z, dk=1) - sh(Z, dk=-2))) / dx,
    ]


def q_restatement(F, B, finv, eta, dt, pi, u, gq, ny, nx, nz):
    """Adds one shot's taup / taus gradient to gq [2][NY][NX][NZ] (float64)."""
    b1, b2, one = np.float32(1.1382), np.float32(-0.046414), np.float32(1.0)
    pi64, u64 = pi.astype(np.float64), u.astype(np.float64)
    for l, f in enumerate(finv):
        fdummy = one / np.float32(2.0 * 2.0 * float(f) * float(f) * math.pi * math.pi)
        w = 2.0 * math.pi * float(f)
        rphi = iphi = 0.0
        for et in eta:
            wt = w * (float(dt) / float(et))
            rphi += wt * wt / (1.0 + wt * wt)
            iphi -= wt / (1.0 + wt * wt)
        fv = stencils(F[0, l], F[1, l], F[2, l], ny, nx, nz, b1, b2, one)
        fi = stencils(F[3, l], F[4, l], F[5, l], ny, nx, nz, b1, b2, one)
        bv = stencils(B[0, l], B[1, l], B[2, l], ny, nx, nz, b1, b2, one)
        bi = stencils(B[3, l], B[4, l], B[5, l], ny, nx, nz, b1, b2, one)
        D = lambda a, q: a[q].astype(np.float64)  # noqa: E731
        fd = -float(fdummy)
        dfr, dfi = D(fv, 0) + fv[4] + fv[8], D(fi, 0) + fi[4] + fi[8]
        dbr, dbi = D(bv, 0) + bv[4] + bv[8], D(bi, 0) + bi[4] + bi[8]
        rl, il = fd * (dfr * dbr + dfi * dbi), fd * (dfi * dbr - dfr * dbi)
        rm = np.zeros_like(rl)
        im = np.zeros_like(rl)
        for q in (0, 4, 8):
            rm = rm + 2.0 * (D(fv, q) * bv[q] + D(fi, q) * bi[q])
            im = im + 2.0 * (D(fi, q) * bv[q] - D(fv, q) * bi[q])
        for a_, b_ in ((1, 3), (2, 6), (5, 7)):
            fr, fim = D(fv, a_) + fv[b_], D(fi, a_) + fi[b_]
            br, bim = D(bv, a_) + bv[b_], D(bi, a_) + bi[b_]
            rm = rm + (fr * br + fim * bim)
            im = im + (fim * br - fr * bim)
        rm, im = rm * fd, im * fd
        gq[0] += pi64 * (rphi * rl - iphi * il)
        gq[1] += u64 * (rphi * (rm - 2.0 * rl) - iphi * (im - 2.0 * il))


def test_q_gradient_matches_restatement():
    c = synth.small_case(nx=30, ny=28, nz=26, nt=150, fw=5, nmech=3, nshots=2, seed=17, free_surf=1,
                         finv=(300.0, 500.0, 800.0))
    p = c["params"]
    m, cp, shots = synth.build_inputs(c)
    e = ifosb.Engine(p, max_shots=2, max_nf=3)
    e.set_cpml(cp)
    e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
    e.set_receivers(c["recpos"])
    e.set_frequencies(c["finv"], 1)
    syn = e.forward(shots)
    e.zero_gradient()
    e.shot_gradient(shots, (0.8 * np.roll(syn, 5, axis=-1)).astype(np.float32))
    gq = e.get_gradient_q()
    want = np.zeros_like(gq)
    for s in range(2):
        q_restatement(e.get_dft(s), e.get_dft(s, back=True), c["finv"], m["eta"], p.dt, m["pi"], m["u"], want,
                      p.ny, p.nx, p.nz)
    assert np.abs(want).max() > 0
    for q in range(2):
        assert np.linalg.norm(gq[q] - want[q]) / np.linalg.norm(want[q]) < 1e-12, q
    # zero_gradient clears it; an elastic engine has none
    e.zero_gradient()
    assert not e.get_gradient_q().any()
    e.close()
    ce = synth.small_case(nx=20, ny=18, nz=20, nt=30, fw=4, nmech=0, nshots=1, seed=3)
    me, cpe, _ = synth.build_inputs(ce)
    ee = ifosb.Engine(ce["params"], max_shots=1, max_nf=1)
    with pytest.raises(ifosb.IfosbError):
        ee.get_gradient_q()
    ee.close()


NX, NY, NZ, FW, NT, FC, DT = 64, 64, 56, 10, 600, 200.0, 1e-4


def test_q_gradient_against_centred_finite_differences():
    L = 3
    rng = np.random.default_rng(7)
    p = ifosb.make_params(NX, NY, NZ, dh=1.0, dt=DT, nt=NT, fdcoeff=2, free_surf=1, fw=FW, nmech=L)
    tau, fl = synth.q_tau_fit(50.0, 20.0, 200.0, L)
    depth = np.linspace(2000, 3500, NY, dtype=np.float32)[:, None, None]
    bg = np.broadcast_to(depth, (NY, NX, NZ)).astype(np.float32)
    pert = 0.03 * synth._gauss_field((NY, NX, NZ), 6.0, rng)
    vpt = (bg * (1 + pert)).astype(np.float32)
    true = (vpt, (vpt / np.float32(math.sqrt(3))).astype(np.float32),
            ((1700 + 0.2 * bg) * (1 + pert)).astype(np.float32))
    start = (bg.copy(), (bg / np.float32(math.sqrt(3))).astype(np.float32), (1700 + 0.2 * bg).astype(np.float32))
    shots = [(sp, ifosb.wavelet(p, 4, sp)) for sp in (synth._src(x, 8, NZ // 2, FC) for x in (20, 44))]
    e = ifosb.Engine(p, max_shots=2, max_nf=16)
    e.set_cpml(ifosb.cpml_coeff(p, 3500.0, FC))
    e.set_receivers(synth._grid_receivers(NX, NZ, 8, 1, 14))
    mt = ifosb.moduli(p, *true, tau=tau, fl=fl)
    ms = ifosb.moduli(p, *start, tau=tau, fl=fl)

    def set_model(m, taup, taus):
        e.set_model(m["rho"], m["pi"], m["u"], taus, taup, m["eta"])

    set_model(mt, mt["taup"], mt["taus"])
    e.set_frequencies(None, 1)
    obs = e.forward(shots)

    def misfit(taup, taus):
        set_model(ms, taup, taus)
        e.set_frequencies(None, 1)
        e.forward(shots)
        return float(np.sum(e.residual(obs)))

    set_model(ms, ms["taup"], ms["taus"])
    e.zero_gradient()
    freqs = np.arange(1, 49) / (NT * DT)
    for c0 in range(0, 48, 16):  # the engine's gradients accumulate over calls
        e.set_frequencies(np.array(freqs[c0:c0 + 16], np.float32), 1)
        e.shot_gradient(shots, obs)
    gq = e.get_gradient_q()
    assert np.all(np.isfinite(gq))

    jj, ii, kk = np.meshgrid(np.arange(1, NY + 1), np.arange(1, NX + 1), np.arange(1, NZ + 1), indexing="ij")

    def ramp(x, lo, hi):
        return np.clip(np.minimum(x - lo, hi - x) / 4.0, 0, 1)

    taper = (ramp(jj, 6, NY - FW - 2) * ramp(ii, FW + 2, NX - FW - 2) * ramp(kk, FW + 2, NZ - FW - 2)).astype(np.float32)
    eps = 0.1
    fd, dots = [], []
    for q in range(12):
        which = q % 2  # taup, taus in turn
        d = (ms["taup"] * taper * synth._gauss_field((NY, NX, NZ), 4.0, rng) * 0.5).astype(np.float32)
        up, dn = [ms["taup"], ms["taus"]], [ms["taup"], ms["taus"]]
        up[which] = (up[which] + eps * d).astype(np.float32)
        dn[which] = (dn[which] - eps * d).astype(np.float32)
        dr = (up[which].astype(np.float64) - dn[which].astype(np.float64)) / (2 * eps)  # after rounding
        fd.append((misfit(*up) - misfit(*dn)) / (2 * eps))
        dots.append(float(np.sum(gq[which] * dr)))
    fd, dots = np.array(fd), np.array(dots)

    def cos(a, b):
        return float(a @ b / np.linalg.norm(a) / np.linalg.norm(b))

    c_all, c_p, c_s = cos(fd, dots), cos(fd[0::2], dots[0::2]), cos(fd[1::2], dots[1::2])
    print(f"cos all {c_all:.4f} taup {c_p:.4f} taus {c_s:.4f}; ratio {np.round(dots / fd, 2)}")
    # measured -0.981 / -0.995 / -0.949 (deterministic kernels, seeded inputs)
    assert c_all < -0.96 and c_p < -0.98 and c_s < -0.92
    # d/dQ for tau proportional to 1/Q is the chain rule on the same arrays
    qg = ifosb.q_gradient(gq, ms["taup"], ms["taus"], 50.0)
    assert np.allclose(qg, -(ms["taup"] * gq[0] + ms["taus"] * gq[1]) / 50.0)
    e.close()
