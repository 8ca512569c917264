"""Physical check of the L=3 viscoelastic model: the attenuation a P wave
measures between two receivers gives the Q the relaxation times were fitted to.

The viscoelastic forward-modelling configuration asks for Q = 50 over 20-200 Hz
with three relaxation mechanisms (the tau method: one tau for all mechanisms,
relaxation frequencies log-spaced over the band; ifosb.synth.q_tau_fit). The
memory-variable update (src/update_s_ssg.c:108-140, generalised to L
mechanisms) makes every modulus act as M(w) = M_R (1 + tau sum_l i w t_l /
(1 + i w t_l)), t_l = 1 / (2 pi FL_l), so a wave of frequency f loses
exp(-pi f d / (c Q(f))) over a distance d, Q(f) = Re M / Im M.

Measured: an explosive source in a homogeneous medium (pure P radiation, no
free surface), two receivers on the x axis at 60 and 220 m. The same run with
the elastic update on the same relaxed moduli gives the spreading and source
spectrum; the log ratio of the two runs' amplitude spectra, differenced between
the receivers, is -pi f (r2 - r1) / (c(f) Q(f)), c(f) the model's phase
velocity. Each P pulse is cut out by a window that is flat over the pulse of
both runs (the viscoelastic pulse arrives earlier: a taper over the pulse would
weigh the two runs differently). Asserted over 30-200 Hz (the 100 Hz sin^3
wavelet's band):
- Q measured at each frequency within 5 % of the model's exact Q(f);
- the band's median Q within 5 % of the fitted 50.
"""
import math

import numpy as np
import pytest

import ifosb
from ifosb import synth

pytestmark = pytest.mark.gpu

NX, NY, NZ, FW, DT, NT, FC = 262, 64, 64, 10, 1e-4, 1000, 100.0
VP, VS, RHO, QTARGET = 3500.0, 3500.0 / 1.8, 2200.0, 50.0
SRC_X, R1, R2 = 20, 60, 220


def _run(nmech, tau, fl):
    p = ifosb.make_params(NX, NY, NZ, dh=1.0, dt=DT, nt=NT, fdcoeff=2, free_surf=0, fw=FW, nmech=nmech)
    shape = (NY, NX, NZ)
    pv = ifosb.make_params(NX, NY, NZ, dh=1.0, dt=DT, nt=NT, fdcoeff=2, free_surf=0, fw=FW, nmech=3)
    m = ifosb.moduli(pv, np.full(shape, VP, np.float32).ravel(), np.full(shape, VS, np.float32).ravel(),
                     np.full(shape, RHO, np.float32).ravel(), tau=tau, fl=fl)  # relaxed moduli of the L=3 model
    e = ifosb.Engine(p, max_shots=1, max_nf=0)
    e.set_cpml(ifosb.cpml_coeff(p, VP, FC))
    if nmech:
        e.set_model(m["rho"].reshape(shape), m["pi"].reshape(shape), m["u"].reshape(shape),
                    m["taus"].reshape(shape), m["taup"].reshape(shape), m["eta"])
    else:
        e.set_model(m["rho"].reshape(shape), m["pi"].reshape(shape), m["u"].reshape(shape), None, None, None)
    rec = np.array([[SRC_X + R1, NY // 2, NZ // 2], [SRC_X + R2, NY // 2, NZ // 2]], np.int32)
    e.set_receivers(rec)
    e.set_frequencies(None, 1)
    sp = synth._src(SRC_X, NY // 2, NZ // 2, FC)
    sec = e.forward([(sp, ifosb.wavelet(p, 4, sp))])
    e.close()
    return sec[0, 0]  # vx (radial) at both receivers, [2][NT]


def _spectrum(trace, r):
    """FFT of the P pulse at distance r: flat from 6 ms before the nominal arrival
    r / VP to 30 ms after it, 6 ms cosine tapers on either side."""
    t = np.arange(NT) * DT
    a, b, tap = r / VP - 0.006, r / VP + 0.030, 0.006
    w = ((t >= a) & (t <= b)).astype(np.float64)
    up, dn = (t >= a - tap) & (t < a), (t > b) & (t <= b + tap)
    w[up] = 0.5 * (1 - np.cos(np.pi * (t[up] - (a - tap)) / tap))
    w[dn] = 0.5 * (1 + np.cos(np.pi * (t[dn] - b) / tap))
    n = 16384
    return np.abs(np.fft.rfft(trace.astype(np.float64) * w, n)), np.fft.rfftfreq(n, DT)


def _model(f, tau, fl):
    """Exact Q(f) and phase velocity c(f) of the L-mechanism update: M(w) = M_R (1 +
    tau sum_l i w t_l / (1 + i w t_l)), M_R the relaxed modulus of readmod (the
    velocity VP at w_s = 2 pi FL[1], src/readmod.c:53-61)."""
    tl = 1.0 / (2 * math.pi * np.asarray(fl, np.float64))
    ws = 2 * math.pi * float(fl[0])
    sump = float((ws * ws * tl * tl * tau / (1 + ws * ws * tl * tl)).sum())
    c_r = VP / math.sqrt(1 + sump)
    x = 2 * math.pi * f[:, None] * tl[None, :]
    m = 1 + tau * (1j * x / (1 + 1j * x)).sum(1)
    return m.real / m.imag, c_r / np.real(m ** -0.5)


def test_three_mechanisms_attenuate_at_the_fitted_q():
    tau, fl = synth.q_tau_fit(QTARGET, 20.0, 200.0, 3)
    v = _run(3, tau, fl)
    el = _run(0, tau, fl)
    (V1, f), (V2, _), (E1, _), (E2, _) = (_spectrum(v[0], R1), _spectrum(v[1], R2), _spectrum(el[0], R1),
                                          _spectrum(el[1], R2))
    band = (f >= 30.0) & (f <= 200.0)
    ratio = np.log(V2[band] / E2[band]) - np.log(V1[band] / E1[band])
    q_model, c = _model(f[band], tau, fl)
    q_meas = -math.pi * f[band] * (R2 - R1) / (c * ratio)
    rel = np.abs(q_meas / q_model - 1)
    print(f"tau={tau:.5f}; Q measured 30/60/120/200 Hz: "
          + ", ".join(f"{q_meas[np.argmin(abs(f[band] - x))]:.1f}" for x in (30, 60, 120, 200))
          + f"; model {q_model.min():.1f}-{q_model.max():.1f}; median {np.median(q_meas):.2f}; "
          f"max rel dev {rel.max():.3f}")
    assert np.all(ratio < 0)  # the viscoelastic wave loses energy against the elastic one
    assert rel.max() < 0.05
    assert abs(np.median(q_meas) / QTARGET - 1) < 0.05
