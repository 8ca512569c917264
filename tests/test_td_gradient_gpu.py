"""Time-domain gradient kernels with checkpointing (ifosb_gradient_td).

1. Against the DFT gradient of gradient_F (src/gradient_F.c:30-171) fed by
   discfourier (src/disc_fourier.c:30-60). discfourier phases the forward step n
   at t = n DT and the adjoint step m at TIME - m DT, so with the DFT frequencies
   f_l = l / (N DT), N = 2 NT, gradient_F's rho term summed over l = 0..N-1 is,
   by Parseval,
       sum_l gradrho_l = N DT^2 sum_{n + m = TIME/DT} v_f(n) . v_b(m)
   (every other lag n + m - TIME/DT lies strictly between -N and N, where the sum
   of cos(2 pi l d / N) over l vanishes). The terms l and N - l are equal, l = 0
   is the product of the two time sums (the engine's dc kernel) and l = N/2 the
   Nyquist term, so the time-domain rho kernel must equal
       (dc + 2 sum_{l=1}^{NT-1} gradrho_l + gradrho_NT) / (N DT^2)
   up to the float rounding of the DFT phases and sums.
2. The lambda and mu kernels correlate running sums of v where gradient_F
   divides by omega^2, so no such identity holds for them. All four kernels are
   checked against a restatement of their definitions over the oracle's
   wavefields instead: the oracle run for NT' = 1..NT steps gives the state after
   each step, and the restatement, in the engine's arithmetic order, must
   reproduce the kernels to FP64 rounding.
3. The checkpoint interval changes no bit of any kernel.
Elastic and viscoelastic (L = 3: the checkpoints carry the memory variables
with the rest of the state)."""
import numpy as np
import pytest

import ifosb
from helpers import engine_for, ifo_params, rel_l2
from ifosb import synth

pytestmark = pytest.mark.gpu


def interior(a, p):
    """[..., NY+5, NX+4, NZ+4] host fields -> [..., NY, NX, NZ] (cells j,i,k = 1..N)."""
    return a[..., 3:p.ny + 3, 2:p.nx + 2, 2:p.nz + 2]


def dft_rho_sum(e, shots, obs, freqs, p):
    """gradient_F's rho term over `freqs` (calls of up to 16 frequencies), summed
    over frequencies and shots in float64 from the engine's DFT fields."""
    rho_sum = np.zeros((p.ny, p.nx, p.nz), np.float64)
    for c0 in range(0, len(freqs), 16):
        e.set_frequencies(freqs[c0:c0 + 16], 1)
        e.forward(shots)
        e.residual(obs)
        e.adjoint()
        for s in range(len(shots)):
            ff = interior(e.get_dft(s), p).astype(np.float64)
            bb = interior(e.get_dft(s, back=True), p).astype(np.float64)
            rho_sum += (ff * bb).sum(axis=(0, 1))  # Re.Re + Im.Im over vx, vy, vz and the frequencies
    return rho_sum


@pytest.mark.parametrize("nmech", [0, 3])
def test_time_domain_rho_kernel_is_the_dense_dft_sum(nmech):
    c = synth.small_case(nx=22, ny=20, nz=18, nt=40, fw=4, nmech=nmech, nshots=2, seed=11, free_surf=1)
    p = c["params"]
    NT = p.nt
    assert round(float(p.time) / float(p.dt)) == NT - 1  # TIME = (NT-1) DT
    e, m, cp, shots = engine_for(c, max_shots=2, nf=16)
    syn = e.forward(shots)
    obs = (0.7 * np.roll(syn, 4, axis=-1)).astype(np.float32)  # a residual with structure
    dt = np.float64(np.float32(p.dt))
    N = 2 * NT
    freqs = (np.arange(1, NT + 1) / (N * dt)).astype(np.float32)
    rho_a = dft_rho_sum(e, shots, obs, freqs[:-1], p)  # l = 1 .. NT-1
    rho_n = dft_rho_sum(e, shots, obs, freqs[-1:], p)  # l = NT (Nyquist)
    e.set_frequencies(freqs[:1], 1)
    e.forward(shots)
    e.residual(obs)
    k1 = e.gradient_td(1)
    k7 = e.gradient_td(7)
    kall = e.gradient_td(10 ** 6)  # one segment: the whole forward history held
    for k in (k7, kall):
        assert np.array_equal(k1, k)  # checkpointing changes no bit
    assert np.isfinite(k1).all() and np.abs(k1[0]).max() > 0
    lhs = N * dt * dt * k1[0]
    rhs = k1[3] + 2.0 * rho_a + rho_n
    err = rel_l2(lhs, rhs)
    print(f"rho Parseval rel-L2 {err:.3e}")
    assert err < 1e-5
    e.close()


def stencils(X, Y, Z, p, b1, b2):
    """gradient_F's nine derivative stencils (gradient_F.c:80-88) at the interior
    cells of padded [NY+5][NX+4][NZ+4] fields, in float32 as the engine forms them."""
    dx, dy, dz = np.float32(p.dx), np.float32(p.dy), np.float32(p.dz)

    def sh(A, dj=0, di=0, dk=0):
        return A[3 + dj:p.ny + 3 + dj, 2 + di:p.nx + 2 + di, 2 + dk:p.nz + 2 + dk]

    return [
        (b1 * (sh(X) - sh(X, di=-1)) + b2 * (sh(X, di=1) - sh(X, di=-2))) / dx,
        (b1 * (sh(X, dj=1) - sh(X)) + b2 * (sh(X, dj=2) - sh(X, dj=-1))) / dy,
        (b1 * (sh(X, dk=1) - sh(X)) + b2 * (sh(X, dk=2) - sh(X, dk=-1))) / dz,
        (b1 * (sh(Y, di=1) - sh(Y)) + b2 * (sh(Y, di=2) - sh(Y, di=-1))) / dx,
        (b1 * (sh(Y) - sh(Y, dj=-1)) + b2 * (sh(Y, dj=1) - sh(Y, dj=-2))) / dy,
        (b1 * (sh(Y, dk=1) - sh(Y)) + b2 * (sh(Y, dk=2) - sh(Y, dk=-1))) / dz,
        (b1 * (sh(Z, di=1) - sh(Z)) + b2 * (sh(Z, di=2) - sh(Z, di=-1))) / dx,
        (b1 * (sh(Z, dj=1) - sh(Z)) + b2 * (sh(Z, dj=2) - sh(Z, dj=-1))) / dy,
        (b1 * (sh(Z) - sh(Z, dk=-1)) + b2 * (sh(Z, dk=1) - sh(Z, dk=-2))) / dz,
    ]


def running_sums(vs, dt):
    """U(n) = U(n-1) + v(n) DT in float32, n = 1..len(vs)."""
    u, out = np.zeros_like(vs[0]), []
    for v in vs:
        u = u + v * dt
        out.append(u)
    return out


def dot3(a, b, p):
    return (interior(a[0], p).astype(np.float64) * interior(b[0], p) +
            interior(a[1], p).astype(np.float64) * interior(b[1], p) +
            interior(a[2], p).astype(np.float64) * interior(b[2], p))


@pytest.mark.parametrize("free_surf,interval,nmech", [(1, 3, 0), (0, 5, 0), (1, 4, 3)])
def test_time_domain_kernels_match_oracle_restatement(oracle, free_surf, interval, nmech):
    c = synth.small_case(nx=16, ny=15, nz=14, nt=18, fw=3, nmech=nmech, nshots=1, seed=23 + free_surf,
                         free_surf=free_surf, stype=3)  # a y-force: its amplitudes do not depend on NT
    p = c["params"]
    NT, P = p.nt, p.nt - 1
    e, m, cp, shots = engine_for(c, max_shots=1, nf=1)
    syn = e.forward(shots)
    obs = (0.6 * np.roll(syn, 3, axis=-1)).astype(np.float32)
    e.residual(obs)
    k = e.gradient_td(interval)
    # the oracle: forward and adjoint states after each step n = 1..NT
    sp, sig = shots[0]
    f = oracle.forward(ifo_params(c), m, cp, sp, sig, c["recpos"])
    diff, _ = oracle.residual(ifo_params(c), obs[0], f["sections"])
    vf, vb = [], []
    for n in range(1, NT + 1):
        q = ifo_params(c)
        q.nt = n
        vf.append(oracle.forward(q, m, cp, sp, np.ascontiguousarray(sig[:, :n]), c["recpos"],
                                 want_state=True)["state"][:3])
        vb.append(oracle.adjoint(q, m, cp, c["recpos"], np.ascontiguousarray(diff[..., :n]), c["finv"][:1],
                                 want_state=True)["state"][:3])
    dt = np.float32(p.dt)
    uf, ub = running_sums(vf, dt), running_sums(vb, dt)
    b1, b2 = ((np.float32(1.1382), np.float32(-0.046414)) if p.fdcoeff == 2
              else (np.float32(9.0 / 8.0), np.float32(-1.0 / 24.0)))
    want = np.zeros_like(k)

    def D(d, q):
        return d[q].astype(np.float64)

    for n in range(P - 1, 0, -1):  # the engine's order: adjoint steps m = P - n ascending
        mb = P - n
        want[0] += dot3(vf[n - 1], vb[mb - 1], p)
        fu = stencils(*uf[n - 1], p, b1, b2)
        bu = stencils(*ub[mb - 1], p, b1, b2)
        want[1] += (D(fu, 0) + fu[4] + fu[8]) * (D(bu, 0) + bu[4] + bu[8])
        want[2] += (2.0 * (D(fu, 0) * bu[0] + D(fu, 4) * bu[4] + D(fu, 8) * bu[8]) +
                    (D(fu, 1) + fu[3]) * (D(bu, 1) + bu[3]) + (D(fu, 2) + fu[6]) * (D(bu, 2) + bu[6]) +
                    (D(fu, 5) + fu[7]) * (D(bu, 5) + bu[7]))
    want[3] = dot3(uf[-1], ub[-1], p)
    assert all(np.abs(want[q]).max() > 0 for q in range(4))
    for q in range(4):
        assert rel_l2(k[q], want[q]) < 1e-12, q
    e.close()


def test_time_domain_preconditions():
    c = synth.small_case(nx=20, ny=18, nz=20, nt=30, fw=4, nmech=0, nshots=1, seed=3)
    e, m, cp, shots = engine_for(c)
    with pytest.raises(ifosb.IfosbError):
        e.gradient_td(5)  # no forward yet
    syn = e.forward(shots)
    with pytest.raises(ifosb.IfosbError):
        e.gradient_td(5)  # no residual yet
    e.residual(syn * 0.5)
    with pytest.raises(ifosb.IfosbError):
        e.gradient_td(0)  # interval below 1
    k = e.gradient_td(4)
    assert np.abs(k[0]).max() > 0
    e.close()


def test_time_domain_partial_batch():
    """A batch smaller than the engine's max_shots (the recomputation's tensor
    maps then cover fewer shots than the engine's own) gives the same kernels."""
    c = synth.small_case(nx=20, ny=22, nz=18, nt=30, fw=4, nmech=0, nshots=2, seed=41, free_surf=1)
    out = []
    for cap in (2, 3):
        e, m, cp, shots = engine_for(c, max_shots=cap, nf=1)
        syn = e.forward(shots)
        e.residual((0.5 * np.roll(syn, 2, axis=-1)).astype(np.float32))
        out.append(e.gradient_td(4))
        e.close()
    assert np.abs(out[0][0]).max() > 0
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("nmech", [0, 3])
def test_forward_checkpoints_and_graphs_change_no_bit(nmech):
    """The checkpoints a forward keeps itself (ifosb_set_td_checkpoints), the
    checkpoints an earlier call left, the captured graph and its replay, and
    plain launches all give the kernels of a plain call bit for bit; arming the
    forward changes no trace."""
    c = synth.small_case(nx=20, ny=22, nz=18, nt=34, fw=4, nmech=nmech, nshots=2, seed=7, free_surf=1)
    e, m, cp, shots = engine_for(c, max_shots=2, nf=1)
    syn = e.forward(shots)
    obs = (0.5 * np.roll(syn, 2, axis=-1)).astype(np.float32)

    def fresh(interval, arm):
        e.set_td_checkpoints(arm)
        s = e.forward(shots)
        e.residual(obs)
        return s, e.gradient_td(interval)

    e.set_launch_mode(1)
    s0, k0 = fresh(4, 0)  # plain launches, the forward run again
    e.set_launch_mode(0)
    s1, k1 = fresh(4, 0)  # graph capture
    c1 = e.graph_captures
    k1b = e.gradient_td(4)  # the checkpoints of the call before: no re-run
    s2, k2 = fresh(4, 4)  # the forward's own checkpoints
    k2b = e.gradient_td(4)
    s3, k3 = fresh(4, 5)  # armed at another interval: run again
    _, k4 = fresh(4, 0)  # replayed graph
    assert np.abs(k0[0]).max() > 0
    for k in (k1, k1b, k2, k2b, k3, k4):
        assert np.array_equal(k, k0)
    for s in (s1, s2, s3):
        assert np.array_equal(s, s0)
    assert e.graph_captures > c1  # the armed forward and the no-re-run loops are graphs of their own
    e.close()
