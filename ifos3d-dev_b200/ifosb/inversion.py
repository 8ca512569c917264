"""The reference driver's inversion iteration on the engine and the device optimiser.

One iteration of src/ifos3d.c:669-1148, in its order:
  constant_boundary (FREE_SURF) and the averaged model            :681-683
  frequency-stage bookkeeping: cdf = 1 on a stage's first iteration :690-701
  shot gradients: forward, residual, adjoint, gradient_F per shot   :712-975
  precon_grad, then lbfgs / lbfgs_savegrad or conjugate             :1005-1015
  two test steps: modelupdate on a copy, forwards of NSHOTS_STEP
  shots, misfits                                                   :1021-1129
  steplength (parabola), modelupdate of the model                   :1133-1138
With Settings.hess, the approximate Hessian of ifos3d.c:882-1002 is formed at
iteration 1 (or read, READ_HESS) and divides the raw gradient every iteration.
With Settings.grad_file / mod_out_file set, the gradient and model files of
:1000 (raw), :1006 (+1000, preconditioned), :1016 (+2000, search direction) and
:1141 (model after the update; iteration 0 at :547) are written in the
reference's format (ifosb.io).
The differences are the ones the engine makes everywhere: shots run in batches,
misfits are summed in FP64, and the optimiser's dot products and the step-length
parabola are FP64. Models are the ghosted [NY+2][NX+2][NZ+2] rho, pi, u arrays of
the reference; their ghost layers are refreshed by the engine (matcopy's wrap).
With L > 0 relaxation mechanisms (p.nmech, visco = (taus, taup, eta)) the
relaxation times stay fixed and the iteration updates the relaxed moduli through
modelupdate's vp, vs, rho exactly as the elastic one does, with the gradient of
the viscoelastic propagation (the reference cannot run this: its viscoelastic
stress calls are commented out, src/ifos3d.c:773/777, and L is 1 there).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import Engine, Optimizer, Params, steplength, wavelet
from . import io as fio
from . import stages as fstages


@dataclass
class Stage:
    finv: list                     # DFT frequencies of the stage (readinv)
    itmax: int                     # iterations of the stage (itpergroup[1])


@dataclass
class Settings:
    teststep: float = 0.02         # TESTSTEP
    weight: tuple = (1.0, 1.0, 1.0)  # WEIGHT[3]
    vp0: float = 3000.0            # VP0, VS0, RHO0
    vs0: float = 1732.0
    rho0: float = 2000.0
    damptype: int = 2              # DAMPTYPE
    lbfgs: bool = False            # LBFGS
    lbfgs_first_normalised: bool = False  # not in the reference: see Inversion.iterate
    exact_gradient: bool = False   # not in the reference: the exact discrete VJP instead of gradient_F
    exact_interval: int = 25       # its checkpoint interval (time steps)
    numpar: int = 1                # NUMPAR
    bfgsnum: int = 3               # BFGSNUM
    nshots_step: int = 1           # NSHOTS_STEP (shots of the step-length test forwards)
    tast: int = 100                # TAST (DFT sampling: ntast = 1 / (f_max TAST DT))
    max_batch: int = 4             # shots per engine launch
    grad_file: str | None = None   # GRAD_FILE: gradients written per iteration (outgrad)
    mod_out_file: str | None = None  # MOD_OUT_FILE: models written per iteration (outmod)
    ids: tuple = (1, 1, 1)         # IDX, IDY, IDZ of the merged model/gradient files
    filt: bool = False             # FILT = 1: low-pass source signals and observed data at each
                                   # stage's highest frequency (ifos3d.c:731, :840-855)
    hess: bool = False             # HESS: approximate Hessian at iteration 1, applied every iteration
    read_hess: bool = False        # READ_HESS: take it from hess_file instead (readhess)
    read_hess_at: tuple = (0.0, 1)  # (finv, iteration) in the names of the files read
    rec_hess: int = 1              # REC_HESS: Green's functions of the first ntr // rec_hess receivers
    water_hess: tuple = (0.0, 0.0, 0.0)  # WATER_HESS_VP, _VS, _RHO
    hess_file: str | None = None   # HESS_FILE
    hess_signal: object = None     # [NT] y-force of the Hessian wavefields; None = the reference's rows


@dataclass
class History:
    misfit: list = field(default_factory=list)   # misfit[0] of every iteration (FP64)
    step: list = field(default_factory=list)     # the accepted step[3]
    beta: list = field(default_factory=list)


def stages_from_workflow(path: str, nstages: int) -> list:
    """Stages of a workflow file (INV_FILE) read as readinv() reads them."""
    return [Stage(list(w.finv), w.itmax) for w in fstages.read_workflow(path, nstages)]


class Inversion:
    def __init__(self, p: Params, cpml, recpos, shots, obs, srcpos_m, rho, pi, u, stages, cfg: Settings,
                 visco=None):
        """visco: (taus, taup, eta) for p.nmech > 0 — [NY][NX][NZ] relaxation times per
        cell and the mechanisms' eta — kept fixed through the inversion."""
        self.p, self.cfg, self.stages = p, cfg, list(stages)
        self.visco = None
        if p.nmech:
            if visco is None:
                raise ValueError("an inversion with L > 0 mechanisms needs visco=(taus, taup, eta)")
            if cfg.hess:
                raise ValueError("the Hessian wavefields are elastic (ifos3d.c:929): no HESS with L > 0")
            self.visco = tuple(np.ascontiguousarray(a, np.float32) for a in visco)
        if cfg.exact_gradient and cfg.hess:
            raise ValueError("the approximate Hessian is formed from gradient_F's wavefields: not with exact_gradient")
        self.shots_raw, self.obs_raw = list(shots), np.ascontiguousarray(obs, np.float32)
        self.shots, self.obs = self.shots_raw, self.obs_raw
        self.recpos = np.ascontiguousarray(recpos, np.int32)
        self.srcpos_m = np.ascontiguousarray(srcpos_m, np.float32)
        self.model = [np.ascontiguousarray(a, np.float32).copy() for a in (rho, pi, u)]
        nf_max = max(len(s.finv) for s in self.stages)
        self.eng = Engine(p, max_shots=min(cfg.max_batch, len(self.shots)), max_nf=nf_max)
        self.eng.set_cpml(cpml)
        self.eng.set_receivers(self.recpos)
        self.opt = Optimizer(p.nx, p.ny, p.nz, numpar=cfg.numpar, bfgsnum=cfg.bfgsnum if cfg.lbfgs else 0)
        self.step = np.zeros(5, np.float64)    # step[0..4] (vector(0,4): zeros)
        self.stage_i, self.it_group, self.itmax, self.iteration = -1, 0, 0, 0
        self.hist = History()
        self.hess = None
        if cfg.hess and cfg.read_hess:  # ifos3d.c:658
            f, it = cfg.read_hess_at
            self.hess = fio.read_hessian(cfg.hess_file, f, it, p.ny, p.nx, p.nz, cfg.vp0, cfg.vs0, cfg.rho0)
        if cfg.mod_out_file:
            self._write_model(0)

    # -- helpers --------------------------------------------------------------
    def _write_model(self, iteration):
        i = self.cfg.ids
        fio.write_model(self.cfg.mod_out_file, iteration, *self.model, ghosted=True, idx=i[0], idy=i[1], idz=i[2])

    def _hess_signals(self, ntr_hess):
        """The Hessian wavefields' y-force per receiver: wavelet(..., 5, ...) of the
        receiver's recpos_loc column with amplitude 1 (a step at t = its trace
        number, ifos3d.c:893-895), low-passed with FILT; or cfg.hess_signal."""
        p, cfg = self.p, self.cfg
        if cfg.hess_signal is not None:
            sig = np.broadcast_to(np.asarray(cfg.hess_signal, np.float32), (ntr_hess, p.nt)).copy()
        else:
            rows = np.zeros((ntr_hess, 7), np.float32)
            rows[:, :3] = self.recpos[:ntr_hess]
            rows[:, 3] = np.arange(1, ntr_hess + 1)  # recpos_loc[4]: the trace number
            rows[:, 5] = 1.0
            sig = wavelet(p, 5, rows)
        if cfg.filt:
            sig = fstages.filt_seis(sig, float(self.finv[-1]), p.dt)
        return sig

    def _filter_stage(self, fc):
        """FILT: the raw source signals and observed data low-passed at fc."""
        dt = self.p.dt
        self.shots = [(sp, fstages.filt_seis(sig, fc, dt)) for sp, sig in self.shots_raw]
        o = self.obs_raw
        self.obs = fstages.filt_seis(o.reshape(-1, o.shape[-1]), fc, dt).reshape(o.shape)

    def _write_grad(self, g, iteration):
        if self.cfg.grad_file:
            i = self.cfg.ids
            fio.write_gradient(self.cfg.grad_file, float(self.finv[0]), iteration, g, idx=i[0], idy=i[1], idz=i[2])

    def _set_model(self, m):
        if self.visco:
            self.eng.set_model(*(a[1:-1, 1:-1, 1:-1] for a in m), *self.visco)
        else:
            self.eng.set_model(*(a[1:-1, 1:-1, 1:-1] for a in m), None, None, None)

    def _velocity_gradient(self, gm):
        """The exact VJP's derivative with respect to (rho, pi, u, taus, taup) onto
        modelupdate's parameters vp = sqrt(pi / rho), vs = sqrt(u / rho), rho (the
        relaxed velocities when L > 0, the relaxation times fixed)."""
        rho, pi, u = (a[1:-1, 1:-1, 1:-1].astype(np.float64) for a in self.model)
        vp, vs = np.sqrt(pi / rho), np.sqrt(u / rho)
        g_rho, g_pi, g_u = gm[0], gm[1], gm[2]
        return np.stack([g_pi * 2.0 * rho * vp, g_u * 2.0 * rho * vs, g_rho + g_pi * vp * vp + g_u * vs * vs])

    def _batches(self, idx):
        b = self.cfg.max_batch
        return [idx[i:i + b] for i in range(0, len(idx), b)]

    def _test_shots(self):
        n, k = len(self.shots), self.cfg.nshots_step
        return [(n // k) * q for q in range(k)]  # ishot1 = (nshots/NSHOTS_STEP)*(ishot-1)+1

    def _forward_misfit(self, m):
        self._set_model(m)
        total = 0.0
        for chunk in self._batches(self._test_shots()):
            self.eng.forward([self.shots[i] for i in chunk], want_sections=False)
            total += float(np.sum(self.eng.residual(self.obs[chunk])))
        return total

    # -- one iteration ----------------------------------------------------------
    def iterate(self):
        p, cfg = self.p, self.cfg
        self.iteration += 1
        if p.free_surf:
            self.opt.constant_boundary(*self.model, p.fw)
        if self.it_group >= self.itmax or self.iteration == 1:  # next frequency stage
            self.stage_i += 1
            st = self.stages[self.stage_i]
            self.finv = np.asarray(st.finv, np.float32)
            ntast = int(1.0 / (float(self.finv[-1]) * cfg.tast * p.dt)) or 1
            self.eng.set_frequencies(self.finv, ntast)
            if cfg.filt:
                self._filter_stage(float(self.finv[-1]))
            cdf, self.itmax, self.it_group = 1, st.itmax, 1
        else:
            cdf = 0
            self.it_group += 1
        # shot gradients and misfit[0] over the NSHOTS_STEP shots
        self._set_model(self.model)
        self.eng.zero_gradient()
        new_hess = cfg.hess and not cfg.read_hess and self.iteration == 1
        if new_hess:  # Hessian wavefields of ifos3d.c:882-938, once for all shots
            ntr_hess = len(self.recpos) // cfg.rec_hess
            self.eng.hessian_green(list(range(ntr_hess)), self._hess_signals(ntr_hess))
            self.eng.zero_hessian()
        mis = np.zeros(len(self.shots))
        gx = None
        if cfg.exact_gradient:
            gx = np.zeros((3, p.ny, p.nx, p.nz), np.float64)
        for chunk in self._batches(list(range(len(self.shots)))):
            if cfg.exact_gradient:
                self.eng.forward([self.shots[i] for i in chunk], want_sections=False)
                mis[chunk] = self.eng.residual(self.obs[chunk])
                gm, _ = self.eng.vjp_exact(cfg.exact_interval, moduli=True)
                gx += self._velocity_gradient(gm)
            else:
                mis[chunk] = self.eng.shot_gradient([self.shots[i] for i in chunk], self.obs[chunk])
            if new_hess:
                self.eng.hessian()  # hess_F of these shots (ifos3d.c:983)
        L2 = np.zeros(4, np.float64)
        L2[0] = float(np.sum(mis[self._test_shots()]))
        if new_hess:
            self.hess = self.eng.get_hessian()
            if cfg.hess_file:  # ifos3d.c:996
                fio.write_gradient(cfg.hess_file, float(self.finv[0]), self.iteration, self.hess,
                                   idx=cfg.ids[0], idy=cfg.ids[1], idz=cfg.ids[2])
        # gradient_F's sign: minus the misfit's derivative (a descent direction)
        g = (-gx).astype(np.float32) if cfg.exact_gradient else self.eng.get_gradient()
        self._write_grad(g, self.iteration)
        if cfg.hess and self.hess is not None:  # ifos3d.c:1002
            self.opt.hess_apply(g, self.hess, np.asarray(cfg.water_hess, np.float32), lbfgs=cfg.lbfgs,
                                vp0=cfg.vp0, vs0=cfg.vs0, rho0=cfg.rho0)
        self.opt.precon_grad(g, cfg.damptype, p.free_surf, p.fw, (p.dx, p.dy, p.dz), self.srcpos_m, self.recpos)
        self._write_grad(g, self.iteration + 1000)
        beta = None
        if cfg.lbfgs:
            if self.it_group > 1:
                self.opt.lbfgs(g, self.it_group)
            else:
                self.opt.lbfgs_savegrad(g)
                if cfg.lbfgs_first_normalised:
                    # The reference's first L-BFGS update of a stage moves the model by
                    # step * the raw gradient (modelupdate normalises only without
                    # L-BFGS), about 1e-20 of vp0: the model does not change and the
                    # history stays empty. With this option that one direction is
                    # normalised as modelupdate.c:105-117 normalises (each parameter
                    # by its largest magnitude; max rho 0 -> 1); the saved gradient
                    # and every later update are the reference's.
                    m = [float(np.abs(g[c]).max()) for c in range(3)]
                    if m[2] == 0.0:
                        m[2] = 1.0
                    if m[0] > 0.0 and m[1] > 0.0:
                        for c in range(3):
                            g[c] /= np.float32(m[c])
        else:
            beta = self.opt.conjugate(g, cdf)
        self._write_grad(g, self.iteration + 2000)
        # step length: two test models
        for steptest in (1, 2):
            if cdf == 1:
                self.step[4] = cfg.teststep
            self.step[steptest] = self.step[4] * steptest
            test = [a.copy() for a in self.model]
            self.opt.modelupdate(g, *test, self.step[steptest], cfg.weight, cfg.vp0, cfg.vs0, cfg.rho0,
                                 lbfgs=cfg.lbfgs, it_group=self.it_group)
            if p.free_surf:
                self.opt.constant_boundary(*test, p.fw)
            L2[steptest] = self._forward_misfit(test)
        steplength(L2, self.step, cfg.lbfgs, self.it_group, cfg.teststep)
        self.opt.modelupdate(g, *self.model, self.step[3], cfg.weight, cfg.vp0, cfg.vs0, cfg.rho0,
                             lbfgs=cfg.lbfgs, it_group=self.it_group)
        if cfg.mod_out_file:
            self._write_model(self.iteration)
        self.hist.misfit.append(L2[0])
        self.hist.step.append(float(self.step[3]))
        self.hist.beta.append(None if beta is None else beta.tolist())
        return L2[0]

    def run(self, iterations: int):
        for _ in range(iterations):
            self.iterate()
        return self.hist

    def close(self):
        self.eng.close()
        self.opt.close()
