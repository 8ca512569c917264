#!/usr/bin/env python
"""Benchmark of the B200 IFOS3D wavefield engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload visco256|elastic128|visco384|multiscale]
                    [--impl ours|reference]

A step is one pass of the hot path over one batch of synthetic input:
  visco256   (default) one viscoelastic (L=3) forward modelling run of a shot,
             256^3 cells, NT=3000, 400 receivers — the plain viscoelastic
             forward-modelling configuration; per GPU one shot (shots shard
             across ranks, no data-path collective: weak scaling).
  elastic128 one shot-gradient (forward + residual + adjoint + DFT gradient),
             128^3, NT=2000, 2 frequencies.
  multiscale a two-grid elastic inversion (the reference driver's iterations:
             shot gradients, precon_grad, CG, step-length test forwards, model
             update) on 96x64x96 cells at 2 m, then on 192x128x192 at 1 m
             from the resampled model, 16 shots, three frequency stages.
  visco384   the batched multi-shot gradient: 32 viscoelastic (L=3) shot-gradients
             (4 frequencies, 1024 receivers) on 384 x 256 x 384 cells, in
             HBM-sized batches of shots that share one launch; NT=200 by default
             (the configuration names no NT). Shots shard across ranks; one FP64
             all-reduce of gradient and misfits per step.
metric: cell-updates per second over all ranks (all NX*NY*NZ cells of every
shot and time step, CPML frame included; forward and adjoint both count).

Rank 0 prints one JSON line. Inputs are seeded synthetic models (no field data).
The state of one 256^3 L=3 shot (about 2.1 GB of fields) is far larger than the
126 MB L2, so every timed step streams from HBM without an explicit flush.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ifos3d-dev_b200"))

import numpy as np  # noqa: E402

METRIC = "Gcell-updates/s and shot-gradients/s, batched vs per-shot, grad rel-err<=1e-4"
UNIT = "Gcell-updates/s"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def slab_memberships(p) -> float:
    """Average number of CPML face slabs a cell lies in (x faces, z faces, bottom y
    face, plus the top y face without a free surface)."""
    n = p.nx * p.ny * p.nz
    fw = p.fw
    m = 2 * fw * p.ny * p.nz + 2 * fw * p.nx * p.ny + (1 if p.free_surf else 2) * fw * p.nx * p.nz
    return m / n


def alg_bytes_per_cell_step(p, nf: int, ntast: int) -> dict:
    """Compulsory HBM bytes per cell-update: every live state word read and written
    once, every model word read once, averaged moduli counted as recomputable.
    Split between the two kernels of a step (velocity / stress)."""
    L = p.nmech
    slab = slab_memberships(p)
    vel = 4 * (3 + 3) + 4 * 1 + 24 * slab            # v R+W, rho, 3 psi R+W per slab
    stress = 4 * (6 + 6) + 4 * 2 + 24 * slab          # sigma R+W, pi, u, 3 psi R+W per slab
    if L:
        stress += 48 * L + 8                           # 6 r R+W per mechanism, taus, taup
    stress += 48.0 * nf / max(ntast, 1)                # 6 DFT accumulators R+W per frequency
    return dict(vel=vel, stress=stress, total=vel + stress)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [x for x in vis.split(",") if x.strip()]
        self.gpu = ids[local_rank] if local_rank < len(ids) else str(local_rank)
        self.proc = None
        self.tmp = None

    def __enter__(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.tmp:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.tmp.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ---------------------------------------------------------------------------
# CPU side: the oracle (reported baseline and the reference arm)

def cpu_model() -> str:
    """The host CPU's model name (first /proc/cpuinfo entry)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _cpu_sample_worker(args):
    """One process: the CPU implementation on a bounded sample grid. With nf > 0 a
    whole shot-gradient (forward, residual, adjoint with the backward DFT,
    gradient_F), else one forward. Returns (seconds, cell-updates)."""
    kind, nx, ny, nz, nmech, nt, nf = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle, IfoParams
    from ifosb import synth
    finv = tuple(float(f) for f in np.linspace(200.0, 800.0, nf)) if nf else ()
    c = synth.small_case(nx=nx, ny=ny, nz=nz, nt=nt, fw=10, nmech=nmech, ntr=16, finv=finv)
    p = c["params"]
    ip = IfoParams(nx=p.nx, ny=p.ny, nz=p.nz, dx=p.dx, dy=p.dy, dz=p.dz, dt=p.dt, nt=p.nt, time=p.time,
                   fdcoeff=p.fdcoeff, free_surf=p.free_surf, fw=p.fw, nmech=p.nmech, ndt=1, ndtshift=0,
                   vppml=c["vppml"], fpml=c["fpml"], alpha=0.0, beta=0.0, source_shape=4)
    O = Oracle(kind, threads=1)  # one core per process
    vp, vs, rho = c["start"]
    m = O.readmod(ip, vp, vs, rho, tau=c["tau"], fl=c["fl"])
    cp = O.cpml_coeff(ip)
    sp = c["shots"][0]
    sig = O.wavelet(ip, sp)
    t0 = time.perf_counter()
    if nf:
        f = O.forward(ip, m, cp, sp, sig, c["recpos"], c["finv"], 1, True)
        obs = (f["sections"] * np.float32(0.9)).astype(np.float32)
        d, _ = O.residual(ip, obs, f["sections"])
        b = O.adjoint(ip, m, cp, c["recpos"], d, c["finv"], 1)
        O.gradient(ip, m, c["finv"], f["dft"], b["dft"])
        cells = 2 * nx * ny * nz * nt
    else:
        O.forward(ip, m, cp, sp, sig, c["recpos"])
        cells = nx * ny * nz * nt
    return time.perf_counter() - t0, cells


def cpu_run(kind, nmech, procs, grid, nt, nf=0):
    """Run `procs` single-threaded oracle processes (spawned) on the sample; returns
    (aggregate Gcell/s over the busiest process's time, over wall time, cells)."""
    import multiprocessing as mp
    args = [(kind, grid[0], grid[1], grid[2], nmech, nt, nf)] * procs
    t0 = time.perf_counter()
    if procs == 1:
        res = [_cpu_sample_worker(args[0])]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            res = pool.map(_cpu_sample_worker, args)
    wall = time.perf_counter() - t0
    cells = sum(r[1] for r in res)
    busy = max(r[0] for r in res)
    return cells / busy / 1e9, cells / wall / 1e9, cells


def cpu_sample(wl):
    """The bounded CPU sample of a workload: (nmech, nf, grid, nt, what)."""
    if wl == "visco384":
        # 1.6 M cells (0.5 GB of state and DFT fields per process, beyond any cache share;
        # a 36 % CPML frame against the full grid's 14 %), 24 steps: about 9 s on one core
        return 3, 4, (128, 96, 128), 24, "shot-gradient (forward + residual + adjoint + DFT + gradient_F)"
    if wl == "elastic128":
        return 0, 2, (64, 64, 64), 40, "shot-gradient (forward + residual + adjoint + DFT + gradient_F)"
    return 3, 0, (64, 64, 64), 40, "forward step"


def cpu_kind(nmech):
    """The reference itself (oracle/_ref) when it can run the workload, else the C restatement."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import have_ref
    return ("ref", "reference") if (nmech <= 1 and have_ref()) else ("oracle", "port")


# ---------------------------------------------------------------------------

def setup_dist(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        # bind this rank's GPU before the communicator exists (barriers and
        # collectives then run on it); the timeout bounds a rank waiting on a dead peer
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local, dist


def reference_arm(args, world, rank, dist):
    """Times the reference's CPU implementation on this host's cores (rank 0 only):
    one single-threaded process per core, each on a bounded sample of the workload's
    step (shot parallelism, as the reference runs its MPI ranks per shot)."""
    if rank != 0:
        return
    import multiprocessing as mp
    wl = args.workload
    nmech, nf, grid, nt, what = cpu_sample(wl)
    nt = args.cpu_nt or nt
    code, kind = cpu_kind(nmech)
    procs = max(1, min(mp.cpu_count(), args.cpu_procs or mp.cpu_count()))
    for _ in range(args.warmup if args.cpu_warmup else 0):
        cpu_run(code, nmech, procs, grid, max(2, nt // 4), nf)
    vals, walls = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        agg, _, cells = cpu_run(code, nmech, procs, grid, nt, nf)
        walls.append(time.perf_counter() - t0)
        vals.append(agg)
    value = float(np.median(vals))
    impl = "the reference's own C functions (oracle/_ref)" if kind == "reference" else \
        "the C restatement of the reference's algorithm (the reference stops at L=1)"
    sample = (f"{procs} single-threaded processes on {cpu_model()}, each one {what} on a "
              f"{grid[0]}x{grid[1]}x{grid[2]} grid x {nt} steps (FW=10 CPML, free surface, L={nmech}, nf={nf}) "
              f"with {impl}; Gcell-updates/s aggregated")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * float(np.median(walls)), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(wl, world),
        "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": procs, "kind": kind, "sample": sample,
                         "cpu_model": cpu_model()},
        "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


NT_VISCO384 = 100  # the batched-gradient configuration names no NT; 100 steps keep a step near 23 s


def workload_config(wl, world, nt=None):
    if wl == "visco384":
        nt = nt or NT_VISCO384
        return {"workload": "visco384: batched viscoelastic L=3 (Q=50, 20-200 Hz) shot-gradients (forward+residual+"
                            f"adjoint+DFT gradient), 384x384 horizontal x 256 deep cells, NT={nt}, 4 frequencies, "
                            "32 shots on an 8x4 surface grid, 1024 receivers, 3 Gaussian blobs in a depth gradient",
                "grid": [384, 256, 384],
                "grid_axes": "NX x NY x NZ with y the reference's depth axis: 384 x 384 horizontal (x, z), 256 deep",
                "nt": nt, "nt_choice": "the configuration names no NT; DT=1e-4 s, NT chosen so that a step "
                                       "(all 32 shot-gradients) takes about 23 s on one B200",
                "nmech": 3, "nf": 4, "shots": 32, "receivers": 1024,
                "parallelism": f"shot-sharded x{world}, FP64 gradient all-reduce per step",
                "l2_flush": "state+DFT about 11 GB per shot > 126 MB L2"}
    if wl == "visco256":
        return {"workload": "visco256: viscoelastic L=3 (Q=50, 20-200 Hz) forward modelling, 256^3 cells, "
                            "NT=3000, 8 layers, sin^3 fc=80 Hz, 400 receivers, 1 shot per GPU",
                "grid": [256, 256, 256], "nt": 3000, "nmech": 3, "shots_per_gpu": 1, "receivers": 400,
                "parallelism": f"shot-sharded x{world}", "l2_flush": "state 2.1 GB per shot > 126 MB L2"}
    return {"workload": "elastic128: elastic FWI shot-gradient (forward+residual+adjoint+DFT gradient), 128^3, "
                        "NT=2000, 2 frequencies, 25 receivers, 1 shot per GPU",
            "grid": [128, 128, 128], "nt": 2000, "nmech": 0, "nf": 2, "shots_per_gpu": 1, "receivers": 25,
            "parallelism": f"shot-sharded x{world}" + (", FP64 gradient all-reduce per step" if world > 1 else ""),
            "l2_flush": "state+DFT 0.37 GB per shot > 126 MB L2"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="visco384",
                    choices=["visco384", "visco256", "elastic128", "multiscale", "multiscale_visco"])
    ap.add_argument("--iterations-per-stage", type=int, default=3, help="multiscale_visco: L-BFGS iterations per stage")
    ap.add_argument("--ms-scale", type=float, default=0.5, help="multiscale_visco: linear size against the configuration")
    ap.add_argument("--ms-shots-side", type=int, default=4, help="multiscale_visco: shots per side of the surface grid")
    ap.add_argument("--ms-iterations", type=int, default=0, help="multiscale_visco: cap on the iterations run (0: all)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nt", type=int, default=None, help="override NT (testing only)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--cpu-procs", type=int, default=0)
    ap.add_argument("--cpu-nt", type=int, default=0, help="time steps of the CPU sample (0 = the workload's)")
    ap.add_argument("--e2e-steps", type=int, default=3, help="timed end-to-end steps (at most --steps)")
    ap.add_argument("--per-shot-n", type=int, default=4, help="shots timed on the one-shot-per-launch path")
    ap.add_argument("--cpu-warmup", action="store_true")
    ap.add_argument("--grid", default=None, help="visco384 only: NX,NY,NZ (profiling runs)")
    ap.add_argument("--nshots", type=int, default=None, help="visco384 only: shots per step (profiling runs)")
    ap.add_argument("--shape", default=None,
                    help="launch shape cy_vel,l2_vel,cy_str,l2_str instead of autotuning (profiling runs)")
    ap.add_argument("--td-interval", type=int, default=0,
                    help="elastic128 only: the step is the time-domain gradient (forward with checkpoints every "
                         "K steps, residual, ifosb_gradient_td) instead of the DFT shot-gradient")
    args = ap.parse_args()
    world, rank, local, dist = setup_dist(args)
    if args.impl == "reference":
        reference_arm(args, world, rank, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.workload in ("multiscale", "multiscale_visco"):
        if rank == 0:
            (multiscale_workload if args.workload == "multiscale" else multiscale_visco_workload)(args, local)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload == "visco384":
        batched_gradient_workload(args, world, rank, local, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch
    import ifosb
    from ifosb import synth
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    wl = args.workload
    td_k = args.td_interval if wl == "elastic128" else 0
    if td_k and dist:
        raise SystemExit("--td-interval runs on one GPU")
    c = synth.case(wl, nt=args.nt)
    p = c["params"]
    # shot sharding: rank r models its own source position (a shifted copy of the case's shot)
    sp = c["shots"][0].copy()
    sp[0, 0] = min(p.nx - p.fw - 1, max(p.fw + 2, int(sp[0, 0]) + 8 * (rank - world // 2)))
    c["shots"] = [sp]
    m, cp, shots = synth.build_inputs(c)
    nf = len(c["finv"])
    eng = ifosb.Engine(p, max_shots=1, max_nf=nf)
    eng.set_stream(stream.cuda_stream)
    eng.set_cpml(cp)
    eng.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
    eng.set_receivers(c["recpos"])
    eng.set_frequencies(c["finv"] if nf else None, c["ntast"])
    cells_step = p.nx * p.ny * p.nz * p.nt * (2 if wl == "elastic128" else 1)

    obs = None
    if wl == "elastic128":
        # observed data: the same shot in the true (anomaly) model
        mt, _, _ = synth.build_inputs(c, "true")
        eng.set_model(mt["rho"], mt["pi"], mt["u"], mt["taus"], mt["taup"], mt["eta"])
        obs = eng.forward(shots)
        eng.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])

    if wl == "elastic128" and dist:
        # N ranks: one shot each, then the exchange step of a gradient iteration, the
        # FP64 all-reduce of the gradient and misfits (ifosb.dist); the entries of the
        # other ranks' shots are placeholders (each rank computes only its own)
        from ifosb.dist import distributed_shot_gradient
        all_shots = [shots[0]] * world
        all_obs = np.zeros((world,) + obs.shape[1:], np.float32)
        all_obs[rank] = obs[0]

    # launch shape for this batch from the engine's autotuner (not timed)
    if args.shape:
        sh = [int(x) for x in args.shape.split(",")]
        eng.set_launch_shape(len(shots), sh)
        tuned = {"velocity": {"y_planes_per_cta": sh[0], "l2_prefetch_planes": sh[1]},
                 "stress": {"y_planes_per_cta": sh[2], "l2_prefetch_planes": sh[3]}}
    else:
        tuned = eng.autotune(shots, steps=min(60, p.nt))

    if td_k:
        eng.set_td_checkpoints(td_k)

    def step():
        if wl == "elastic128" and dist:
            distributed_shot_gradient(eng, all_shots, all_obs, max_batch=1, dist=dist)
        elif td_k:
            eng.forward(shots, want_sections=False)
            eng.residual(obs)
            eng.gradient_td(td_k)
        elif wl == "elastic128":
            eng.shot_gradient(shots, obs)
        else:
            eng.forward(shots, want_sections=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
    clocks = clk.summary()
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    # our kernels per step: 2 per time step (velocity, stress); a shot-gradient adds the
    # adjoint loop, residual + misfit and the gradient kernel
    launches = args.steps * (2 * p.nt if wl == "visco256" else 4 * p.nt + 3)
    if td_k:
        # forward 2 NT + NT sums; residual 2; recomputed steps 2 last + last sums, adjoint
        # 2 NT + NT sums, last correlations, one dc kernel (last = TIME/DT - 1)
        last = round(float(p.time) / float(p.dt)) - 1
        launches = args.steps * (3 * p.nt + 2 + 3 * last + 3 * p.nt + last + 1)
    value = world * cells_step * args.steps / (ms / 1000.0) / 1e9

    # ---- end to end through the public API: host model + wavelet in, traces out, every step
    pin = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(ifosb.ghost_wrap(a))).pin_memory()
    hm = {k: pin(m[k]) for k in ("rho", "pi", "u", "taus", "taup")}
    sig_pinned = torch.from_numpy(shots[0][1]).pin_memory()
    h2d = sum(t.numel() * 4 for t in hm.values() if t is not None) + sig_pinned.numel() * 4 + sp.size * 4
    d2h = 3 * eng.ntr * eng.ns * 4 * (1 if wl == "visco256" else 2)
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev2.record(stream)
    for _ in range(args.steps):
        eng.set_model(*[None if hm[k] is None else hm[k].numpy() for k in ("rho", "pi", "u", "taus", "taup")],
                      m["eta"], ghosted=True)
        if td_k:
            eng.forward([(sp, sig_pinned.numpy())], want_sections=False)
            eng.residual(obs)
            eng.gradient_td(td_k)
        elif wl == "elastic128":
            eng.shot_gradient([(sp, sig_pinned.numpy())], obs)
            eng.get_gradient()
        else:
            eng.forward([(sp, sig_pinned.numpy())], want_sections=True)
    ev3.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = ev2.elapsed_time(ev3)
    if dist:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = world * cells_step * args.steps / (ms_e2e / 1000.0) / 1e9
    if wl == "elastic128":
        d2h = 3 * eng.ntr * eng.ns * 4 + 3 * p.nx * p.ny * p.nz * 4
    if td_k:
        h2d += obs.nbytes
        d2h = 4 * p.nx * p.ny * p.nz * 8 + 8  # the four FP64 kernels and the misfit

    # ---- roofline: per-kernel CUDA events on the launching stream over one profiled step
    eng.set_profiling(True)
    eng.forward(shots, want_sections=False)
    tv, ts, nsteps = eng.kernel_times()
    eng.set_profiling(False)
    b = alg_bytes_per_cell_step(p, nf if wl == "elastic128" else 0, c["ntast"])
    ncell = p.nx * p.ny * p.nz
    peak, peak_kind = load_peaks()
    ach_step = b["total"] * ncell / ((tv + ts) / nsteps / 1000.0) / 1e9
    ach_str = b["stress"] * ncell / (ts / nsteps / 1000.0) / 1e9
    ach_vel = b["vel"] * ncell / (tv / nsteps / 1000.0) / 1e9
    # DRAM bytes per launch from an ncu capture of the same kernels (committed
    # summary, not this run); null when no capture of this workload exists
    traffic = load_traffic(wl, ncell)
    roofline = {"bound": "hbm", "kernel": "time step = k_velocity + k_stress<L> (one launch each)",
                "achieved": round(ach_step, 1), "peak": peak, "unit": "GB/s", "frac": round(ach_step / peak, 4),
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": traffic["time_step"] if traffic else None,
                "traffic_source": traffic["source"] if traffic else "no ncu capture of this workload",
                "alg_bytes_per_step": round(b["total"] * ncell), "alg_bytes_per_cell_step": round(b["total"], 2),
                "per_kernel": {"k_stress": {"alg_bytes_per_cell": round(b["stress"], 2), "ms": round(ts / nsteps, 4),
                                            "achieved_gbs": round(ach_str, 1), "frac": round(ach_str / peak, 4),
                                            "traffic": traffic["k_stress"] if traffic else None},
                               "k_velocity": {"alg_bytes_per_cell": round(b["vel"], 2), "ms": round(tv / nsteps, 4),
                                              "achieved_gbs": round(ach_vel, 1), "frac": round(ach_vel / peak, 4),
                                              "traffic": traffic["k_velocity"] if traffic else None}}}

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(workload_config(wl, world),
                       launch_shape=dict(tuned, picked_by="--shape" if args.shape else "ifosb_autotune")),
        "clocks": clocks,
        "e2e": {"value": round(e2e, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches), "roofline": roofline, "graph_captures": eng.graph_captures,
    }
    if wl == "elastic128":
        out["shot_gradients_per_s"] = round(world * args.steps / (ms / 1000.0), 4)
    if td_k:
        out["config"]["gradient"] = (f"time-domain kernels (ifosb_gradient_td, interval {td_k}, checkpoints kept by "
                                     "the forward) instead of the DFT shot-gradient")

    # ---- extras (rank 0, one GPU): batched vs one-shot-per-launch shot-gradients of elastic128
    if rank == 0 and world == 1 and not args.no_extras and not td_k:
        eng.close()
        out["shot_gradients"] = shot_gradient_comparison(torch, ifosb, synth, dev, stream, args.nt)
        out["shot_gradients_small_grid"] = small_grid_comparison(torch, ifosb, synth, dev, stream, args.nt)
        if wl == "elastic128":
            out["time_domain_gradient"] = time_domain_comparison(torch, ifosb, synth, dev, stream, args.nt)
    # ---- CPU baseline (rank 0, N=1): the oracle on a bounded sample of this workload
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline_line(wl, args)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _pinned(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def batched_gradient_workload(args, world, rank, local, dist):
    """visco384 (the default): every rank takes its share of the 32 shots in batches
    as large as its HBM holds (one launch per kernel and time step for a whole
    batch, the time loop replayed from a CUDA graph); a step is the gradient of all
    32 shots, summed in FP64 on every rank.

    value: observed traces already resident in HBM, the gradient left there (and
           all-reduced there when N > 1);
    e2e:   the same step through the public API from host memory: the model and
           the observed traces copied in from pinned buffers, the FP64 gradient and
           the misfits read back, every step."""
    import torch
    import ifosb
    from ifosb import synth
    from ifosb.dist import batches, distributed_shot_gradient, shard
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    nt = args.nt or NT_VISCO384
    grid = tuple(int(x) for x in args.grid.split(",")) if args.grid else None
    c = synth.case("visco384", nt=nt, nshots=args.nshots, grid=grid)
    p = c["params"]
    m, cp, shots = synth.build_inputs(c)
    nf, nshots = len(c["finv"]), len(shots)
    mine = shard(nshots, world, rank)

    def engine(nb, mode=0):
        e = ifosb.Engine(p, max_shots=nb, max_nf=nf)
        e.set_stream(stream.cuda_stream)
        e.set_launch_mode(mode)
        e.set_cpml(cp)
        e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
        e.set_receivers(c["recpos"])
        e.set_frequencies(c["finv"], c["ntast"])
        return e

    # batch size: the shots this GPU's free memory holds next to a 6 GB margin
    e = engine(1)
    b1 = e.device_bytes
    e.close()
    e = engine(2)
    per_shot = e.device_bytes - b1
    e.close()
    free, _ = torch.cuda.mem_get_info(dev)
    cap = max(1, int((free - 6e9 - (b1 - per_shot)) // per_shot))
    nbatch = -(-len(mine) // min(cap, len(mine)))
    B = -(-len(mine) // nbatch)
    eng = engine(B)
    last = len(mine) - (nbatch - 1) * B
    if args.shape:
        sh = [int(x) for x in args.shape.split(",")]
        for nb in {B, last}:
            eng.set_launch_shape(nb, sh)
        tuned = {"velocity": {"y_planes_per_cta": sh[0], "l2_prefetch_planes": sh[1]},
                 "stress": {"y_planes_per_cta": sh[2], "l2_prefetch_planes": sh[3]}}
    else:
        tuned = eng.autotune([shots[i] for i in mine[:B]], steps=min(40, p.nt))
        if last != B:  # a shorter last batch gets its own launch shape
            eng.autotune([shots[i] for i in mine[-last:]], steps=min(40, p.nt))
    # observed data: this rank's shots modelled in the same (true = start) model and
    # scaled, so that the residual is not zero; other ranks' entries are placeholders
    obs = np.zeros((nshots, 3, eng.ntr, eng.ns), np.float32)
    for chunk in batches(mine, B):
        obs[chunk] = eng.forward([shots[i] for i in chunk]) * np.float32(0.9)
    obs_dev = torch.from_numpy(obs).to(dev)

    def step():
        return distributed_shot_gradient(eng, shots, obs_dev, max_batch=B, dist=dist)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        for _ in range(args.steps):
            grad, mis = step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
    clocks = clk.summary()
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ncell = p.nx * p.ny * p.nz
    cells_step = 2 * ncell * p.nt * nshots
    value = cells_step * args.steps / (ms / 1000.0) / 1e9
    launches = args.steps * nbatch * (4 * p.nt + 3)

    # ---- end to end: host model and host observed traces in, FP64 gradient out, every step
    hm = {k: _pinned(torch, ifosb.ghost_wrap(m[k])) for k in ("rho", "pi", "u", "taus", "taup")}
    obs_pin = _pinned(torch, obs)
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    for _ in range(e2e_steps):
        eng.set_model(*(hm[k].numpy() for k in ("rho", "pi", "u", "taus", "taup")), m["eta"], ghosted=True)
        hgrad, hmis = distributed_shot_gradient(eng, shots, obs_pin.numpy(), max_batch=B, dist=dist)
    ev3.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = ev2.elapsed_time(ev3)
    if dist:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = cells_step * e2e_steps / (ms_e2e / 1000.0) / 1e9
    # the device-resident and host paths give the same gradient
    same = bool(np.array_equal(grad.cpu().numpy(), hgrad) and np.array_equal(mis, hmis))
    h2d = int(obs[mine].nbytes + sum(t.numel() * 4 for t in hm.values()))
    d2h = int(hgrad.nbytes + hmis.nbytes)

    # ---- roofline: per-kernel CUDA events over one profiled batched forward (with DFT)
    eng.set_profiling(True)
    eng.forward([shots[i] for i in mine[:B]], want_sections=False)
    tv, ts, nsteps = eng.kernel_times()
    eng.shot_gradient([shots[i] for i in mine[:B]], obs[mine[:B]])
    atv, ats, ansteps = eng.kernel_times()  # the adjoint loop of that shot-gradient
    eng.set_profiling(False)
    b = alg_bytes_per_cell_step(p, nf, c["ntast"])
    peak, peak_kind = load_peaks()
    cb = ncell * B
    ach = b["total"] * cb / ((tv + ts) / nsteps / 1000.0) / 1e9
    ach_s = b["stress"] * cb / (ts / nsteps / 1000.0) / 1e9
    ach_v = b["vel"] * cb / (tv / nsteps / 1000.0) / 1e9
    traffic = load_traffic("visco384", cb)
    roofline = {"bound": "hbm", "kernel": f"time step of a {B}-shot batch = k_velocity + k_stress<3> with DFT",
                "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": traffic["time_step"] if traffic else None,
                "traffic_source": traffic["source"] if traffic else "no ncu capture of this workload",
                "alg_bytes_per_cell_step": round(b["total"], 2), "alg_bytes_per_step": round(b["total"] * cb),
                "per_kernel": {"k_stress": {"alg_bytes_per_cell": round(b["stress"], 2), "ms": round(ts / nsteps, 4),
                                            "achieved_gbs": round(ach_s, 1), "frac": round(ach_s / peak, 4),
                                            "traffic": traffic["k_stress"] if traffic else None},
                               "k_velocity": {"alg_bytes_per_cell": round(b["vel"], 2), "ms": round(tv / nsteps, 4),
                                              "achieved_gbs": round(ach_v, 1), "frac": round(ach_v / peak, 4),
                                              "traffic": traffic["k_velocity"] if traffic else None}},
                "adjoint_ms_per_step": {"k_stress": round(ats / ansteps, 4), "k_velocity": round(atv / ansteps, 4)},
                "timing": "CUDA events around every launch of one forward and one adjoint, on the engine's stream"}
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(workload_config("visco384", world, p.nt), shots_per_batch=B, batches_per_gpu=nbatch,
                       launch_shape=dict(tuned, picked_by="--shape" if args.shape else "ifosb_autotune")),
        "clocks": clocks,
        "e2e": {"value": round(e2e, 3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps, "shot_gradients_per_s": round(nshots * e2e_steps / (ms_e2e / 1000.0), 4),
                "inputs": "ghosted model (rho, pi, u, taus, taup) and observed traces from pinned host memory",
                "outputs": "FP64 gradient [3][NY][NX][NZ] and per-shot FP64 misfits to host",
                "same_gradient_as_device_path": same},
        "gpu_launches": int(launches), "graph_captures": eng.graph_captures, "roofline": roofline,
        "shot_gradients_per_s": round(nshots * args.steps / (ms / 1000.0), 4),
    }
    eng.close()
    del obs_dev
    if rank == 0 and world == 1 and not args.no_extras:
        out["per_shot_path"] = per_shot_comparison(torch, ifosb, dev, stream, engine, shots, obs, B, tuned,
                                                   nshots * args.steps / (ms / 1000.0), args.per_shot_n)
        out["visco256_forward"] = visco256_forward(torch, ifosb, synth, dev, stream)
        out["shot_gradients_elastic128"] = shot_gradient_comparison(torch, ifosb, synth, dev, stream, None)
        out["shot_gradients_small_grid"] = small_grid_comparison(torch, ifosb, synth, dev, stream, None)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline_line("visco384", args)
    if grid or args.nshots:  # a reduced case: name what ran
        out["config"].update(grid=[p.nx, p.ny, p.nz], shots=nshots, workload="visco384 reduced for profiling: "
                             f"{p.nx}x{p.ny}x{p.nz} cells, {nshots} shots, NT={p.nt}")
    if rank == 0:
        print(json.dumps(out), flush=True)


def cpu_baseline_line(wl, args):
    """The CPU implementation on one host core over a bounded sample of the workload's step."""
    nmech, nf, grid, nt, what = cpu_sample(wl)
    nt = args.cpu_nt or nt
    code, kind = cpu_kind(nmech)
    v1, _, _ = cpu_run(code, nmech, 1, grid, nt, nf)
    impl = "the reference's own C functions (oracle/_ref)" if kind == "reference" else \
        "the C restatement of the reference's algorithm (the reference stops at L=1)"
    return {"value": round(v1, 5), "unit": UNIT, "cores": 1, "kind": kind, "cpu_model": cpu_model(),
            "sample": f"one core, one {what} on a {grid[0]}x{grid[1]}x{grid[2]} grid x {nt} steps "
                      f"(L={nmech}, nf={nf}, FW=10 CPML, free surface) with {impl}"}


def per_shot_comparison(torch, ifosb, dev, stream, engine, shots, obs, B, tuned_batch, batched_rate, n):
    """One shot per launch sequence on the same GPU, the time loop also replayed
    from a CUDA graph (so the ratio isolates batching), autotuned for one shot;
    its gradient of the first shots compared bit for bit with one batched launch."""
    e1 = engine(1, 0)
    tuned1 = e1.autotune(shots[:1], steps=min(40, e1.p.nt))
    e1.shot_gradient(shots[:1], obs[:1])  # warm-up: graph capture
    e1.zero_gradient()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for s in range(n):
        e1.shot_gradient(shots[s:s + 1], obs[s:s + 1])
    torch.cuda.synchronize(dev)
    t1 = (time.perf_counter() - t0) / n
    g1 = e1.get_gradient()
    e1.close()
    # and kernel by kernel, without the graph (the plain one-shot-per-launch path)
    e1 = engine(1, 1)
    e1.set_launch_shape(1, tuned1)
    e1.shot_gradient(shots[:1], obs[:1])
    e1.zero_gradient()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for s in range(n):
        e1.shot_gradient(shots[s:s + 1], obs[s:s + 1])
    torch.cuda.synchronize(dev)
    tp = (time.perf_counter() - t0) / n
    same_modes = np.array_equal(e1.get_gradient(), g1)
    e1.close()
    eb = engine(B, 0)
    eb.set_launch_shape(n, tuned_batch)
    eb.shot_gradient(shots[:n], obs[:n])
    gb = eb.get_gradient()
    eb.close()
    return {"shot_gradients_per_s": round(1.0 / t1, 4), "batched_speedup": round(batched_rate * t1, 3),
            "launch": "CUDA graph per shot (the same time-loop replay as the batched path)",
            "plain_launch_shot_gradients_per_s": round(1.0 / tp, 4),
            "batched_speedup_vs_plain_launch": round(batched_rate * tp, 3),
            "launch_shape_one_shot": tuned1,
            "timing": f"host wall clock around {n} synchronised one-shot gradients after a warm-up",
            "gradients_bit_identical": bool(np.array_equal(g1, gb) and same_modes),
            "compared": f"gradient of shots 0..{n - 1}: one shot per launch vs one {n}-shot launch"}


def visco256_forward(torch, ifosb, synth, dev, stream, steps=2):
    """The plain viscoelastic forward-modelling configuration (256^3, L=3, NT=3000,
    400 receivers, one shot): Gcell-updates/s and the time-step roofline."""
    c = synth.case("visco256")
    p = c["params"]
    m, cp, shots = synth.build_inputs(c)
    e = ifosb.Engine(p, max_shots=1, max_nf=0)
    e.set_stream(stream.cuda_stream)
    e.set_cpml(cp)
    e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
    e.set_receivers(c["recpos"])
    e.set_frequencies(None, 1)
    tuned = e.autotune(shots, steps=60)
    e.forward(shots, want_sections=False)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        e.forward(shots, want_sections=False)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1) / steps
    e.set_profiling(True)
    e.forward(shots, want_sections=False)
    tv, ts, n = e.kernel_times()
    e.close()
    ncell = p.nx * p.ny * p.nz
    b = alg_bytes_per_cell_step(p, 0, 1)
    peak, _ = load_peaks()
    ach = b["total"] * ncell / ((tv + ts) / n / 1000.0) / 1e9
    return {"workload": "visco256: L=3 forward modelling, 256^3, NT=3000, 400 receivers, 1 shot",
            "gcell_updates_per_s": round(ncell * p.nt / (ms / 1000.0) / 1e9, 3), "ms_per_forward": round(ms, 1),
            "steps": steps, "launch_shape": tuned,
            "roofline_time_step": {"alg_bytes_per_cell_step": round(b["total"], 2), "achieved_gbs": round(ach, 1),
                                   "frac": round(ach / peak, 4), "k_velocity_ms": round(tv / n, 4),
                                   "k_stress_ms": round(ts / n, 4)}}


def load_traffic(wl, cell_shots):
    """DRAM bytes per launch from the committed ncu summaries (profiles/traffic.json),
    per cell-shot scaled to this launch when the capture ran a smaller case; None
    when no capture of the workload exists."""
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(tf)).get(wl)
    except Exception:
        return None
    if not d:
        return None
    scale = cell_shots / d["cell_shots"] if d.get("cell_shots") else 1.0
    src = "profiles/traffic.json (an earlier ncu capture, not this run)"
    if scale != 1.0:
        src += f": {d['captured']}, scaled by cell-shots x{scale:.1f}"
    return {"k_velocity": int(d["k_velocity"] * scale), "k_stress": int(d["k_stress"] * scale),
            "time_step": int(d["time_step"] * scale), "source": src}


def multiscale_workload(args, local):
    """The multiscale inversion loop reduced to one GPU and about a minute: the
    reference driver's iterations (ifosb.inversion) on a 2 m grid for two
    frequency stages, the model resampled to a 1 m grid, one more stage there.
    The true model is four layers and two Gaussian blobs (+10 % vp); the start
    model is it smoothed by a 15 m Gaussian. Elastic, as the reference's
    inversion path is (its viscoelastic stress calls are commented out), CG
    updating vp (WEIGHT 1 0 0), no free surface (precon_grad's damping types 0-2
    zero the gradient with one). Timed by the host clock around the synchronous
    calls: an inversion has no repeatable step to warm up."""
    import torch
    from scipy.ndimage import gaussian_filter
    import ifosb
    from ifosb import stages as fst
    from ifosb import synth
    from ifosb.inversion import Inversion, Settings, Stage
    torch.cuda.set_device(local)
    rng = np.random.default_rng(5)
    fw, fc, nsh_side, h_fine = 10, 150.0, 4, 1.0
    fine = (128, 192, 192)  # (NY, NX, NZ), y down
    jj, ii, kk = np.meshgrid(*(np.arange(n) for n in fine), indexing="ij")
    bounds = np.sort(rng.choice(np.arange(20, fine[0] - 20), 3, replace=False))
    vps = np.array([2500.0, 3000.0, 3500.0, 4000.0], np.float32)
    vp_t = vps[np.searchsorted(bounds, np.arange(fine[0]), side="right")][:, None, None] * np.ones(fine, np.float32)
    for _ in range(2):
        c = [rng.uniform(40, n - 40) for n in fine]
        vp_t *= 1 + 0.1 * np.exp(-((jj - c[0]) ** 2 + (ii - c[1]) ** 2 + (kk - c[2]) ** 2) / (2 * 12.0 ** 2))
    vp_t = vp_t.astype(np.float32)
    true = (vp_t, (vp_t / np.float32(math.sqrt(3))).astype(np.float32), (1700 + 0.2 * vp_t).astype(np.float32))
    start = tuple(gaussian_filter(a.astype(np.float64), 15.0, mode="nearest").astype(np.float32) for a in true)
    grids = [dict(h=2.0, dt=2e-4, nt=500, stages=[Stage([27.0, 53.0, 80.0], 2), Stage([80.0, 120.0, 160.0], 2)]),
             dict(h=1.0, dt=1e-4, nt=1000, stages=[Stage([160.0, 213.0, 267.0], 2)])]
    inner = lambda a: a[fw:-fw, fw:-fw, fw:-fw]  # noqa: E731
    err = lambda vp: float(np.linalg.norm(inner(vp) - inner(vp_t)) / np.linalg.norm(inner(vp_t)))  # noqa: E731
    cur = start
    hist, cells, t_total = [], 0, 0.0
    vp_err = {"start": err(start[0])}
    for gi, gd in enumerate(grids):
        s = gd["h"] / h_fine
        shape = tuple(int(n / s) for n in fine)
        ny, nx, nz = shape
        if s != 1:
            mt = [fst.resample(a, (h_fine,) * 3, shape, (gd["h"],) * 3) for a in true]
            m0 = [fst.resample(a, (h_fine,) * 3, shape, (gd["h"],) * 3) for a in cur]
        else:
            mt, m0 = list(true), list(cur)
        p = ifosb.make_params(nx, ny, nz, dh=gd["h"], dt=gd["dt"], nt=gd["nt"], fdcoeff=2, free_surf=0, fw=fw,
                              nmech=0)
        xs = np.linspace(fw + 6, nx - fw - 6, nsh_side).round().astype(int)
        zs = np.linspace(fw + 6, nz - fw - 6, nsh_side).round().astype(int)
        shots = [(sp, ifosb.wavelet(p, 4, sp)) for sp in (synth._src(int(x), fw + 3, int(z), fc) for x in xs for z in zs)]
        rec = synth._grid_receivers(nx, nz, 16, fw + 2, fw + 3)
        cp = ifosb.cpml_coeff(p, 4000.0, fc)
        e = ifosb.Engine(p, max_shots=len(shots), max_nf=0)
        e.set_cpml(cp)
        e.set_receivers(rec)
        mod = ifosb.moduli(p, *(a.ravel() for a in mt))
        e.set_model(*(mod[k].reshape(shape) for k in ("rho", "pi", "u")), None, None, None)
        obs = e.forward(shots)
        e.close()
        mod0 = ifosb.moduli(p, *(a.ravel() for a in m0))
        ghost = [ifosb.ghost_wrap(mod0[k].reshape(shape)) for k in ("rho", "pi", "u")]
        srcpos_m = np.array([[sp[0, 0] * gd["h"], sp[0, 1] * gd["h"], sp[0, 2] * gd["h"]] for sp, _ in shots], np.float32)
        cfg = Settings(teststep=0.02, damptype=2, lbfgs=False, nshots_step=4, max_batch=len(shots),
                       weight=(1.0, 0.0, 0.0))
        inv = Inversion(p, cp, rec, shots, obs, srcpos_m, *ghost, gd["stages"], cfg)
        iters = sum(st.itmax for st in gd["stages"])
        ncell = nx * ny * nz
        for _ in range(iters):
            t0 = time.perf_counter()
            mis = inv.iterate()
            t_total += time.perf_counter() - t0
            cells += ncell * p.nt * (2 * len(shots) + 2 * cfg.nshots_step)
            hist.append({"grid": gi, "misfit": mis, "t_s": round(t_total, 3), "step": inv.hist.step[-1]})
        rho, pi, u = (a[1:-1, 1:-1, 1:-1].astype(np.float64) for a in inv.model)
        got = ((np.sqrt(pi / rho)).astype(np.float32), (np.sqrt(u / rho)).astype(np.float32), rho.astype(np.float32))
        inv.close()
        cur = tuple(fst.resample(a, (gd["h"],) * 3, fine, (h_fine,) * 3) for a in got) if s != 1 else got
        vp_err[f"after_grid{gi}"] = err(cur[0])
    per_grid = {}
    for gi in range(len(grids)):
        m = [x["misfit"] for x in hist if x["grid"] == gi]
        per_grid[f"grid{gi}"] = {"first": m[0], "last": m[-1], "reduction": round(1 - m[-1] / m[0], 4)}
    out = {
        "metric": METRIC, "value": round(cells / t_total / 1e9, 3), "unit": UNIT, "n_gpus": 1,
        "steps": len(hist), "warmup": 0, "ms_per_step": round(1000 * t_total / len(hist), 1),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "multiscale: elastic inversion, 96x64x96 @ 2 m (NT=500, 2 stages x 2 iterations) "
                               "then 192x128x192 @ 1 m (NT=1000, 1 stage x 2 iterations), 16 shots, 256 receivers, "
                               "CG on vp, 4 layers + 2 blobs, start smoothed by 15 m",
                   "timing": "host clock around synchronous calls; value counts the shot gradients and the "
                             "step-length test forwards"},
        "inversion": {"iterations": hist, "misfit_per_grid": per_grid, "vp_rel_error": vp_err,
                      "seconds": round(t_total, 2)},
    }
    print(json.dumps(out), flush=True)


def time_domain_comparison(torch, ifosb, synth, dev, stream, nt_override, interval=50, reps=2):
    """One elastic128 shot-gradient by the DFT path (forward + residual + adjoint +
    gradient_F at the case's 2 frequencies) against the time-domain path (forward
    keeping checkpoints every `interval` steps + residual + ifosb_gradient_td),
    elastic and L=3 (Q=50 over 20-200 Hz): seconds per shot-gradient, CUDA events
    over `reps` repetitions after one warm-up each."""
    out = {"interval": interval}
    for nmech in (0, 3):
        c = synth.case("elastic128", nt=nt_override)
        p = c["params"]
        if nmech:
            p.nmech = 3
            c["tau"], c["fl"] = synth.q_tau_fit(50.0, 20.0, 200.0, 3)
        m, cp, shots = synth.build_inputs(c)
        e = ifosb.Engine(p, max_shots=1, max_nf=2)
        e.set_stream(stream.cuda_stream)
        e.set_cpml(cp)
        e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
        e.set_receivers(c["recpos"])
        e.set_frequencies(c["finv"], c["ntast"])
        obs = (0.9 * e.forward(shots)).astype(np.float32)

        def dft():
            e.shot_gradient(shots, obs)

        def td():
            e.forward(shots, want_sections=False)
            e.residual(obs)
            e.gradient_td(interval)

        res = {}
        for name, fn in (("dft_s", dft), ("time_domain_s", td)):
            e.set_td_checkpoints(interval if name == "time_domain_s" else 0)
            fn()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            ev0.record(stream)
            for _ in range(reps):
                fn()
            ev1.record(stream)
            torch.cuda.synchronize(dev)
            res[name] = round(ev0.elapsed_time(ev1) / 1000.0 / reps, 4)
        res["ratio"] = round(res["time_domain_s"] / res["dft_s"], 3)
        out[f"nmech{nmech}"] = res
        e.close()
    return out


def multiscale_visco_workload(args, local):
    """The viscoelastic multiscale configuration on one GPU: L=3 with Q from 30 to
    100 (fixed), three frequency stages (10-30, 30-60, 60-100 Hz), L-BFGS on vp
    (NUMPAR 1, WEIGHT 1 0 0, BFGSNUM 3; the first update of a stage normalised,
    as the reference's would otherwise not move the model), the first two stages
    on a 2 m grid, then the model resampled to a 1 m grid for the third. The
    configuration's grids are 256x256x160 at 2 m and 512x512x320 at 1 m (NX x NZ
    horizontal, NY deep) with 64 shots and 10 iterations per stage; by default
    this runs it at half the linear size with 16 shots and --iterations-per-stage
    iterations; --ms-scale 1 --ms-shots-side 8 gives the configuration's grids and
    shots, and --ms-iterations caps the iterations run (the rest of the schedule is
    skipped). Shots go in HBM-sized batches. True model: four layers, three
    Gaussian blobs (+10 % vp, -40 % Q); start: the true model smoothed by a 15 m
    Gaussian. No free surface (precon_grad's damping types 0-2 zero the gradient
    with one). Timed by the host clock around the synchronous calls."""
    import torch
    from scipy.ndimage import gaussian_filter
    import ifosb
    from ifosb import stages as fst
    from ifosb import synth
    from ifosb.inversion import Inversion, Settings, Stage
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rng = np.random.default_rng(11)
    sc, nsh_side = args.ms_scale, args.ms_shots_side
    fw, fc, h_fine, fmin_q, fmax_q = 10, 50.0, 1.0, 10.0, 100.0
    fine = tuple(int(round(n * sc)) for n in (320, 512, 512))  # (NY, NX, NZ), y down
    its = args.iterations_per_stage
    cap_it = args.ms_iterations or 10 ** 9
    jj, ii, kk = np.meshgrid(*(np.arange(n, dtype=np.float32) for n in fine), indexing="ij")
    bounds = np.sort(rng.choice(np.arange(int(50 * sc), fine[0] - int(50 * sc)), 3, replace=False))
    layer = np.searchsorted(bounds, np.arange(fine[0]), side="right")
    vp_t = np.array([2500.0, 2900.0, 3200.0, 3500.0], np.float32)[layer][:, None, None] * np.ones(fine, np.float32)
    q_t = np.array([30.0, 50.0, 75.0, 100.0], np.float32)[layer][:, None, None] * np.ones(fine, np.float32)
    for _ in range(3):
        c = [rng.uniform(0.3 * n, 0.7 * n) for n in fine]
        g = np.exp(-((jj - c[0]) ** 2 + (ii - c[1]) ** 2 + (kk - c[2]) ** 2) / (2 * (28.0 * sc) ** 2))
        vp_t *= 1 + 0.1 * g
        q_t *= 1 - 0.4 * g
    del jj, ii, kk
    vp_t, q_t = vp_t.astype(np.float32), np.clip(q_t, 30.0, 100.0).astype(np.float32)
    true = (vp_t, (vp_t / np.float32(math.sqrt(3))).astype(np.float32), (1700 + 0.2 * vp_t).astype(np.float32))
    start = tuple(gaussian_filter(a.astype(np.float64), 15.0, mode="nearest").astype(np.float32) for a in true)
    nt_c, nt_f = int(round(2000 * sc)), int(round(4000 * sc))
    grids = [dict(h=2.0, dt=2e-4, nt=nt_c, stages=[Stage([10.0, 20.0, 30.0], its), Stage([30.0, 45.0, 60.0], its)]),
             dict(h=1.0, dt=1e-4, nt=nt_f, stages=[Stage([60.0, 80.0, 100.0], its)])]
    inner = lambda a: a[fw:-fw, fw:-fw, fw:-fw]  # noqa: E731
    err = lambda vp: float(np.linalg.norm(inner(vp) - inner(vp_t)) / np.linalg.norm(inner(vp_t)))  # noqa: E731
    cur = start
    hist, cells, t_total, t_obs, stage0, batches = [], 0, 0.0, 0.0, 0, []
    vp_err = {"start": err(start[0])}
    for gi, gd in enumerate(grids):
        if len(hist) >= cap_it:
            break
        s = gd["h"] / h_fine
        shape = tuple(int(n / s) for n in fine)
        ny, nx, nz = shape
        rs = (lambda a: fst.resample(a, (h_fine,) * 3, shape, (gd["h"],) * 3)) if s != 1 else (lambda a: a)
        mt, m0, q = [rs(a) for a in true], [rs(a) for a in cur], rs(q_t)
        p = ifosb.make_params(nx, ny, nz, dh=gd["h"], dt=gd["dt"], nt=gd["nt"], fdcoeff=2, free_surf=0, fw=fw,
                              nmech=3)
        xs = np.linspace(fw + 6, nx - fw - 6, nsh_side).round().astype(int)
        zs = np.linspace(fw + 6, nz - fw - 6, nsh_side).round().astype(int)
        shots = [(sp, ifosb.wavelet(p, 4, sp)) for sp in (synth._src(int(x), fw + 3, int(z), fc) for x in xs for z in zs)]
        rec = synth._grid_receivers(nx, nz, 16, fw + 2, fw + 3)
        cp = ifosb.cpml_coeff(p, 4000.0, fc)
        # batch size: the shots the free memory holds next to a 6 GB margin
        sizes = []
        for nb in (1, 2):
            e = ifosb.Engine(p, max_shots=nb, max_nf=3)
            sizes.append(e.device_bytes)
            e.close()
        per_shot = sizes[1] - sizes[0]
        free, _ = torch.cuda.mem_get_info(dev)
        B = max(1, min(len(shots), int((free - 6e9 - (sizes[0] - per_shot)) // per_shot)))
        batches.append(B)
        tau_q, fl_q = synth.tau_of_q(q, fmin_q, fmax_q, 3)
        mod = synth.q_moduli(p, *mt, tau_q, fl_q)
        e = ifosb.Engine(p, max_shots=B, max_nf=0)
        e.set_cpml(cp)
        e.set_receivers(rec)
        e.set_model(mod["rho"], mod["pi"], mod["u"], mod["taus"], mod["taup"], mod["eta"])
        t0 = time.perf_counter()
        obs = np.concatenate([e.forward(shots[i:i + B]) for i in range(0, len(shots), B)])
        t_obs += time.perf_counter() - t0
        e.close()
        mod0 = synth.q_moduli(p, *m0, tau_q, fl_q)
        ghost = [ifosb.ghost_wrap(mod0[k]) for k in ("rho", "pi", "u")]
        srcpos_m = np.array([[sp[0, 0] * gd["h"], sp[0, 1] * gd["h"], sp[0, 2] * gd["h"]] for sp, _ in shots], np.float32)
        cfg = Settings(teststep=0.02, damptype=2, lbfgs=True, numpar=1, bfgsnum=3, nshots_step=4,
                       max_batch=B, weight=(1.0, 0.0, 0.0), lbfgs_first_normalised=True)
        inv = Inversion(p, cp, rec, shots, obs, srcpos_m, *ghost, gd["stages"], cfg,
                        visco=(mod0["taus"], mod0["taup"], mod0["eta"]))
        iters = min(sum(st.itmax for st in gd["stages"]), cap_it - len(hist))
        ncell = nx * ny * nz
        for _ in range(iters):
            t0 = time.perf_counter()
            mis = inv.iterate()
            t_total += time.perf_counter() - t0
            cells += ncell * p.nt * (2 * len(shots) + 2 * cfg.nshots_step)
            hist.append({"grid": gi, "stage": stage0 + inv.stage_i, "misfit": mis, "t_s": round(t_total, 3),
                         "step": inv.hist.step[-1]})
        stage0 += len(gd["stages"])
        rho, pi, u = (a[1:-1, 1:-1, 1:-1].astype(np.float64) for a in inv.model)
        got = ((np.sqrt(pi / rho)).astype(np.float32), (np.sqrt(u / rho)).astype(np.float32), rho.astype(np.float32))
        inv.close()
        # the inversion's relaxed-modulus velocity back to the velocity at FL[1] (readmod's scaling)
        scale = np.sqrt(np.float32(1.0) + mod0["taup"] * np.float32(_sum_relax(fmin_q, fmax_q)))
        got = (got[0] * scale, got[1] * scale, got[2])
        cur = tuple(fst.resample(a, (gd["h"],) * 3, fine, (h_fine,) * 3) for a in got) if s != 1 else got
        vp_err[f"after_grid{gi}"] = err(cur[0])
    per_stage = {}
    for st in sorted({x["stage"] for x in hist}):
        m = [x["misfit"] for x in hist if x["stage"] == st]
        per_stage[f"stage{st}"] = {"first": m[0], "last": m[-1], "reduction": round(1 - m[-1] / m[0], 4)}
    g0 = tuple(int(n / 2) for n in fine)
    out = {
        "metric": METRIC, "value": round(cells / t_total / 1e9, 3), "unit": UNIT, "n_gpus": 1,
        "steps": len(hist), "warmup": 0, "ms_per_step": round(1000 * t_total / len(hist), 1),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"multiscale_visco: L=3 (Q 30-100) inversion, {g0[1]}x{g0[0]}x{g0[2]} (NX x NY x NZ, y "
                               f"deep) @ 2 m (NT={nt_c}, stages 10-30 and 30-60 Hz) then {fine[1]}x{fine[0]}x{fine[2]} "
                               f"@ 1 m (NT={nt_f}, stage 60-100 Hz), {its} L-BFGS iterations per stage"
                               + (f" (capped at {args.ms_iterations} in all)" if args.ms_iterations else "")
                               + f", {len(shots)} shots in HBM batches of {batches}, 256 receivers, 4 layers + 3 "
                                 "blobs, start smoothed by 15 m",
                   "scale": sc,
                   "timing": "host clock around synchronous calls; value counts the shot gradients and the "
                             "step-length test forwards; the observed-data forwards are not counted",
                   "full_configuration": "256x256x160 @ 2 m -> 512x512x320 @ 1 m, 64 shots, 10 iterations per stage"},
        "inversion": {"iterations": hist, "misfit_per_stage": per_stage, "vp_rel_error": vp_err,
                      "seconds": round(t_total, 2), "observed_data_seconds": round(t_obs, 2)},
    }
    print(json.dumps(out), flush=True)


def _sum_relax(fmin, fmax, nmech=3):
    """readmod's sum_l ws^2 t_l^2 / (1 + ws^2 t_l^2) per unit tau (tau = 1), ws = 2 pi FL[1]."""
    from ifosb import synth
    _, fl = synth.q_tau_fit(1.0, fmin, fmax, nmech)
    t = 1.0 / (2 * math.pi * fl.astype(np.float64))
    ws = 2 * math.pi * float(fl[0])
    return float((ws * ws * t * t / (1 + ws * ws * t * t)).sum())


def shot_gradient_comparison(torch, ifosb, synth, dev, stream, nt_override, nshots=4):
    """elastic128 shot-gradients/s: the plain path (one shot per launch sequence,
    kernel-by-kernel launches) against the batched path (all shots in one launch
    per kernel, time loop replayed from a CUDA graph)."""
    c = synth.case("elastic128", nt=nt_override)
    base = c["shots"][0]
    shots_sp = []
    for s in range(nshots):
        q = base.copy()
        q[0, 0] = 40 + 16 * s
        shots_sp.append(q)
    c["shots"] = shots_sp
    return _compare_batched(torch, ifosb, synth, dev, stream, c, nshots, f"elastic128, {nshots} shots")


def small_grid_comparison(torch, ifosb, synth, dev, stream, nt_override, nshots=32):
    """The same comparison where one shot cannot fill the GPU: 64^3 elastic cells
    (10-cell CPML, free surface), 32 shots on an 8x4 surface grid, nf = 2."""
    c = synth.small_case(nx=64, ny=64, nz=64, nt=nt_override or 800, fw=10, free_surf=1, nmech=0, seed=11,
                         nshots=nshots, ntr=16, finv=(300.0, 500.0))
    for s, sp in enumerate(c["shots"]):
        sp[0, 0] = 12 + 6 * (s % 8)
        sp[0, 2] = 16 + 10 * (s // 8)
    return _compare_batched(torch, ifosb, synth, dev, stream, c, nshots, f"elastic 64^3, {nshots} shots")


def _compare_batched(torch, ifosb, synth, dev, stream, c, nshots, label):
    p = c["params"]
    m, cp, shots = synth.build_inputs(c)
    mt, _, _ = synth.build_inputs(c, "true")
    same_model = all(np.array_equal(a, b) for a, b in zip(c["true"], c["start"]))

    def make(nb, mode):
        e = ifosb.Engine(p, max_shots=nb, max_nf=len(c["finv"]))
        e.set_stream(stream.cuda_stream)
        e.set_launch_mode(mode)
        e.set_cpml(cp)
        e.set_receivers(c["recpos"])
        e.set_frequencies(c["finv"], c["ntast"])
        e.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
        e.autotune(shots[:nb], steps=20)  # each path with its own best launch shape
        return e

    eb = make(nshots, 0)
    eb.set_model(mt["rho"], mt["pi"], mt["u"], mt["taus"], mt["taup"], mt["eta"])
    obs = eb.forward(shots)
    if same_model:  # observed data: a scaled copy, so the residual is not zero
        obs = (obs * np.float32(0.9)).astype(np.float32)
    eb.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
    eb.shot_gradient(shots, obs)  # warm-up (graph capture)
    eb.zero_gradient()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    eb.shot_gradient(shots, obs)
    torch.cuda.synchronize(dev)
    tb = time.perf_counter() - t0
    gb = eb.get_gradient()
    eb.close()
    per_shot, g1 = {}, None
    for mode, name in ((0, "graph"), (1, "plain")):
        e1 = make(1, mode)
        e1.set_model(m["rho"], m["pi"], m["u"], m["taus"], m["taup"], m["eta"])
        e1.shot_gradient(shots[:1], obs[:1])  # warm-up (graph capture in mode 0)
        e1.zero_gradient()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for s in range(nshots):
            e1.shot_gradient(shots[s:s + 1], obs[s:s + 1])
        torch.cuda.synchronize(dev)
        per_shot[name] = time.perf_counter() - t0
        g = e1.get_gradient()
        g1 = g if g1 is None else g1
        same_modes = np.array_equal(g, g1)
        e1.close()
    t1 = per_shot["graph"]
    return {"workload": f"{label}, NT={p.nt}, nf={len(c['finv'])}", "batched_per_s": round(nshots / tb, 4),
            "per_shot_per_s": round(nshots / t1, 4), "speedup": round(t1 / tb, 3),
            "per_shot_plain_launch_per_s": round(nshots / per_shot["plain"], 4),
            "speedup_vs_plain_launch": round(per_shot["plain"] / tb, 3),
            "gcells_batched": round(2 * nshots * p.nx * p.ny * p.nz * p.nt / tb / 1e9, 3),
            "gradients_bit_identical": bool(np.array_equal(gb, g1) and same_modes),
            "per_shot": "one shot per launch sequence, the time loop replayed from a CUDA graph (per_shot_per_s, "
                        "speedup) or launched kernel by kernel (plain_launch)",
            "timing": "host wall clock around synchronised calls"}


if __name__ == "__main__":
    main()
