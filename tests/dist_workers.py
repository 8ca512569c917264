"""Worker processes for the gloo (CPU) tests of ifosb.dist — a fake engine
stands in for the GPU so the host logic of shot sharding, the FP64 all-reduce
and the failure agreement run with world_size 2 on CPU."""
import datetime
import os

import numpy as np

SHAPE = (3, 4, 5, 6)
NSHOTS = 7


def shot_contribution(i):
    return np.random.default_rng(100 + i).standard_normal(SHAPE)


def make_inputs():
    shots = [(np.array([[i, 1, 1, 0, 0, 1, 1]], np.float32), None) for i in range(NSHOTS)]
    obs = np.stack([np.full((3, 2, 5), float(i + 1), np.float32) for i in range(NSHOTS)])
    return shots, obs


class FakeEngine:
    """zero_gradient / shot_gradient / get_gradient with known per-shot results."""

    def __init__(self, fail_shot=None):
        self.g = np.zeros(SHAPE)
        self.seen = []
        self.fail_shot = fail_shot

    def zero_gradient(self):
        self.g[...] = 0.0

    def shot_gradient(self, shots, obs):
        mis = []
        for (sp, _), o in zip(shots, obs):
            i = int(sp[0, 0])
            if i == self.fail_shot:
                raise RuntimeError(f"shot {i} unstable")
            self.seen.append(i)
            self.g += shot_contribution(i)
            mis.append(float(np.sum(o, dtype=np.float64)))
        return np.array(mis)

    def get_gradient(self, fp64=False):
        return self.g.copy()


def worker(rank, world, port, mode, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    from ifosb.dist import ShotGradientError, distributed_shot_gradient

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    shots, obs = make_inputs()
    fail = 4 if (mode == "fail" and rank == 0) else None  # shot 4 belongs to rank 0
    eng = FakeEngine(fail)
    try:
        if mode == "leave" and rank == 1:
            q.put((rank, "left", None, None, None))
            return  # never takes part in the collectives
        g, m = distributed_shot_gradient(eng, shots, obs, max_batch=2, dist=dist)
        q.put((rank, "ok", g, m, eng.seen))
    except ShotGradientError as e:
        q.put((rank, "shot_error", e.failed_ranks, None, None))
    except Exception as e:  # a collective that ended with an error
        q.put((rank, "collective_error", type(e).__name__, None, None))
    finally:
        if not (mode == "leave" and rank == 1):
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def seis_worker(rank, world, port, wdir, q):
    """Two ranks write their receivers' SU files through ifosb.io.save_seis with a
    gloo barrier between the writes and rank 0's merge."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    from ifosb import io as fio

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        os.chdir(wdir)
        ntr, ns = 3 + rank, 17
        rng = np.random.default_rng(100 + rank)
        secs = rng.standard_normal((3, ntr, ns)).astype(np.float32)
        rec = np.stack([np.arange(ntr) + 5 * rank + 1, np.ones(ntr, int), np.full(ntr, 4)], 1).astype(np.int32)
        tn = (np.arange(ntr) + 1 + 3 * rank).astype(np.int32)  # global trace numbers
        fio.save_seis("seis", secs, rec, np.array([10.0, 2.0, 5.0], np.float32), ishot=1, iteration=0, dx=1.0,
                      dy=1.0, dz=1.0, ndt=1, dt=1e-4, trace_no=tn, rank=rank, nranks=world, barrier=dist.barrier)
        q.put((rank, "ok", secs))
    except Exception as e:
        q.put((rank, "error", repr(e)))
    finally:
        dist.destroy_process_group()
