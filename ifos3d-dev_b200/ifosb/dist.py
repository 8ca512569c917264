"""Shot-parallel gradients over several GPUs (one process per GPU).

The reference runs its shots one after another on all ranks, each rank owning a
sub-domain (src/ifos3d.c:712 shot loop; gradient_F accumulates grad1..3 over the
shots, src/gradient_F.c:122-139; the misfit is summed with MPI_Allreduce,
src/ifos3d.c:864). Here the domain is whole on every GPU and the shots are
sharded instead: rank r takes shots r, r+W, r+2W, ... in batches, and the only
exchange is one FP64 all-reduce of the gradient and the per-shot misfits
(NCCL on GPUs, gloo on CPU). The optimiser then runs redundantly on every rank
from identical inputs, so no further collective is needed.

Every rank takes the same collective steps in the same order, on the error path
too: a status all-reduce comes first, and if any rank failed every rank raises
instead of entering the data all-reduce.
"""
from __future__ import annotations

import numpy as np


def shard(nshots: int, world: int, rank: int) -> list[int]:
    """Round-robin shot indices of one rank."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    return list(range(rank, nshots, world))


def batches(idx: list[int], max_batch: int) -> list[list[int]]:
    if max_batch < 1:
        raise ValueError("max_batch must be >= 1")
    return [idx[i:i + max_batch] for i in range(0, len(idx), max_batch)]


class ShotGradientError(RuntimeError):
    """Some rank failed its shots; carries the ranks that failed."""

    def __init__(self, failed_ranks, local_error=None):
        super().__init__(f"shot gradient failed on rank(s) {sorted(failed_ranks)}"
                         + (f": {local_error}" if local_error else ""))
        self.failed_ranks = sorted(failed_ranks)
        self.local_error = local_error


def _buffer(torch, dist, group, arr):
    t = torch.from_numpy(np.ascontiguousarray(arr, np.float64))
    if dist.get_backend(group) == "nccl":
        t = t.to(torch.device("cuda", torch.cuda.current_device()))
    return t


def distributed_shot_gradient(eng, shots, obs, max_batch: int, dist=None, group=None):
    """forward + residual + adjoint + gradient of all ``shots`` across the ranks.

    eng: this rank's engine (``ifosb.Engine`` or an object with the same
    ``zero_gradient``/``shot_gradient``/``get_gradient`` methods); shots: the
    full list of (srcpos, signals); obs: [nshots][3][ntr][ns] observed traces,
    host (numpy) or already resident on this rank's GPU (a float32 CUDA tensor).
    Returns (gradient FP64 [3][NY][NX][NZ] summed over all shots, misfit FP64
    [nshots]) — identical on every rank. With host traces the gradient comes back
    as a host array; with device traces it stays on the device (a CUDA tensor)
    and the exchange runs there."""
    world = dist.get_world_size(group) if dist is not None else 1
    rank = dist.get_rank(group) if dist is not None else 0
    nshots = len(shots)
    device = hasattr(obs, "is_cuda") and obs.is_cuda
    mis = np.zeros(nshots, np.float64)
    grad = None
    err = None
    try:
        eng.zero_gradient()
        for chunk in batches(shard(nshots, world, rank), max_batch):
            if device:
                contiguous = chunk == list(range(chunk[0], chunk[-1] + 1))
                o = obs[chunk[0]:chunk[-1] + 1] if contiguous else obs[chunk].contiguous()
            else:
                o = np.asarray(obs)[chunk]
            mis[chunk] = eng.shot_gradient([shots[i] for i in chunk], o)
        if device:
            import torch
            grad = torch.empty((3, eng.p.ny, eng.p.nx, eng.p.nz), dtype=torch.float64, device=obs.device)
            eng.get_gradient(fp64=True, out=grad)
        else:
            grad = np.asarray(eng.get_gradient(fp64=True), np.float64)
    except Exception as e:  # reported to every rank below, then raised everywhere
        err = e
    if dist is None or world == 1:
        if err is not None:
            raise ShotGradientError([rank], err) from err
        return grad, mis
    import torch

    status = np.zeros(world, np.float64)
    status[rank] = 1.0 if err is not None else 0.0
    st = _buffer(torch, dist, group, status)
    dist.all_reduce(st, op=dist.ReduceOp.SUM, group=group)
    failed = [r for r, v in enumerate(st.cpu().numpy()) if v != 0.0]
    if failed:
        raise ShotGradientError(failed, err) from err
    if device:
        # the gradient stays where it is: one all-reduce of it, one of the misfits
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
        mt = _buffer(torch, dist, group, mis)
        dist.all_reduce(mt, op=dist.ReduceOp.SUM, group=group)
        return grad, mt.cpu().numpy()
    buf = _buffer(torch, dist, group, np.concatenate([grad.ravel(), mis]))
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    return out[:grad.size].reshape(grad.shape), out[grad.size:].copy()
