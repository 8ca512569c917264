"""Shot sharding and the FP64 gradient all-reduce of ifosb.dist with two gloo
ranks on CPU (fake engines): every shot once, the same gradient and misfits on
both ranks as a single process computes, and failures that end every rank
with an error instead of a hang."""
import multiprocessing as mp
import socket

import numpy as np
import pytest

import dist_workers as dw
from ifosb.dist import ShotGradientError, batches, distributed_shot_gradient, shard


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(mode, world=2, timeout=90):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=dw.worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(world):
            r = q.get(timeout=timeout)
            out[r[0]] = r[1:]
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    return out


def test_shard_and_batches():
    assert shard(7, 2, 0) == [0, 2, 4, 6] and shard(7, 2, 1) == [1, 3, 5]
    assert sorted(shard(10, 3, 0) + shard(10, 3, 1) + shard(10, 3, 2)) == list(range(10))
    assert batches([0, 2, 4, 6], 3) == [[0, 2, 4], [6]]
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def test_single_process_matches_sum():
    shots, obs = dw.make_inputs()
    g, m = distributed_shot_gradient(dw.FakeEngine(), shots, obs, max_batch=3)
    ref = sum(dw.shot_contribution(i) for i in range(dw.NSHOTS))
    np.testing.assert_allclose(g, ref, rtol=1e-14, atol=1e-14)
    assert np.array_equal(m, [float(obs[i].sum()) for i in range(dw.NSHOTS)])


def test_two_ranks_allreduce_fp64():
    out = _run("ok")
    assert out[0][0] == "ok" and out[1][0] == "ok"
    (g0, m0, seen0), (g1, m1, seen1) = out[0][1:], out[1][1:]
    assert sorted(seen0 + seen1) == list(range(dw.NSHOTS)) and not set(seen0) & set(seen1)
    assert np.array_equal(g0, g1) and np.array_equal(m0, m1)
    ref = sum(dw.shot_contribution(i) for i in range(dw.NSHOTS))
    np.testing.assert_allclose(g0, ref, rtol=1e-14, atol=1e-14)
    _, obs = dw.make_inputs()
    assert np.array_equal(m0, [float(obs[i].sum()) for i in range(dw.NSHOTS)])


def test_failed_rank_ends_every_rank_with_an_error():
    out = _run("fail")
    assert out[0] == ("shot_error", [0], None, None)
    assert out[1] == ("shot_error", [0], None, None)


def test_rank_that_never_joins_ends_the_collective_with_an_error():
    out = _run("leave")
    assert out[1][0] == "left"
    assert out[0][0] == "collective_error"


def test_single_rank_failure_raises():
    shots, obs = dw.make_inputs()
    with pytest.raises(ShotGradientError):
        distributed_shot_gradient(dw.FakeEngine(fail_shot=2), shots, obs, max_batch=2)


def test_two_ranks_save_and_merge_seismograms(tmp_path):
    """saveseis across two ranks: each rank's SU file, then rank 0's merged file
    holding rank 0's traces followed by rank 1's (saveseis.c:86-229)."""
    from ifosb import io as fio
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=dw.seis_worker, args=(r, 2, port, str(tmp_path), q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(2):
            r = q.get(timeout=90)
            out[r[0]] = r[1:]
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    assert out[0][0] == "ok" and out[1][0] == "ok", out
    for c, name in enumerate(fio.COMPONENTS):
        merged = fio.read_seis(str(tmp_path / fio.seis_merged_file("seis", name, 0, 1, 1)), 7, 17)
        want = np.concatenate([out[0][1][c], out[1][1][c]])
        assert np.array_equal(merged, want)
        raw = open(tmp_path / fio.seis_merged_file("seis", name, 0, 1, 1), "rb").read()
        tracl = [int.from_bytes(raw[t * (240 + 68):t * (240 + 68) + 4], "little") for t in range(7)]
        assert tracl == [1, 2, 3, 4, 5, 6, 7]
