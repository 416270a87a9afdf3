"""Multi-GPU replica logic on CPU: world_size-2 gloo process groups run the
sharding and gather of a frequency sweep with a host-side stand-in for the
per-point solve (the oracle's port formula on a fixed complex function), a
rank that fails, and the bench's design sharding."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

PKG = "matlab-cuda-efief-vs-cpu_b200"


def _rep():
    return importlib.import_module(PKG + ".replicas")


def test_shard_covers_every_item_once():
    rep = _rep()
    for n in (0, 1, 7, 101):
        for world in (1, 2, 3, 8):
            for mode in ("strided", "block"):
                idx = np.concatenate([rep.shard(n, r, world, mode) for r in range(world)])
                assert np.array_equal(np.sort(idx), np.arange(n))
                sizes = [rep.shard(n, r, world, mode).size for r in range(world)]
                assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        rep.shard(5, 2, 2)


def _fake_run(f):
    # a smooth complex "Zin(f)" and its S11; the same on every rank
    z = 30.0 + 20.0j * np.sin(f / 1e9) + 5.0 * (f / 1e9)
    return z, (z - 50.0) / (z + 50.0)


def _worker(rank, world, port, mode, fail_rank, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rep = _rep()
    freqs = np.linspace(2e9, 3e9, 37)

    def run(fr):
        if rank == fail_rank:
            raise RuntimeError("solver failed on this rank")
        return _fake_run(fr)

    try:
        Zin, S11 = rep.sharded_sweep(run, freqs, rank, world, mode=mode)
        q.put((rank, "ok", Zin, S11))
    except RuntimeError as e:
        q.put((rank, "error", str(e), None))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run(world, mode, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, fail_rank, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


@pytest.mark.parametrize("mode", ["strided", "block"])
def test_sharded_sweep_matches_serial(mode):
    out = _run(2, mode)
    Zs, Ss = _fake_run(np.linspace(2e9, 3e9, 37))
    for rank, status, Zin, S11 in out:
        assert status == "ok"
        assert np.array_equal(Zin, Zs) and np.array_equal(S11, Ss)


def test_failed_rank_is_reported_to_every_rank():
    out = _run(2, "strided", fail_rank=1)
    for rank, status, msg, _ in out:
        assert status == "error" and "rank 1" in msg


def test_bench_family_sharding_is_a_partition():
    # run_family gives step i of rank r the design (i * world + r) mod n
    n, world, steps = 64, 2, 32
    got = sorted((i * world + r) % n for r in range(world) for i in range(steps))
    assert got == list(range(n))
