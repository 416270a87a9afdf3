"""The replica runner (replicas.sharded_sweep) driving real sweeps: each rank
runs SweepPlan.run on its shard of the frequency points and the results are
gathered over a gloo process group.  World 1 runs in this process; world 2
runs as two spawned processes that share cuda:0 (the replicas never wait on
each other on the device: each rank sweeps independently and only the host
gather connects them).  Both must return exactly the single-process sweep."""
import importlib
import os
import socket

import numpy as np
import pytest

import efie_oracle as eo
from conftest import pkg, small_design

pytestmark = pytest.mark.gpu

PKG = "matlab-cuda-efief-vs-cpu_b200"


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _plan(m, p, d):
    r = p["rwg"]
    return m.SweepPlan(p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"],
                       r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], p["prepack"], d.mu, d.eps, p["patchEdge"],
                       p["groundEdge"], d.V0, p["spread"], d.Z0, opts=m.sweep_opts(solver="fp64"))


def _freqs():
    return np.linspace(2.0e9, 3.0e9, 7)


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for d_ in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        if d_ not in sys.path:
            sys.path.insert(0, d_)
    import torch.distributed as dist
    import efie_oracle as eo_
    from conftest import small_design as sd
    m = importlib.import_module(PKG)
    rep = importlib.import_module(PKG + ".replicas")
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        d = sd("grid")
        p = eo_.build_problem(d)
        plan = _plan(m, p, d)
        Zin, S11 = rep.sharded_sweep(lambda f: plan.run(f), _freqs(), rank, world)
        plan.close()
        q.put((rank, Zin, S11))
    finally:
        dist.destroy_process_group()


def test_sharded_sweep_matches_single_process_sweep():
    import torch.distributed as dist
    import torch.multiprocessing as mp
    m = pkg()
    rep = importlib.import_module(PKG + ".replicas")
    d = small_design("grid")
    p = eo.build_problem(d)
    plan = _plan(m, p, d)
    Z1, S1 = plan.run(_freqs())
    # world 1, in this process
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % _port(), rank=0, world_size=1)
    try:
        Zw, Sw = rep.sharded_sweep(lambda f: plan.run(f), _freqs(), 0, 1)
    finally:
        dist.destroy_process_group()
    plan.close()
    assert np.array_equal(Zw, Z1) and np.array_equal(Sw, S1)
    # world 2, two spawned processes on cuda:0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=300) for _ in procs]
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    for _, Zr, Sr in res:
        assert np.array_equal(Zr, Z1) and np.array_equal(Sr, S1)
