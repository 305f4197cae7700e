"""The multi-GPU path of the benchmark is replicas only (one independent LP per rank, no collective on the data
path): its host logic, run as two gloo ranks on the CPU -- the whole-job time is the maximum over ranks, every rank
takes its own seed, and only rank 0 of the reference arm runs and prints."""
import datetime
import io
import os
import socket
import sys
import types
from contextlib import redirect_stdout
from pathlib import Path

import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.dist_max(1.5 + rank, True, device="cpu")  # rank r "took" 1.5 + r seconds
        buf = io.StringIO()
        with redirect_stdout(buf):
            if rank != 0:  # the reference arm does nothing on other ranks
                bench.reference_arm(types.SimpleNamespace(warmup=3, steps=1), rank, world)
        torch.distributed.barrier()
        out[rank] = (t, buf.getvalue())
    finally:
        torch.distributed.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        ps = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.5  # max over ranks
    assert res[1][1] == ""                # rank 1 of the reference arm printed nothing


def test_each_rank_solves_its_own_seed():
    sys.path.insert(0, str(ROOT))
    import bench
    import lpgen
    # the replica of rank r is the benchmark's planted LP with seed r (bench.make_lp(rank)): same shape, other data
    w = dict(bench.WORKLOAD)
    a = lpgen.planted(2000, 5000, 5, seed=0, zipf=w["zipf"], cap=w["cap"], floor=w["floor"])
    b = lpgen.planted(2000, 5000, 5, seed=1, zipf=w["zipf"], cap=w["cap"], floor=w["floor"])
    assert a.digest() != b.digest() and (a.m, a.n) == (b.m, b.n)
