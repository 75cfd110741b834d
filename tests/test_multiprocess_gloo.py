"""The replica path's host logic with two processes on the CPU (torch.distributed, gloo):
the per-step tally average every rank applies before its material update, the replica mean
of the ledger terms, and bench.py's whole-job timing (slowest rank, summed counts)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from radtranbook_b200._gray import allreduce_mean, replica_mean

        rng = np.random.default_rng(100 + rank)
        dep = torch.as_tensor(rng.random(37))
        si = torch.as_tensor(rng.random((4, 5)))
        allreduce_mean(dist, [dep, si])
        vals = replica_mean(dist, [1.0 + rank, 10.0 * rank, -2.0], torch.device("cpu"))
        tmax, totals = bench.max_time_and_totals(dist, 3.0 + rank, [100 + rank, 7], torch.device("cpu"))
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), dep=dep.numpy(), si=si.numpy(), vals=np.array(vals),
                 tmax=tmax, totals=np.array(totals))
    finally:
        dist.destroy_process_group()


def test_replica_reductions_two_ranks(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, _free_port_cached(), str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a gloo rank did not finish")
        assert p.exitcode == 0
    r = [np.load(tmp_path / f"r{k}.npz") for k in range(world)]
    ref_dep = np.mean([np.random.default_rng(100 + k).random(37) for k in range(world)], axis=0)
    g = [np.random.default_rng(100 + k) for k in range(world)]
    for x in g:
        x.random(37)
    ref_si = np.mean([x.random((4, 5)) for x in g], axis=0)
    for k in range(world):
        np.testing.assert_allclose(r[k]["dep"], ref_dep, rtol=1e-15)
        np.testing.assert_allclose(r[k]["si"], ref_si, rtol=1e-15)
        np.testing.assert_allclose(r[k]["vals"], [1.5, 5.0, -2.0])
        assert float(r[k]["tmax"]) == 4.0
        np.testing.assert_allclose(r[k]["totals"], [201.0, 14.0])


_PORT = []


def _free_port_cached() -> int:
    if not _PORT:
        _PORT.append(_free_port())
    return _PORT[0]
