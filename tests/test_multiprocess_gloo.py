"""The partitioned step's host logic with two processes on the CPU (torch.distributed, gloo):
each rank's particle share and Philox id range, the per-step SUM of the per-cell tallies, the
SUM of the ledger terms of a step summary, the check that a state belongs to the partition,
and bench.py's whole-job timing (slowest rank, summed counts)."""
import os
import socket
import types

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


def _fake_summary(rank: int):
    """An object with the imc_step_summary fields summary_totals reads."""
    return types.SimpleNamespace(comb_after=1.0 + rank, comb_before=2.0 + rank, e_side=[0.5, 0.0, 0.25 * rank, 0.0],
                                 escaped=[0.1, 0.2, 0.0, rank], source_emission=3.0, emission_total=4.0 + rank,
                                 weight_sum=10.0 * (rank + 1), n_bank=100 + rank,
                                 stats=[7 + rank, 1, 2, 3, 0, 0, 0, 0, rank])


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from radtranbook_b200 import partition as P
        from radtranbook_b200._gray import check_partition

        rng = np.random.default_rng(100 + rank)
        dep = torch.as_tensor(rng.random(37))
        si = torch.as_tensor(rng.random((4, 5)))
        P.sum_tensors(dist, [dep, si])
        vals = P.sum_scalars(dist, [1.0 + rank, 10.0 * rank, -2.0], torch.device("cpu"))
        tot = P.summary_totals(dist, _fake_summary(rank), 50 + rank, torch.device("cpu"))
        eng = types.SimpleNamespace(rank=rank, world=world)
        check_partition(eng, dist)
        wrong = types.SimpleNamespace(rank=0, world=1)
        try:
            check_partition(wrong, dist)
            mismatch = False
        except ValueError:
            mismatch = True
        tmax, totals = bench.max_time_and_totals(dist, 3.0 + rank, [100 + rank, 7], torch.device("cpu"))
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), dep=dep.numpy(), si=si.numpy(), vals=np.array(vals),
                 rad=tot["rad"], e_side=tot["e_side"], escaped=tot["escaped"], stats=tot["stats"],
                 n_particles=tot["n_particles"], n_bank=tot["n_bank"], weight_sum=tot["weight_sum"],
                 local=np.array([P.local_count(n, rank, world) for n in (0, 1, 7, 2_000_001)]),
                 id_base=P.id_base(rank, world), key=np.uint64(P.rank_key(0x5EED0001, rank)),
                 mismatch=mismatch, tmax=tmax, totals=np.array(totals))
    finally:
        dist.destroy_process_group()


def test_partition_host_logic_two_ranks(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
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
    ref_dep = np.sum([np.random.default_rng(100 + k).random(37) for k in range(world)], axis=0)
    g = [np.random.default_rng(100 + k) for k in range(world)]
    for x in g:
        x.random(37)
    ref_si = np.sum([x.random((4, 5)) for x in g], axis=0)
    for k in range(world):
        # the per-cell tallies and the ledger terms are summed, and every rank holds the sums
        np.testing.assert_allclose(r[k]["dep"], ref_dep, rtol=1e-15)
        np.testing.assert_allclose(r[k]["si"], ref_si, rtol=1e-15)
        np.testing.assert_allclose(r[k]["vals"], [3.0, 10.0, -4.0])
        assert float(r[k]["rad"]) == 3.0 and int(r[k]["n_particles"]) == 101 and int(r[k]["n_bank"]) == 201
        np.testing.assert_allclose(r[k]["e_side"], [1.0, 0.0, 0.25, 0.0])
        np.testing.assert_allclose(r[k]["escaped"], [0.2, 0.4, 0.0, 1.0])
        np.testing.assert_array_equal(r[k]["stats"], [15, 2, 4, 6, 0, 0, 0, 0, 1])
        assert float(r[k]["weight_sum"]) == 30.0
        assert bool(r[k]["mismatch"])  # a state initialised for another partition is refused
        assert float(r[k]["tmax"]) == 4.0
        np.testing.assert_allclose(r[k]["totals"], [201.0, 14.0])
    # the ranks' shares add up to the totals; id ranges and keys are disjoint
    np.testing.assert_array_equal(r[0]["local"] + r[1]["local"], [0, 1, 7, 2_000_001])
    assert int(r[0]["id_base"]) == 0 and int(r[1]["id_base"]) == 1 << 31
    assert int(r[0]["key"]) == 0x5EED0001 and int(r[1]["key"]) != 0x5EED0001
