"""The particle-partitioned step (radtranbook_b200.partition) on one GPU.

  - Id ranges: a bank split in two (a census twice over, so that both halves keep the
    unsplit bank's mean weight and hence its weight floor), each half tracked by its own
    engine with the Philox id offset of its position in the bank (what a rank of a partition
    does with its share), gives exactly the histories of the unsplit bank: the two ranks' event and
    escape counts add up to the unsplit step's exactly, and their summed deposition and
    intensity equal the unsplit tallies to FP64 round-off (relative 1e-12; each part's
    fixed-point deposition is exact to 2^-60 of its own weight total).
  - Two ranks in one process: the drop-in gray steps (slab and RZ) run as a 2-rank partition
    on two host threads whose all-reduce is a host-side sum behind a barrier (no kernel
    waits on another; the ranks' kernels run one after the other on the GPU).  Checked: both
    ranks hold the same material state after every step, the partitioned ledger closes to
    1e-12 every step, the ranks' sources together issue the unpartitioned step's boundary
    energy to FP32 weight rounding (relative 1e-6), and the census count is the sum of the
    ranks' combs to their shares of Nmax.
"""
import threading

import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200 import imc1d, imc2d, problems
from radtranbook_b200.engine import Engine

pytestmark = pytest.mark.gpu


def test_id_ranges_split_a_bank_exactly(cuda):
    p = problems.crooked_pipe(scale=0.02, nr=30, nz=105)
    e1, e2 = p["edges1"], p["edges2"]
    vol = O.flat2d(np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :])
    T = O.flat2d(p["Tinit"])
    dev = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=cuda)  # noqa: E731
    sig, cv = dev(O.flat2d(p["sigma_host"](p["Tinit"]))), dev(O.flat2d(p["cv_host"](p["Tinit"])))
    # the unsplit bank is one census twice over, so each half has the unsplit bank's mean
    # weight and therefore its weight floor (1e-10 of the mean weight, which wall histories reach)
    ic = Engine("rz", e1, e2, vol, seed=0x1D5)
    ic.init_census(dev(T), 60000)
    m = ic.bank.size
    census = {k: ic.bank.view(k).clone() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2", "cell")}

    def engine_with(copies, id_base):
        eng = Engine("rz", e1, e2, vol, seed=0x1D5)
        eng.bank.ensure(copies * m + 1024)
        for k, v in census.items():
            getattr(eng.bank, k)[: copies * m].copy_(v.repeat(copies))
        eng.bank.size = copies * m
        eng.id_base = id_base
        return eng

    full = engine_with(2, 0)
    parts = [engine_with(1, 0), engine_with(1, m)]  # the two halves with their id ranges
    out = []
    for eng in [full] + parts:
        # tracking only (no sources): the census of each part, Philox ids id_base + k
        eng.transport(dev(T), sig, cv, None, 4, 0.01, 1.0, 0, 0, 0, [None] * 4, p["reflect"], max_events=1_000_000)
        stats, esc = eng.host_stats()
        out.append((eng.dep.cpu().numpy(), eng.si.cpu().numpy(), stats, esc))
    (d, s, st, es), (d0, s0, st0, es0), (d1, s1, st1, es1) = out
    np.testing.assert_array_equal(st0 + st1, st)  # every event of every history, exactly
    np.testing.assert_allclose(es0[:4] + es1[:4], es[:4], rtol=1e-12, atol=1e-300)
    assert np.abs(d0 + d1 - d).sum() <= 1e-12 * np.abs(d).sum()
    assert np.abs(s0 + s1 - s).sum() <= 1e-12 * np.abs(s).sum()
    assert st[0] > 100000


class _ThreadGroup:
    """all_reduce across threads of one process: host-side sum behind a barrier."""

    def __init__(self, world: int):
        self.world = world
        self.barrier = threading.Barrier(world, timeout=120)
        self.bufs = [None] * world


class _ThreadDist:
    class ReduceOp:
        SUM = "sum"

    def __init__(self, group: _ThreadGroup, rank: int):
        self.g, self.rank = group, rank

    def get_rank(self):
        return self.rank

    def get_world_size(self):
        return self.g.world

    def all_reduce(self, t, op=None):
        self.g.bufs[self.rank] = t.detach().to("cpu", copy=True)
        self.g.barrier.wait()
        total = sum(self.g.bufs[1:], self.g.bufs[0].clone())
        self.g.barrier.wait()
        t.copy_(total.to(t.device))


def _run_ranks(world, fn):
    group = _ThreadGroup(world)
    res, err = [None] * world, []

    def body(r):
        try:
            res[r] = fn(_ThreadDist(group, r))
        except BaseException as ex:  # noqa: BLE001
            err.append(ex)
            group.barrier.abort()

    th = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    if err:
        raise err[0]
    assert all(r is not None for r in res)
    return res


def _slab_run(dist, steps=4):
    q = problems.marshak_slab(scale=0.5)
    st = imc1d.init_simulation(q["Ntarget"], q["Tinit"], q["Tr_init"], q["mesh"], q["eos_dev"], q["inv_eos_dev"],
                               seed=0xD157, _allreduce=dist)
    rec = []
    for _ in range(steps):
        st, info = imc1d.step(st, q["Ntarget"], q["Nboundary"], 0, q["Nmax"], q["T_boundary"], q["dt"], q["mesh"],
                              q["sigma_dev"], q["inv_eos_dev"], q["cv_dev"], q["source"], _allreduce=dist)
        rec.append((info["ledger"]["relative_closure"], info["boundary_emission"], info["N_particles"],
                    info["total_energy"]))
    return st.temperature.copy(), rec, st._engine.bank.size


def _rz_run(dist, steps=3):
    p = problems.crooked_pipe(scale=0.02, nr=30, nz=105)
    st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                               p["inv_eos_dev"], geometry="rz", seed=0xD158, _allreduce=dist)
    rec = []
    for _ in range(steps):
        st, info = imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], p["edges1"],
                              p["edges2"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"],
                              reflect=p["reflect"], geometry="rz", boundary_source_func=p["boundary_source_func"],
                              _allreduce=dist)
        rec.append((info["ledger"]["relative_closure"], info["boundary_emission"], info["N_particles"],
                    info["total_energy"]))
    return st.temperature.copy(), rec, st._engine.bank.size


@pytest.mark.parametrize("run", [_slab_run, _rz_run], ids=["slab", "rz"])
def test_two_rank_partition_in_one_process(cuda, run):
    single_T, single, _ = run(None)
    ranks = _run_ranks(2, run)
    (T0, rec0, n0), (T1, rec1, n1) = ranks
    np.testing.assert_array_equal(T0, T1)  # both ranks apply the same summed tallies
    for (c0, b0, N0, E0), (c1, b1, N1, E1), (_, b, _, E) in zip(rec0, rec1, single):
        assert abs(c0) < 1e-12 and abs(c1) < 1e-12, (c0, c1)
        assert b0 == b1 and N0 == N1  # the summed ledger terms and census count, on every rank
        np.testing.assert_allclose(b0, b, rtol=1e-6)  # the ranks' sources carry the energy once
    assert N0 == n0 + n1
    # the same problem (independent histories): the partitioned run's temperatures follow the
    # single run's within Monte Carlo noise
    hot = single_T > 2 * single_T.min()
    assert np.abs(T0[hot] - single_T[hot]).mean() < 0.1 * single_T[hot].mean()
