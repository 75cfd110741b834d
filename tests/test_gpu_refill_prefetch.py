"""Prefetched refills of the persistent tracking kernel (imc_step_params.reserved bit 4: each
lane copies its next history's bank record into shared memory while it tracks the current
one) against the plain refill, one transport step from the same census with the same sources.

Only the assignment of histories to lanes differs, so every history takes the same path: the
event statistics agree exactly, the fixed-point deposition and escaped energy agree to FP64
round-off of the tally conversion (relative 1e-12), the intensity tally to FP64 atomic-order
round-off (relative L1 1e-12), and the census left in the bank is the same entry by entry.
Covered: RZ with the cell table in shared memory and in global memory (the full 60 x 210
crooked-pipe mesh), the slab with block tallies in shared memory, multigroup XY.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200 import problems
from radtranbook_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _run(geometry, e1, e2, vol, T, sig, cv, face, reflect, nt, nb, prefetch, cuda, ng=1, gedges=None,
         max_events=1_000_000, launch=None):
    eng = Engine(geometry, e1, e2, vol, seed=0x9F3A, n_groups=ng, group_edges=gedges)
    eng.launch.update(launch or {})
    eng.launch["prefetch"] = int(prefetch)
    dev = lambda a: None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=cuda)  # noqa: E731
    eng.init_census(dev(T), 20000)
    eng.transport(dev(T), dev(sig), dev(cv), None, 2, 0.01, 1.0, nt, nb, 0, [dev(f) for f in face], reflect,
                  max_events=max_events, rz_linear_source=geometry == "rz")
    stats, esc = eng.host_stats()
    bank = {k: eng.bank.view(k).cpu().numpy() for k in ("weight", "pos1", "dir1", "cell")}
    return stats, esc, eng.dep.cpu().numpy(), eng.si.cpu().numpy(), bank


def _same(a, b):
    st1, esc1, d1, s1, b1 = a
    st2, esc2, d2, s2, b2 = b
    np.testing.assert_array_equal(st1, st2)
    np.testing.assert_allclose(esc1, esc2, rtol=1e-12, atol=0)
    np.testing.assert_allclose(d1, d2, rtol=1e-12, atol=0)
    assert np.abs(s1 - s2).sum() <= 1e-12 * np.abs(s1).sum()
    np.testing.assert_array_equal(b1["weight"], b2["weight"])
    live = b1["weight"] > 0
    assert live.sum() > 1000
    for k in ("pos1", "dir1", "cell"):
        np.testing.assert_array_equal(b1[k][live], b2[k][live])
    assert st1[0] > 10000


def _rz_args(nr, nz, scale):
    p = problems.crooked_pipe(scale=scale, nr=nr, nz=nz)
    e1, e2 = p["edges1"], p["edges2"]
    vol = O.flat2d(np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :])
    T = O.flat2d(p["Tinit"])
    rc = 0.5 * (e1[:-1] + e1[1:])
    face = [None, None, np.where(rc < 0.5, 0.5, 0.0), None]
    return ("rz", e1, e2, vol, T, O.flat2d(p["sigma_host"](p["Tinit"])), O.flat2d(p["cv_host"](p["Tinit"])), face,
            p["reflect"], 20000, 10000)


@pytest.mark.parametrize("block", [128, 256])
def test_prefetch_matches_plain_refill_rz(cuda, block):
    args = _rz_args(30, 105, 0.02)
    launch = {"block_size": block, "blocks_per_sm": 4, "chunk": 512}
    _same(_run(*args, False, cuda, launch=launch), _run(*args, True, cuda, launch=launch))


def test_prefetch_matches_plain_refill_rz_full_mesh(cuda):
    # 12,600 cells: the cell table stays in global memory
    args = _rz_args(60, 210, 0.02)
    launch = {"block_size": 128, "blocks_per_sm": 8, "chunk": 8192}
    _same(_run(*args, False, cuda, launch=launch), _run(*args, True, cuda, launch=launch))


def test_prefetch_matches_plain_refill_slab(cuda):
    e1 = np.linspace(0.0, 0.2, 101)
    T = np.linspace(0.9, 0.02, 100)
    args = ("slab", e1, np.array([0.0, 1.0]), np.diff(e1), T, 300 * T ** -3.0, np.full(100, 0.3),
            [np.array([1.0]), None], (False, False), 20000, 20000)
    _same(_run(*args, False, cuda, max_events=0), _run(*args, True, cuda, max_events=0))


def test_prefetch_matches_plain_refill_multigroup(cuda):
    G = 6
    edges = np.logspace(-3, np.log10(20.0), G + 1)
    nu = 0.5 * (edges[:-1] + edges[1:])
    e1, e2 = np.linspace(0.0, 1.0, 13), np.linspace(0.0, 2.0, 21)
    vol = O.flat2d(np.diff(e1)[:, None] * np.diff(e2)[None, :])
    T = O.flat2d(np.outer(np.linspace(0.1, 1.0, 12), np.linspace(1.0, 0.3, 20)))
    sig = np.stack([np.clip(5.0 * n ** -3 * T ** -0.5, 1e-2, 1e5) for n in nu]).reshape(-1)
    args = ("xy", e1, e2, vol, T, sig, np.full(240, 0.2), [np.full(20, 1.0), None, None, None],
            (False, False, True, True), 20000, 10000)
    _same(_run(*args, False, cuda, ng=G, gedges=edges), _run(*args, True, cuda, ng=G, gedges=edges))
