"""Edge cases of the CUDA path against the FP64 oracle (same Philox streams).

Tolerances as tests/test_gpu_parity.py: counts exact, per-cell tallies relative L1 <= 2e-4,
FP64 ledger closure <= 1e-12 per step.

  - an empty step (no census, no sources) and an empty comb;
  - dead entries (zero weight) in the bank are skipped, as the oracle skips them;
  - the 2-D events-per-history cap (IMC/IMC2D.py:974-977): capped histories stay in census,
    counted like the oracle's;
  - a one-cell mesh;
  - a closed box (every face reflecting): nothing escapes and the ledger closes;
  - a non-finite opacity raises AssertionError (the reference's material checks raise it);
    the plan turns every emission count to zero for it, so nothing is sampled from it.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200 import _lib, imc2d
from radtranbook_b200.engine import Engine

pytestmark = pytest.mark.gpu

SEED = 0x5EED00E0


def _xy(nx, ny, L=1.0):
    e1 = np.linspace(0.0, L, nx + 1)
    e2 = np.linspace(0.0, L, ny + 1)
    return e1, e2, O.flat2d(np.diff(e1)[:, None] * np.diff(e2)[None, :])


def _dev(a, cuda):
    return None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64), device=cuda)


def _l1(a, b):
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def test_empty_step_and_empty_comb(cuda):
    e1, e2, vol = _xy(8, 8)
    eng = Engine("xy", e1, e2, vol, seed=SEED)
    nc = 64
    T = np.full(nc, 0.1)
    res = eng.transport(_dev(T, cuda), _dev(np.full(nc, 5.0), cuda), _dev(np.full(nc, 0.1), cuda), None, 0, 0.01, 1.0,
                        0, 0, 0, [None] * 4, (False,) * 4)
    assert res.report.n_transported == 0
    stats, esc = eng.host_stats()
    assert int(stats[_lib.STAT_EVENTS]) == 0 and esc.sum() == 0.0
    assert float(eng.dep.abs().sum()) == 0.0 and float(eng.si.abs().sum()) == 0.0
    rep = eng.comb(1000, 1)
    assert rep.n_out == 0 and eng.bank.size == 0


def test_dead_entries_are_skipped(cuda):
    e1, e2, vol = _xy(12, 12)
    nc = 144
    eng = Engine("xy", e1, e2, vol, seed=SEED)
    orc = O.Oracle("xy", e1, e2, vol, SEED)
    T = O.flat2d(np.outer(np.linspace(0.6, 0.1, 12), np.ones(12)))
    eng.init_census(_dev(T, cuda), 6000)
    w = eng.bank.view("weight")
    w[::3] = 0.0  # every third entry dead
    b = eng.bank
    orc.set_bank(*(b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")),
                 b.view("cell").cpu().numpy())
    sig, cv = 20.0 / T, np.full(nc, 0.1)
    face = [np.full(12, 1.0), None, None, None]
    refl = (False, False, True, True)
    res = eng.transport(_dev(T, cuda), _dev(sig, cuda), _dev(cv, cuda), None, 2, 0.01, 1.0, 2000, 2000, 0,
                        [_dev(f, cuda) for f in face], refl, max_events=1_000_000)
    ro = orc.transport(T, sig, cv, None, 2, 0.01, 1.0, 2000, 2000, 0, face, refl, max_events=1_000_000)
    assert res.report.n_transported == ro["n_transported"]
    assert _l1(eng.dep.cpu().numpy(), ro["dep"]) < 2e-4
    stats, _ = eng.host_stats()
    np.testing.assert_allclose(stats[_lib.STAT_EVENTS], ro["stats"][_lib.STAT_EVENTS], rtol=1e-3)


def test_event_cap_matches_oracle(cuda):
    e1, e2, vol = _xy(16, 16)
    nc = 256
    eng = Engine("xy", e1, e2, vol, seed=SEED)
    orc = O.Oracle("xy", e1, e2, vol, SEED)
    T = np.full(nc, 0.3)
    eng.init_census(_dev(T, cuda), 4000)
    b = eng.bank
    orc.set_bank(*(b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")),
                 b.view("cell").cpu().numpy())
    sig, cv = np.full(nc, 50.0), np.full(nc, 10.0)  # optically thick, weakly coupled: many scatters
    refl = (True,) * 4
    res = eng.transport(_dev(T, cuda), _dev(sig, cuda), _dev(cv, cuda), None, 1, 0.01, 1.0, 0, 0, 0, [None] * 4, refl,
                        max_events=5)
    ro = orc.transport(T, sig, cv, None, 1, 0.01, 1.0, 0, 0, 0, [None] * 4, refl, max_events=5)
    stats, _ = eng.host_stats()
    cap_o = ro["stats"][_lib.STAT_CAP]
    assert cap_o > 1000
    assert abs(int(stats[_lib.STAT_CAP]) - int(cap_o)) <= max(2e-3 * cap_o, 3)
    assert res.report.n_transported == ro["n_transported"]
    # capped histories keep their weight in census: the weight sum equals the oracle's
    wsum = float(eng.bank.view("weight").double().sum())
    np.testing.assert_allclose(wsum, orc.get_bank()["weight"].sum(), rtol=2e-4)


def test_one_cell_mesh(cuda):
    e1, e2, vol = _xy(1, 1, L=0.2)
    eng = Engine("xy", e1, e2, vol, seed=SEED)
    orc = O.Oracle("xy", e1, e2, vol, SEED)
    T = np.array([0.5])
    eng.init_census(_dev(T, cuda), 3000)
    b = eng.bank
    orc.set_bank(*(b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")),
                 b.view("cell").cpu().numpy())
    face = [np.array([1.0]), None, None, None]
    res = eng.transport(_dev(T, cuda), _dev(np.array([8.0]), cuda), _dev(np.array([0.1]), cuda), None, 4, 0.005, 1.0,
                        2000, 1000, 0, [_dev(f, cuda) for f in face], (False,) * 4, max_events=1_000_000)
    ro = orc.transport(T, np.array([8.0]), np.array([0.1]), None, 4, 0.005, 1.0, 2000, 1000, 0, face, (False,) * 4,
                       max_events=1_000_000)
    assert res.report.n_transported == ro["n_transported"]
    np.testing.assert_allclose(eng.dep.cpu().numpy(), ro["dep"], rtol=2e-4)
    np.testing.assert_allclose(eng.si.cpu().numpy(), ro["si"], rtol=2e-4)
    _, esc = eng.host_stats()
    np.testing.assert_allclose(esc[:4], ro["escaped"][:4], rtol=2e-4, atol=1e-9 * esc.sum())


def test_closed_box_keeps_everything(cuda):
    e1, e2 = np.linspace(0, 1, 11), np.linspace(0, 1, 11)
    T0 = np.outer(np.linspace(0.8, 0.2, 10), np.ones(10))
    st = imc2d.init_simulation(5000, T0, T0, e1, e2, lambda T: 0.1 * T, lambda u: u / 0.1, geometry="xy", seed=SEED)
    for _ in range(4):
        st, info = imc2d.step(st, 5000, 0, 0, 20000, (0.0,) * 4, 0.005, e1, e2, lambda T: 10.0 + 0 * T,
                              lambda u: u / 0.1, lambda T: 0.1 + 0 * T, np.zeros((10, 10)), reflect=(True,) * 4)
        assert info["boundary_loss"] == 0.0 and info["boundary_emission"] == 0.0
        assert abs(info["ledger"]["relative_closure"]) < 1e-12
        assert info["profiling"]["transport_events"]["reflections"] > 0


def test_nonfinite_opacity_raises(cuda):
    e1, e2 = np.linspace(0, 1, 5), np.linspace(0, 1, 5)
    T0 = np.full((4, 4), 0.1)
    st = imc2d.init_simulation(1000, T0, T0, e1, e2, lambda T: 0.1 * T, lambda u: u / 0.1, geometry="xy", seed=SEED)

    def sigma(T):
        s = 10.0 + 0 * T
        s[1, 1] = np.nan
        return s

    with pytest.raises(AssertionError):
        imc2d.step(st, 1000, 1000, 0, 4000, (1.0, 0.0, 0.0, 0.0), 0.01, e1, e2, sigma, lambda u: u / 0.1,
                   lambda T: 0.1 + 0 * T, np.zeros((4, 4)))
