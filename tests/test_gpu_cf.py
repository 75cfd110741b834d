"""GPU parity of the Carter-Forest path (IMC/IMC1D_CarterForest.py, IMC/IMC2D_CarterForest.py)
against the FP64 oracle, and of the drop-in steps against the reference's own statistics.

Tolerances:
  - one step from an identical bank: source counts exact, issued emission energy per cell
    to FP32 weight rounding, per-cell deposition and scalar intensity relative L1 <= 5e-4,
    event, capture and re-emission counts within 2e-3 relative or 3 (a history whose event
    order flips on an FP32 near-tie diverges from the oracle's);
  - drop-in steps: FP64 energy closure <= 1e-12 per step;
  - 32-seed means of T (and Tr in xy) within the combined standard errors of the reference
    runs (tests/golden/stats_cf_*.npz).
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200 import _lib
from radtranbook_b200.engine import Engine
from tests import stat_problems as SP

pytestmark = pytest.mark.gpu

SEED = 0x5EED00CF
G = os.path.join(os.path.dirname(__file__), "golden")


def _setup(geometry):
    if geometry in ("slab", "spherical"):
        e1 = np.linspace(0.0, 0.3, 61)
        e2 = np.array([0.0, 1.0])
        vol = np.diff(e1) if geometry == "slab" else 4 / 3 * np.pi * np.diff(e1 ** 3)
        T = np.linspace(0.8, 0.05, 60)
        src = np.zeros(60)
        src[10:20] = 3.0
        face = [np.array([1.0]), None] if geometry == "slab" else [None, np.array([1.0])]
        reflect = (False, False) if geometry == "slab" else (True, False)
        me = 0
    else:
        e1 = np.linspace(0.0, 0.6, 13)
        e2 = np.linspace(0.0, 1.2, 21)
        v = np.diff(e1)[:, None] * np.diff(e2)[None, :] if geometry == "xy" else \
            np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :]
        vol = O.flat2d(v)
        T = O.flat2d(np.outer(np.linspace(0.8, 0.05, 12), np.linspace(1.0, 0.5, 20)))
        src = np.zeros(240)
        src[50:60] = 3.0
        face = [np.full(20, 1.0), None, None, None] if geometry == "xy" else [None, None, np.full(12, 1.0), None]
        reflect = (False, False, True, True) if geometry == "xy" else (True, False, False, False)
        me = 1_000_000
    sigma = 4.0 * np.maximum(T, 0.02) ** -2
    cv = np.full(len(T), 0.1)
    return e1, e2, vol, T, sigma, cv, src, face, reflect, me


@pytest.mark.parametrize("geometry", ["slab", "spherical", "xy", "rz"])
def test_cf_transport_matches_oracle(cuda, geometry):
    e1, e2, vol, T, sigma, cv, src, face, reflect, me = _setup(geometry)
    eng = Engine(geometry, e1, e2, vol, seed=SEED)
    orc = O.Oracle(geometry, e1, e2, vol, SEED)
    dev = lambda a: None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64), device=cuda)  # noqa: E731
    eng.init_census(dev(T), 4000)
    b = eng.bank
    orc.set_bank(*(b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")),
                 b.view("cell").cpu().numpy())
    res = eng.transport(dev(T), dev(sigma), dev(cv), dev(src), 2, 0.004, 1.0, 4000, 3000, 2000,
                        [dev(f) for f in face], reflect, max_events=me, method=_lib.METHOD_CARTER_FOREST)
    ro = orc.transport(T, sigma, cv, src, 2, 0.004, 1.0, 4000, 3000, 2000, face, reflect, max_events=me,
                       method="cf")
    rep = res.report
    assert rep.n_transported == ro["n_transported"]
    np.testing.assert_allclose(rep.boundary_emission, ro["boundary_emission"], rtol=1e-7)
    np.testing.assert_allclose(rep.source_emission, ro["source_emission"], rtol=1e-6)
    np.testing.assert_allclose(eng.emitted.cpu().numpy(), ro["emitted"], rtol=1e-7, atol=1e-300)
    np.testing.assert_allclose(eng.sigma_a.cpu().numpy(), sigma, rtol=0)  # true opacity, no Fleck factor
    l1 = lambda a, b: np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)  # noqa: E731
    dep, si = eng.dep.cpu().numpy(), eng.si.cpu().numpy()
    assert l1(dep, ro["dep"]) < 5e-4, l1(dep, ro["dep"])
    assert l1(si, ro["si"]) < 5e-4, l1(si, ro["si"])
    stats, esc = eng.host_stats()
    for k in (_lib.STAT_EVENTS, _lib.STAT_CAPTURE, _lib.STAT_SCATTER):
        assert abs(int(stats[k]) - int(ro["stats"][k])) <= max(2e-3 * ro["stats"][k], 3), (k, stats[k], ro["stats"][k])
    assert stats[_lib.STAT_CAPTURE] > 100 and stats[_lib.STAT_SCATTER] > 100
    tot_in = ro["boundary_emission"] + ro["source_emission"] + float(np.sum(ro["emitted"]))
    assert abs(esc[:4].sum() - ro["escaped"].sum()) <= 5e-4 * tot_in


@pytest.mark.parametrize("geometry", ["slab", "spherical", "xy", "rz"])
def test_cf_dropin_ledger_closes(cuda, geometry):
    from radtranbook_b200 import imc1d_cf, imc2d_cf

    cv = 0.1
    sig = lambda T: 4.0 * np.maximum(T, 0.02) ** -2  # noqa: E731
    if geometry in ("slab", "spherical"):
        e = np.linspace(0.0, 0.3, 61)
        mesh = np.stack([e[:-1], e[1:]], axis=1)
        st = imc1d_cf.init_simulation(3000, np.full(60, 0.05), np.full(60, 0.05), mesh, lambda T: cv * T,
                                      lambda u: u / cv, geometry=geometry)
        src = np.zeros(60)
        src[5:10] = 2.0
        for _ in range(4):
            st, info = imc1d_cf.step(st, 3000, 2000, 1000, 9000, (1.0, 0.0), 0.004, mesh, sig, lambda u: u / cv,
                                     lambda T: cv + 0 * T, src, geometry=geometry)
            assert abs(info["ledger"]["relative_closure"]) < 1e-12, info["ledger"]
    else:
        e1, e2 = np.linspace(0, 0.6, 13), np.linspace(0, 1.2, 21)
        st = imc2d_cf.init_simulation(3000, np.full((12, 20), 0.05), np.full((12, 20), 0.05), e1, e2,
                                      lambda T: cv * T, lambda u: u / cv, geometry=geometry)
        src = np.zeros((12, 20))
        src[3:5, 2:6] = 2.0
        for _ in range(4):
            st, info = imc2d_cf.step(st, 3000, 2000, 1000, 9000, (1.0, 0.0, 0.0, 0.0), 0.004, e1, e2, sig,
                                     lambda u: u / cv, lambda T: cv + 0 * T, src, geometry=geometry)
            assert abs(info["ledger"]["relative_closure"]) < 1e-12, info["ledger"]
    te = info["profiling"]["transport_events"]
    assert te["absorption_capture_events"] > 0 and te["absorption_continue_events"] > 0


def test_cf_slab_dropin_matches_reference_statistically(cuda):
    from radtranbook_b200 import imc1d_cf

    ref = np.load(os.path.join(G, "stats_cf_slab.npz"))
    S = SP.SLAB
    mesh = SP.slab_mesh()
    cv = S["cv"]
    A = float(ref["A"])
    seeds = int(ref["seeds"])
    Ts = []
    for s in range(seeds):
        st = imc1d_cf.init_simulation(S["Ntarget"], np.full(S["I"], S["T0"]), np.full(S["I"], S["T0"]), mesh,
                                      lambda T: cv * T, lambda u: u / cv, seed=0xCF00 + s)
        for _ in range(int(ref["steps"])):
            st, info = imc1d_cf.step(st, S["Ntarget"], S["Nboundary"], 0, S["NMax"], (1.0, 0.0), S["dt"], mesh,
                                     lambda T: A * T ** -3, lambda u: u / cv, lambda T: cv + 0 * T, np.zeros(S["I"]))
        Ts.append(st.temperature.copy())
    Ts = np.array(Ts)
    roi = ref["T_mean"] > 10 * S["T0"]
    SP.compare_means(Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds), ref["T_mean"], ref["T_se"], roi)


def test_cf_xy_dropin_matches_reference_statistically(cuda):
    from radtranbook_b200 import imc2d_cf

    ref = np.load(os.path.join(G, "stats_cf_xy.npz"))
    nx, ny, cv, T0 = int(ref["nx"]), int(ref["ny"]), float(ref["cv"]), float(ref["T0"])
    x_e = np.linspace(0, float(ref["L"]), nx + 1)
    y_e = np.linspace(0, 0.1, ny + 1)
    seeds = int(ref["seeds"])
    Ts, Trs = [], []
    for s in range(seeds):
        st = imc2d_cf.init_simulation(int(ref["Ntarget"]), np.full((nx, ny), T0), np.full((nx, ny), T0), x_e, y_e,
                                      lambda T: cv * T, lambda u: u / cv, geometry="xy", seed=0xCF80 + s)
        for _ in range(int(ref["steps"])):
            st, info = imc2d_cf.step(st, int(ref["Ntarget"]), int(ref["Nboundary"]), 0, int(ref["Nmax"]),
                                     (1.0, 0.0, 0.0, 0.0), float(ref["dt"]), x_e, y_e,
                                     lambda T: np.maximum(T, 1e-3) ** -3, lambda u: u / cv, lambda T: cv + 0 * T,
                                     np.zeros((nx, ny)), reflect=(False, False, True, True), geometry="xy")
        Ts.append(st.temperature.copy())
        Trs.append(st.radiation_temperature.copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    roi = ref["T_mean"] > 1.5 * T0
    SP.compare_means(Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds), ref["T_mean"], ref["T_se"], roi)
    SP.compare_means(Trs.mean(0), Trs.std(0, ddof=1) / np.sqrt(seeds), ref["Tr_mean"], ref["Tr_se"], roi)


def test_cf_zero_d_equilibrates_to_exact_temperature(cuda):
    """IMC/test_simple_equilibration.py set-up through the drop-in: the closed cell reaches
    cv T + a T^4 = cv T0 + a Tr0^4 (0.894 keV) within 1 %."""
    from scipy.optimize import brentq

    from radtranbook_b200 import imc1d_cf

    Teq = brentq(lambda T: 0.01 * T + 0.01372 * T ** 4 - (0.01 * 0.4 + 0.01372), 0.0, 10.0)
    mesh = np.array([[0.0, 0.1]])
    st = imc1d_cf.init_simulation(20000, np.array([0.4]), np.array([1.0]), mesh, lambda T: 0.01 * T,
                                  lambda u: u / 0.01)
    for _ in range(5):
        st, info = imc1d_cf.step(st, 20000, 0, 0, 20000, (0.0, 0.0), 0.01, mesh, lambda T: 100.0 + 0 * T,
                                 lambda u: u / 0.01, lambda T: 0.01 + 0 * T, np.zeros(1), reflect=(True, True),
                                 use_scalar_intensity_Tr=False, conserve_comb_energy=True)
        assert abs(info["ledger"]["relative_closure"]) < 1e-12
    assert abs(st.temperature[0] - Teq) < 0.01 * Teq, (st.temperature[0], Teq)
