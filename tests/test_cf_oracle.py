"""Carter-Forest oracle checks, no GPU (IMC/IMC1D_CarterForest.py, IMC/IMC2D_CarterForest.py):
the four event functions and the emission samplers against golden vectors recorded from
the reference (tests/golden/cf.npz, its draws replayed), the emission-time distribution,
energy closure in every geometry, and statistical parity of whole steps with the
reference's own runs (tests/golden/stats_cf_*.npz).

Tolerances as the Fleck-Cummings pins: integers (event kind, face, counts) exact, FP64
arithmetic restated in another order ~1e-12 relative, positions after a 2-D face crossing
within the reference's 1e-12 relative nudge.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import stat_problems as SP

G = os.path.join(os.path.dirname(__file__), "golden")
C = 29.98
A = 0.01372


def _pins():
    return np.load(os.path.join(G, "cf.npz"))


def _oracle_inputs(geo, row, r):
    """Reference draws -> the oracle's (u0 distance, direction, delay) and the rate."""
    oned = geo in ("slab", "spherical")
    thr = 1e-10 if oned else 1e-12
    sa, beta, fp = row[9], row[10], row[12]
    L = (row[6] - row[5]) if oned else min(row[6] - row[5], row[8] - row[7])
    k, u0 = 0, 0.5
    if sa > thr:
        u0, k = 1.0 - r[0], 1
    if sa * L > 1e4:
        u0, k = 1.0 - r[k], k + 1
    rate = C * sa * beta if (beta > 1e-15 and sa > 1e-15) else 0.0
    if rate > 0:
        ud, d = r[k], (r[k + 1], r[k + 2])
    else:
        ud, d = 0.5, (r[k], r[k + 1])
    u = [u0, d[0], ud, 0.0] if oned else [u0, d[0], d[1], ud]
    return list(row[:10]) + [rate, row[11], fp] + u


@pytest.mark.parametrize("geo,key", [("slab", "slab"), ("spherical", "sphere"), ("xy", "xy"), ("rz", "rz")])
def test_cf_event_matches_reference(geo, key):
    d = _pins()
    ins, rs, outs = d[f"{key}_in"], d[f"{key}_r"], d[f"{key}_out"]
    for row, r, ref in zip(ins, rs, outs):
        got = O.event_cf(geo, _oracle_inputs(geo, row, r))
        assert int(got[9]) == int(ref[9]), (geo, row, got, ref)   # census / boundary / continue / capture
        assert int(got[8]) == int(ref[8]), (geo, row, got, ref)   # face crossed
        np.testing.assert_allclose(got[0], ref[0], rtol=1e-15)     # weight (unchanged or 0)
        np.testing.assert_allclose(got[5], ref[5], rtol=1e-15)     # captured weight
        np.testing.assert_allclose(got[6], ref[6], rtol=1e-9, atol=1e-300)  # path-length estimator
        if int(ref[9]) != 4:  # a captured photon's remaining distance is meaningless (1-D returns its old one)
            np.testing.assert_allclose(got[7], ref[7], rtol=1e-9, atol=1e-13)   # distance to census
        np.testing.assert_allclose(got[3], ref[3], rtol=1e-10, atol=1e-12)  # position 1
        if int(ref[9]) != 4:
            np.testing.assert_allclose(got[1], ref[1], rtol=1e-9, atol=1e-10)  # direction (new after re-emission)
        if geo in ("xy", "rz"):
            np.testing.assert_allclose(got[4], ref[4], rtol=1e-10, atol=1e-12)
            if int(ref[9]) != 4:
                np.testing.assert_allclose(got[2], ref[2], rtol=1e-9, atol=1e-10)
    assert set(np.unique(outs[:, 9]).astype(int)) == {0, 1, 2, 4}


def _cf_sources(geo, T, sa, cv, N, dt=0.01):
    if geo in ("slab", "spherical"):
        I = len(T)
        e = np.linspace(0.0, 1.0, I + 1)
        vol = np.diff(e) if geo == "slab" else 4.0 / 3.0 * np.pi * (e[1:] ** 3 - e[:-1] ** 3)
        o = O.Oracle(geo, e, [0.0, 1.0], vol, 1)
    else:
        nx, ny = T.shape
        e1, e2 = np.linspace(0, 1, nx + 1), np.linspace(0, 2, ny + 1)
        o = O.Oracle("xy", e1, e2, O.flat2d(np.diff(e1)[:, None] * np.diff(e2)[None, :]), 1)
        T, sa, cv = O.flat2d(T), O.flat2d(sa), O.flat2d(cv)
    r = o.transport(T, sa, cv, None, 0, dt, 1.0, N, 0, 0, [None] * 4, (False,) * 4, rz_linear_source=False,
                    sources_only=True, method="cf")
    return o, r


@pytest.mark.parametrize("geo", ["slab", "spherical", "xy"])
def test_cf_emission_counts_weights_energies_match_reference(geo):
    d = _pins()
    key = {"slab": "slab", "spherical": "spherical", "xy": "xy"}[geo]
    for q in range(len(d[f"em_{key}_N"])):
        T, sa, cv = d[f"em_{key}_T"][q], d[f"em_{key}_sa"][q], d[f"em_{key}_cv"][q]
        o, r = _cf_sources(geo, T, sa, cv, int(d[f"em_{key}_N"][q]))
        b = o.get_bank()
        nc = o.nc
        cnt = np.bincount(b["cell"], minlength=nc)
        w = np.zeros(nc)
        w[b["cell"]] = b["weight"]
        ref_E = d[f"em_{key}_E"][q]
        ref_E = O.flat2d(ref_E) if geo == "xy" else ref_E
        np.testing.assert_array_equal(cnt, d[f"em_{key}_counts"][q])
        # the reference forms 1 - exp(-x) directly: relative error ~ 1e-16 / x for small x = rate dt
        Tf = O.flat2d(T) if geo == "xy" else T
        cvf = O.flat2d(cv) if geo == "xy" else cv
        x = C * (O.flat2d(sa) if geo == "xy" else sa) * 4 * A * np.maximum(Tf, 1e-12) ** 3 / cvf * 0.01
        tol = 1e-12 + 4e-16 / np.minimum(x, 1.0)
        assert np.all(np.abs(w - d[f"em_{key}_w"][q]) <= tol * np.abs(d[f"em_{key}_w"][q]))
        assert np.all(np.abs(r["emitted"] - ref_E) <= tol * np.abs(ref_E))
        assert np.all((b["time"] >= 0) & (b["time"] <= 0.01))


def test_cf_emission_times_follow_truncated_exponential():
    """Birth times in a cell of rate k: density k e^{-k t} / (1 - e^{-k dt}) on [0, dt]."""
    from scipy import stats

    T = np.full(4, 0.5)
    sa = np.array([1.0, 10.0, 100.0, 1000.0])
    cv = np.full(4, 0.05)
    o, _ = _cf_sources("slab", T, sa, cv, 40000)
    b = o.get_bank()
    beta = 4 * A * 0.5 ** 3 / 0.05
    for c in range(4):
        k = C * sa[c] * beta
        t = b["time"][b["cell"] == c]
        cdf = lambda x, k=k: (1 - np.exp(-k * x)) / (1 - np.exp(-k * 0.01))  # noqa: E731
        assert stats.kstest(t, cdf).pvalue > 1e-3


def _run_cf(geo, seed, steps=3, nthreads=2, conserve=False):
    if geo in ("slab", "spherical"):
        I = 40
        e = np.linspace(0.0, 0.2, I + 1)
        vol = np.diff(e) if geo == "slab" else 4.0 / 3.0 * np.pi * (e[1:] ** 3 - e[:-1] ** 3)
        run = O.OracleGray(geo, e, [0.0, 1.0], vol, seed, 3000, np.full(I, 0.05), np.full(I, 0.05),
                           lambda T: 0.1 * T, lambda u: u / 0.1, nthreads=nthreads)
        face = [None, np.array([1.0])] if geo == "spherical" else [np.array([1.0]), None]
        src = np.zeros(I)
        src[5:10] = 2.0
        kw = dict(reflect=(True, False))
    else:
        e1, e2 = np.linspace(0, 0.5, 11), np.linspace(0, 1.0, 9)
        v = np.diff(e1)[:, None] * np.diff(e2)[None, :] if geo == "xy" else \
            np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :]
        run = O.OracleGray(geo, e1, e2, O.flat2d(v), seed, 3000, np.full((10, 8), 0.05), np.full((10, 8), 0.05),
                           lambda T: 0.1 * T, lambda u: u / 0.1, nthreads=nthreads)
        face = [np.full(8, 1.0), None, None, None] if geo == "xy" else [None, None, np.full(10, 1.0), None]
        src = np.zeros((10, 8))
        src[3:5, 2:4] = 2.0
        kw = dict(reflect=(False, False, True, False) if geo == "xy" else (True, False, False, False),
                  max_events=1_000_000)
    out = []
    for _ in range(steps):
        r = run.step(3000, 2000, 1000, 9000, face, 0.005, lambda T: 5.0 * np.maximum(T, 0.01) ** -2,
                     lambda u: u / 0.1, lambda T: np.full_like(T, 0.1), source=src, conserve_comb_energy=conserve,
                     method="cf", **kw)
        out.append(r)
    return run, out


@pytest.mark.parametrize("geo", ["slab", "spherical", "xy", "rz"])
def test_cf_oracle_closes_energy(geo):
    run, out = _run_cf(geo, 7)
    for r in out:
        assert abs(r["closure"]) < 1e-12 * r["total_energy"], r["closure"]
        st = r["stats"]
        assert st[4] > 0 and st[2] > 0  # captures and re-emissions both happen
        assert st[1] > 0


def test_cf_slab_matches_reference_statistically():
    ref = np.load(os.path.join(G, "stats_cf_slab.npz"))
    S = SP.SLAB
    mesh = SP.slab_mesh()
    e = np.concatenate([mesh[:, 0], mesh[-1:, 1]])
    cv = S["cv"]
    Ts = []
    seeds = int(ref["seeds"])
    for s in range(seeds):
        run = O.OracleGray("slab", e, [0.0, 1.0], np.diff(e), 5000 + s, S["Ntarget"], np.full(S["I"], S["T0"]),
                           np.full(S["I"], S["T0"]), lambda T: cv * T, lambda u: u / cv, nthreads=2)
        for _ in range(int(ref["steps"])):
            run.step(S["Ntarget"], S["Nboundary"], 0, S["NMax"], [np.array([1.0]), None], S["dt"],
                     lambda T: float(ref["A"]) * T ** -3, lambda u: u / cv, lambda T: np.full_like(T, cv), method="cf")
        Ts.append(run.T.copy())
    Ts = np.array(Ts)
    roi = ref["T_mean"] > 10 * S["T0"]
    SP.compare_means(Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds), ref["T_mean"], ref["T_se"], roi)


def test_cf_xy_matches_reference_statistically():
    ref = np.load(os.path.join(G, "stats_cf_xy.npz"))
    nx, ny, cv, T0 = int(ref["nx"]), int(ref["ny"]), float(ref["cv"]), float(ref["T0"])
    x_e = np.linspace(0, float(ref["L"]), nx + 1)
    y_e = np.linspace(0, 0.1, ny + 1)
    vol = O.flat2d(np.diff(x_e)[:, None] * np.diff(y_e)[None, :])
    seeds = int(ref["seeds"])
    Ts, Trs = [], []
    for s in range(seeds):
        run = O.OracleGray("xy", x_e, y_e, vol, 6000 + s, int(ref["Ntarget"]), np.full((nx, ny), T0),
                           np.full((nx, ny), T0), lambda T: cv * T, lambda u: u / cv, nthreads=2)
        for _ in range(int(ref["steps"])):
            run.step(int(ref["Ntarget"]), int(ref["Nboundary"]), 0, int(ref["Nmax"]), [np.full(ny, 1.0), None, None, None],
                     float(ref["dt"]), lambda T: np.maximum(T, 1e-3) ** -3, lambda u: u / cv,
                     lambda T: np.full_like(T, cv), reflect=(False, False, True, True), max_events=1_000_000,
                     method="cf")
        Ts.append(run.grid(run.T).copy())
        Trs.append(run.grid(run.Tr).copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    roi = ref["T_mean"] > 1.5 * T0
    SP.compare_means(Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds), ref["T_mean"], ref["T_se"], roi)
    SP.compare_means(Trs.mean(0), Trs.std(0, ddof=1) / np.sqrt(seeds), ref["Tr_mean"], ref["Tr_se"], roi)


def _equilibrium(cv, T0, Tr0):
    """cv T + a T^4 = cv T0 + a Tr0^4 (the closed cell's conserved energy density)."""
    from scipy.optimize import brentq

    E = cv * T0 + A * Tr0 ** 4
    return brentq(lambda T: cv * T + A * T ** 4 - E, 0.0, 10.0)


def test_cf_zero_d_equilibrates_to_exact_temperature():
    """IMC/test_simple_equilibration.py set-up (one reflecting cell, sigma = 100, cv = 0.01,
    T = 0.4, Tr = 1.0, dt = 0.01): after 5 steps the material sits at the exact equilibrium
    (the reference prints ~0.88 keV; the exact value is 0.894)."""
    Teq = _equilibrium(0.01, 0.4, 1.0)
    e = np.array([0.0, 0.1])
    run = O.OracleGray("slab", e, [0.0, 1.0], np.diff(e), 11, 20000, np.array([0.4]), np.array([1.0]),
                       lambda T: 0.01 * T, lambda u: u / 0.01, nthreads=2)
    for _ in range(5):
        r = run.step(20000, 0, 0, 20000, [None, None], 0.01, lambda T: 100.0 + 0 * T, lambda u: u / 0.01,
                     lambda T: np.full_like(T, 0.01), reflect=(True, True), conserve_comb_energy=True, method="cf")
        assert abs(r["closure"]) < 1e-12 * r["total_energy"]
    assert abs(run.T[0] - Teq) < 0.01 * Teq, (run.T[0], Teq)
