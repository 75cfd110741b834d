"""Whole-step statistical parity of the FP64 oracle with the reference's own Numba runs
(fixtures tests/golden/stats_*.npz, made by tests/golden/make_golden.py), and the 0-D
equilibration fixture of IMC/0-DTests.py:55-93 against its exact equilibrium.

Criterion: per-cell means over independent seeds agree within combined standard errors
(no heated cell beyond 4.5 sigma, at most 8% beyond 3 sigma).
"""
import os

import numpy as np

from oracle import oracle as O
from tests import stat_problems as SP

G = os.path.join(os.path.dirname(__file__), "golden")


def test_slab_marshak_matches_reference_statistically():
    ref = np.load(os.path.join(G, "stats_slab.npz"))
    S = SP.SLAB
    mesh = SP.slab_mesh()
    e = np.concatenate([mesh[:, 0], mesh[-1:, 1]])
    cv = S["cv"]
    Ts = []
    seeds = int(ref["seeds"])
    for s in range(seeds):
        run = O.OracleGray("slab", e, [0.0, 1.0], np.diff(e), 1000 + s, S["Ntarget"], np.full(S["I"], S["T0"]),
                           np.full(S["I"], S["T0"]), lambda T: cv * T, lambda u: u / cv, nthreads=2)
        for _ in range(int(ref["steps"])):
            run.step(S["Ntarget"], S["Nboundary"], 0, S["NMax"], [np.array([1.0]), None], S["dt"],
                     lambda T: 300.0 * T ** -3, lambda u: u / cv, lambda T: np.full_like(T, cv))
        Ts.append(run.T.copy())
    Ts = np.array(Ts)
    m, se = Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds)
    roi = ref["T_mean"] > 10 * S["T0"]
    SP.compare_means(m, se, ref["T_mean"], ref["T_se"], roi)


def test_rz_crooked_pipe_matches_reference_statistically():
    ref = np.load(os.path.join(G, "stats_rz.npz"))
    R = SP.RZ
    r_e, z_e, sig, cvg, face = SP.rz_setup()
    vol = O.flat2d(np.pi * (r_e[1:] ** 2 - r_e[:-1] ** 2)[:, None] * np.diff(z_e)[None, :])
    seeds = int(ref["seeds"])
    Ts = []
    for s in range(seeds):
        run = O.OracleGray("rz", r_e, z_e, vol, 2000 + s, R["Ntarget"], np.full(sig.shape, R["T0"]),
                           np.full(sig.shape, R["T0"]), lambda T: cvg * T, lambda u: u / cvg, nthreads=4)
        for _ in range(int(ref["steps"])):
            run.step(R["Ntarget"], R["Nboundary"], 0, R["Nmax"], [None, None, face, None], R["dt"],
                     lambda T: sig.copy(), lambda u: u / cvg, lambda T: cvg.copy(),
                     reflect=(True, False, False, False), max_events=1_000_000)
        Ts.append(run.grid(run.T).copy())
    Ts = np.array(Ts)
    m, se = Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds)
    roi = ref["T_mean"] > 1.05 * R["T0"]
    SP.compare_means(m, se, ref["T_mean"], ref["T_se"], roi)


def test_zero_d_equilibration_reaches_exact_equilibrium():
    """IMC/0-DTests.py: one reflecting cell, sigma=1, cv=0.01, T0=0.4, Tr0=1.0, dt=0.025."""
    from scipy.optimize import brentq

    a, cv = 0.01372, 0.01
    e0 = cv * 0.4 + a * 1.0 ** 4
    Teq = brentq(lambda T: cv * T + a * T ** 4 - e0, 0.0, 2.0)
    e = np.array([0.0, 0.1])
    run = O.OracleGray("slab", e, [0.0, 1.0], np.diff(e), 77, 20000, np.array([0.4]), np.array([1.0]),
                       lambda T: cv * T, lambda u: u / cv, nthreads=2)
    for _ in range(15):
        r = run.step(20000, 0, 0, 100000, [None, None], 0.025, lambda T: np.ones_like(T), lambda u: u / cv,
                     lambda T: np.full_like(T, cv), reflect=(True, True), conserve_comb_energy=True)
        assert abs(r["closure"]) < 1e-12 * r["total_energy"]
    assert abs(run.T[0] - Teq) < 0.01 * Teq, (run.T[0], Teq)
