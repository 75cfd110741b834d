"""Whole-step statistical parity of the GPU drop-in Fleck-Cummings steps with the reference's
own Numba runs: per-cell material (and radiation) temperature means over independent seeds
against the reference's means over 32 seeds (fixtures tests/golden/stats_slab.npz,
stats_rz.npz and stats_mg.npz, written by tests/golden/make_golden.py --stats-only from
IMC1D.step, IMC2D.step and MG_IMC2D.step with the step counts stored in each fixture).

Criterion (tests/stat_problems.compare_means): in the region of interest no cell beyond 4.5
combined standard errors and at most 8 % of the cells beyond 3.
"""
import os

import numpy as np
import pytest

from radtranbook_b200 import imc1d, imc2d, mg_imc2d
from tests import stat_problems as SP

pytestmark = pytest.mark.gpu

G = os.path.join(os.path.dirname(__file__), "golden")


def _stats(xs):
    xs = np.array(xs)
    return xs.mean(0), xs.std(0, ddof=1) / np.sqrt(len(xs))


def test_slab_dropin_matches_reference_statistically(cuda):
    ref = np.load(os.path.join(G, "stats_slab.npz"))
    S = SP.SLAB
    mesh = SP.slab_mesh()
    cv = S["cv"]
    Ts, Trs = [], []
    for s in range(int(ref["seeds"])):
        st = imc1d.init_simulation(S["Ntarget"], np.full(S["I"], S["T0"]), np.full(S["I"], S["T0"]), mesh,
                                   lambda T: cv * T, lambda u: u / cv, seed=0x51AB00 + s)
        for _ in range(int(ref["steps"])):
            st, info = imc1d.step(st, S["Ntarget"], S["Nboundary"], 0, S["NMax"], (1.0, 0.0), S["dt"], mesh,
                                  lambda T: 300.0 * T ** -3, lambda u: u / cv, lambda T: cv + 0 * T, np.zeros(S["I"]))
            assert abs(info["ledger"]["relative_closure"]) < 1e-12
        Ts.append(st.temperature.copy())
        Trs.append(st.radiation_temperature.copy())
    roi = ref["T_mean"] > 10 * S["T0"]
    SP.compare_means(*_stats(Ts), ref["T_mean"], ref["T_se"], roi)
    SP.compare_means(*_stats(Trs), ref["Tr_mean"], ref["Tr_se"], roi)


def test_rz_crooked_pipe_dropin_matches_reference_statistically(cuda):
    ref = np.load(os.path.join(G, "stats_rz.npz"))
    R = SP.RZ
    r_e, z_e, sig, cvg, _ = SP.rz_setup()
    bsf = lambda r, z, side: 0.5 if (side == "zmin" and r < 0.5) else 0.0  # noqa: E731
    Ts, Trs = [], []
    for s in range(int(ref["seeds"])):
        st = imc2d.init_simulation(R["Ntarget"], np.full(sig.shape, R["T0"]), np.full(sig.shape, R["T0"]), r_e, z_e,
                                   lambda T: cvg * T, lambda u: u / cvg, geometry="rz", seed=0x52B200 + s)
        for _ in range(int(ref["steps"])):
            st, info = imc2d.step(st, R["Ntarget"], R["Nboundary"], 0, R["Nmax"], (0.0, 0.0, 0.0, 0.0), R["dt"], r_e,
                                  z_e, lambda T: sig.copy(), lambda u: u / cvg, lambda T: cvg.copy(),
                                  np.zeros(sig.shape), reflect=(True, False, False, False), geometry="rz",
                                  boundary_source_func=bsf)
            assert abs(info["ledger"]["relative_closure"]) < 1e-12
        Ts.append(st.temperature.copy())
        Trs.append(st.radiation_temperature.copy())
    roi = ref["T_mean"] > 1.05 * R["T0"]
    SP.compare_means(*_stats(Ts), ref["T_mean"], ref["T_se"], roi)
    SP.compare_means(*_stats(Trs), ref["Tr_mean"], ref["Tr_se"], roi)


def test_mg_marshak_dropin_matches_reference_statistically(cuda):
    ref = np.load(os.path.join(G, "stats_mg.npz"))
    nx, L, Gn, cv, T0 = int(ref["nx"]), float(ref["L"]), int(ref["G"]), float(ref["cv"]), float(ref["T0"])
    edges = np.logspace(-4, np.log10(20.0), Gn + 1)
    nu = 0.5 * (edges[:-1] + edges[1:])
    funcs = [(lambda T, n=n: np.clip(10.0 * n ** -3 * np.power(T, -0.5), 1e-2, 1e6)) for n in nu]
    x_e, y_e = np.linspace(0, L, nx + 1), np.array([0.0, 1.0])
    Ts, Trs = [], []
    for s in range(int(ref["seeds"])):
        st = mg_imc2d.init_simulation(int(ref["Ntarget"]), np.full((nx, 1), T0), np.full((nx, 1), T0), x_e, y_e, edges,
                                      lambda T: cv * T, lambda e: e / cv, geometry="xy", seed=0x53C300 + s)
        for _ in range(int(ref["steps"])):
            st, info = mg_imc2d.step(st, int(ref["Ntarget"]), int(ref["Nboundary"]), 0, int(ref["Nmax"]),
                                     (1.0, 0.0, 0.0, 0.0), float(ref["dt"]), x_e, y_e, edges, funcs, lambda e: e / cv,
                                     lambda T: cv + 0 * T, np.zeros((nx, 1)), reflect=(False, False, True, True),
                                     geometry="xy")
            assert abs(info["ledger"]["relative_closure"]) < 1e-12
        Ts.append(st.temperature[:, 0].copy())
        Trs.append(st.radiation_temperature[:, 0].copy())
    roi = ref["T_mean"] > 10 * T0
    SP.compare_means(*_stats(Ts), ref["T_mean"], ref["T_se"], roi)
    SP.compare_means(*_stats(Trs), ref["Tr_mean"], ref["Tr_se"], roi)
