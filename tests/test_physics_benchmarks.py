"""Analytic gray benchmarks on the FP64 oracle (CPU).

* Su–Olson at tau = 1: radiation (Tr^4) and material (T^4) energy densities against the
  analytic tables shipped with the reference, read from the reference checkout at test time
  (its path in the RADTRANBOOK_REF environment variable; skipped when that is unset).  Tolerance: absolute
  0.025 on the radiation energy (peak 0.64) and 0.015 on the material energy (peak 0.27),
  the Monte Carlo noise of 3x10^4 particles per step plus the cell averaging at the source
  edge x = 0.5.
* 0-D equilibration at dt = 0.002 ns: T(t) and Tr(t) within 2 % of the exchange ODE at every
  step (Monte Carlo noise and the comb's random energy drift; dt/tau ~ 0.07).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import physics_problems as PP

REF = os.environ.get("RADTRANBOOK_REF", "")


def run_su_olson_oracle(p, seed=0x5EED):
    run = O.OracleGray("slab", p["edges"], np.array([0.0, 1.0]), np.diff(p["edges"]), seed, p["Ntarget"], p["T0"],
                       p["T0"], p["eos"], p["inv_eos"])
    for _ in range(p["steps"]):
        run.step(p["Ntarget"], 0, p["Nsource"], p["Nmax"], [None, None], p["dt"], p["sigma"], p["inv_eos"], p["cv"],
                 source=p["source"], reflect=(True, False))
    return run.T ** 4, run.Tr ** 4


def run_zero_d_oracle(p, seed=0x0D0D):
    run = O.OracleGray("slab", p["edges"], np.array([0.0, 1.0]), np.diff(p["edges"]), seed, p["Ntarget"],
                       np.array([p["T0"]]), np.array([p["Tr0"]]), p["eos"], p["inv_eos"])
    T, Tr = [], []
    for _ in range(p["steps"]):
        run.step(p["Ntarget"], 0, 0, p["Nmax"], [None, None], p["dt"], p["sigma"], p["inv_eos"], p["cvf"],
                 reflect=(True, True))
        T.append(run.T[0])
        Tr.append(run.Tr[0])
    return np.array(T), np.array(Tr)


@pytest.mark.skipif(not REF or not os.path.exists(os.path.join(REF, "IMC", "SuOlson.py")),
                    reason="RADTRANBOOK_REF does not name a reference checkout")
def test_su_olson_oracle_matches_analytic_tables():
    p = PP.su_olson(1.0)
    T4, Tr4 = run_su_olson_oracle(p)
    rad, mat = PP.su_olson_tables(REF)
    col = PP.SU_OLSON_TAUS.index(1.0) + 1
    L = p["edges"][-1]
    for table, ours, tol in ((rad, Tr4, 0.025), (mat, T4, 0.015)):
        x = table[:, 0]
        inside = x < L
        got = np.interp(x[inside], p["mid"], ours)
        err = np.abs(got - table[inside, col])
        assert err.max() <= tol, (err.max(), x[inside][np.argmax(err)])


def test_zero_d_oracle_matches_exchange_ode():
    p = PP.zero_d()
    T, Tr = run_zero_d_oracle(p)
    times = p["dt"] * np.arange(1, p["steps"] + 1)
    Tex, Trex = PP.zero_d_exact(p, times)
    assert np.max(np.abs(T - Tex) / Tex) < 0.02
    assert np.max(np.abs(Tr - Trex) / Trex) < 0.02
