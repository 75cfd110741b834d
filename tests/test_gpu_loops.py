"""The drop-in time loops and info dicts against the reference's own.

tests/golden/loops.json was recorded by tests/golden/make_golden.py (--loops-only) from the
reference's run_simulation loops (IMC/IMC1D.py:1127-1169, IMC/IMC2D.py:1900-1984,
MG_IMC/MG_IMC2D.py:2125-2259, MG_IMC/MG_IMC1D.py:1312-1369, IMC/IMC1D_CarterForest.py:1381-1413,
IMC/IMC2D_CarterForest.py:1162-1250) on small problems whose final time is not a multiple of
dt (every loop ends with a short step) with output_freq = 3, and from one step() of each
module.  Checked here, for every drop-in module with the same arguments:

  - the output times, exactly as the reference's loop produces them (its output cadence,
    including the reference's own quirks: IMC1D outputs every step, IMC1D_CarterForest and
    MG_IMC1D count steps differently from the 2-D loops);
  - the shapes of the radiation and material temperature histories;
  - for MG_IMC2D the times of the returned info history and its key tree (the loop adds
    cumulative_energy_residual and net_boundary_energy), for MG_IMC1D the info history's times;
  - every key of the reference's step() info dict, nested dicts included, is present
    (the drop-in adds info['ledger']).
"""
import json
import os

import numpy as np
import pytest

from radtranbook_b200 import imc1d, imc1d_cf, imc2d, imc2d_cf, mg_imc1d, mg_imc2d

pytestmark = pytest.mark.gpu

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "loops.json")))
L = FIX["problem"]
cv, N, Nmax, dt, tf, of = L["cv"], L["N"], L["Nmax"], L["dt"], L["final_time"], L["output_freq"]
eos, inv = (lambda T: cv * T), (lambda e: e / cv)
cvf = lambda T: cv + 0 * T  # noqa: E731
sig = lambda T: 10.0 + 0 * T  # noqa: E731
I = 10
MESH = np.array([[i * 0.01, (i + 1) * 0.01] for i in range(I)])
T1 = np.full(I, L["T0"])
GEDGES = np.array([1e-2, 0.3, 2.0, 20.0])
GSIG = [lambda T, k=k: (5.0 + 0 * T) * k for k in (1.0, 2.0, 4.0)]
EDGES2D = {"xy": (np.linspace(0, 0.06, 7), np.linspace(0, 0.05, 6)),
           "rz": (np.linspace(0, 0.06, 7), np.linspace(0, 0.05, 6))}


def _has_keys(ours, ref, path=""):
    for k, sub in ref.items():
        assert k in ours, f"info key {path + k} missing"
        if sub:
            assert isinstance(ours[k], dict), path + k
            _has_keys(ours[k], sub, path + k + ".")


def _check_hist(name, times, Tr, T):
    ref = FIX[name]
    np.testing.assert_allclose(np.asarray(times), ref["times"], rtol=0, atol=1e-15)
    assert list(np.shape(Tr)) == ref["Tr_shape"] and list(np.shape(T)) == ref["T_shape"]


def test_imc1d_loop_and_info(cuda):
    _check_hist("imc1d", *imc1d.run_simulation(N, N, 0, Nmax, T1, T1, (1.0, 0.0), dt, MESH, sig, eos, inv, cvf,
                                               np.zeros(I), tf, output_freq=of))
    st = imc1d.init_simulation(N, T1, T1, MESH, eos, inv)
    _, info = imc1d.step(st, N, N, 0, Nmax, (1.0, 0.0), dt, MESH, sig, inv, cvf, np.zeros(I))
    _has_keys(info, FIX["imc1d"]["info_keys"])


def test_imc1d_cf_loop_and_info(cuda):
    _check_hist("imc1d_cf", *imc1d_cf.run_simulation(N, N, 0, Nmax, T1, T1, (1.0, 0.0), dt, MESH, sig, eos, inv,
                                                     cvf, np.zeros(I), tf, output_freq=of))
    st = imc1d_cf.init_simulation(N, T1, T1, MESH, eos, inv)
    _, info = imc1d_cf.step(st, N, N, 0, Nmax, (1.0, 0.0), dt, MESH, sig, inv, cvf, np.zeros(I))
    _has_keys(info, FIX["imc1d_cf"]["info_keys"])


@pytest.mark.parametrize("geo", ["xy", "rz"])
@pytest.mark.parametrize("mod,name", [(imc2d, "imc2d"), (imc2d_cf, "imc2d_cf")], ids=["fc", "cf"])
def test_imc2d_loop_and_info(cuda, mod, name, geo):
    e1, e2 = EDGES2D[geo]
    T2 = np.full((len(e1) - 1, len(e2) - 1), L["T0"])
    _check_hist(f"{name}_{geo}", *mod.run_simulation(N, N, 0, Nmax, T2, T2, (1.0, 0.0, 0.0, 0.0), dt, e1, e2, sig,
                                                     eos, inv, cvf, np.zeros_like(T2), tf, output_freq=of,
                                                     geometry=geo))
    st = mod.init_simulation(N, T2, T2, e1, e2, eos, inv, geometry=geo)
    _, info = mod.step(st, N, N, 0, Nmax, (1.0, 0.0, 0.0, 0.0), dt, e1, e2, sig, inv, cvf, np.zeros_like(T2),
                       geometry=geo)
    _has_keys(info, FIX[f"{name}_{geo}"]["info_keys"])


def test_mg_imc2d_loop_and_info(cuda):
    m_e, m_y = np.linspace(0, 0.06, 7), np.array([0.0, 1.0])
    Tm = np.full((len(m_e) - 1, 1), L["T0"])
    history, state = mg_imc2d.run_simulation(N, N, 0, Nmax, Tm, Tm, (1.0, 0.0, 0.0, 0.0), dt, m_e, m_y, GEDGES, GSIG,
                                             eos, inv, cvf, np.zeros_like(Tm), tf, reflect=(False, False, True, True),
                                             output_freq=of)
    ref = FIX["mg_imc2d"]
    np.testing.assert_allclose([h["time"] for h in history], ref["history_times"], rtol=0, atol=1e-15)
    _has_keys(history[-1], ref["history_keys"])
    assert abs(state.time - tf) < 1e-12
    st = mg_imc2d.init_simulation(N, Tm, Tm, m_e, m_y, GEDGES, eos, inv)
    _, info = mg_imc2d.step(st, N, N, 0, Nmax, (1.0, 0.0, 0.0, 0.0), dt, m_e, m_y, GEDGES, GSIG, inv, cvf,
                            np.zeros_like(Tm), reflect=(False, False, True, True))
    _has_keys(info, ref["info_keys"])


def test_mg_imc1d_loop_and_info(cuda):
    Ts = np.full(6, L["T0"])
    smesh = np.array([[i * 0.01, (i + 1) * 0.01] for i in range(6)])
    times, Tr, T, state, history = mg_imc1d.run_simulation(N, N, 0, Nmax, Ts, Ts, (0.0, 1.0), dt, smesh, GEDGES, GSIG,
                                                           eos, inv, cvf, np.zeros(6), tf, output_freq=of)
    _check_hist("mg_imc1d", times, Tr, T)
    np.testing.assert_allclose([h["time"] for h in history], FIX["mg_imc1d"]["history_times"], rtol=0, atol=1e-15)
    st = mg_imc1d.init_simulation(N, Ts, Ts, smesh, GEDGES, eos, inv)
    _, info = mg_imc1d.step(st, N, N, 0, Nmax, (0.0, 1.0), dt, smesh, GEDGES, GSIG, inv, cvf, np.zeros(6))
    _has_keys(info, FIX["mg_imc1d"]["info_keys"])
