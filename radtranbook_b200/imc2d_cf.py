"""Drop-in for the reference's IMC/IMC2D_CarterForest.py (Carter-Forest IMC, xy and rz), on
the B200 engine.

Same entry points, argument names, defaults and return values as
IMC/IMC2D_CarterForest.py:25 (init_simulation, the IMC2D one), :909 (step) and :1162
(run_simulation); boundary and fixed sources are those of IMC2D.  The emission is
a T^4 (1 - e^{-k dt}) / beta V per cell (k = c sigma_a beta, beta = 4 a max(T, 1e-12)^3 / cv)
with birth times of density ~ e^{-k t}; an absorbed photon is re-emitted isotropically after a
delay ~ Exp(k) if that falls inside the step, else deposited.
Differences from the reference, all deliberate:
  - Philox random streams keyed by `seed`;
  - FP32 tracking with the cell index deciding the cell: no 1e-12 face nudges, no minimum
    step at a face, no census snap within 1e-12 of the census distance, so the
    no-progress guard (no_progress_rel_tol, no_progress_max_streak) has nothing to catch;
    the event cap (max_events_per_particle) bounds every history;
  - internal energy is not clamped at 1e-12 (IMC/IMC2D_CarterForest.py:1061), so the ledger
    closes;
  - info['ledger'] adds the FP64 energy-balance closure.
"""
from __future__ import annotations

import numpy as np

from . import imc2d as _imc2d
from ._gray import GrayState, gray_step, tune  # noqa: F401

__c = 29.98
__a = 0.01372

SimulationState2D = GrayState
_NO_PROGRESS_REL_TOL = 1e-12
_NO_PROGRESS_MAX_STREAK = 8


def init_simulation(Ntarget, Tinit, Tr_init, edges1, edges2, eos, inv_eos, Ntarget_ic=None, geometry="xy",
                    seed=0x5EED0001, _allreduce=None):
    return _imc2d.init_simulation(Ntarget, Tinit, Tr_init, edges1, edges2, eos, inv_eos, Ntarget_ic=Ntarget_ic,
                                  geometry=geometry, seed=seed, _allreduce=_allreduce)


def step(state, Ntarget, Nboundary, Nsource, Nmax, T_boundary, dt, edges1, edges2, sigma_a_func, inv_eos, cv,
         source, reflect=(False, False, False, False), theta=1.0, use_scalar_intensity_Tr=True,
         conserve_comb_energy=False, geometry="xy", rz_linear_source=True, max_events_per_particle=1_000_000,
         boundary_source_func=None, fastpath_threshold=0.0, no_progress_rel_tol=_NO_PROGRESS_REL_TOL,
         no_progress_max_streak=_NO_PROGRESS_MAX_STREAK, _allreduce=None):
    del theta  # Carter-Forest has no Fleck factor
    if geometry not in ("xy", "rz"):
        raise ValueError(f"Unknown geometry: {geometry}")
    return gray_step(state, Ntarget=Ntarget, Nboundary=Nboundary, Nsource=Nsource, Nmax=Nmax,
                     T_boundary=T_boundary, dt=dt, sigma_a_func=sigma_a_func, inv_eos=inv_eos, cv=cv, source=source,
                     reflect=reflect, theta=1.0, use_scalar_intensity_Tr=use_scalar_intensity_Tr,
                     conserve_comb_energy=conserve_comb_energy, rz_linear_source=rz_linear_source,
                     max_events=max_events_per_particle, boundary_source_func=boundary_source_func,
                     geometry=geometry, allreduce=_allreduce, method="cf", cf_fastpath=fastpath_threshold)


def run_simulation(Ntarget, Nboundary, Nsource, Nmax, Tinit, Tr_init, T_boundary, dt, edges1, edges2, sigma_a_func,
                   eos, inv_eos, cv, source, final_time, reflect=(False, False, False, False), output_freq=1,
                   theta=1.0, use_scalar_intensity_Tr=True, Ntarget_ic=None, conserve_comb_energy=False,
                   geometry="xy", rz_linear_source=True, max_events_per_particle=1_000_000, fastpath_threshold=0.0,
                   no_progress_rel_tol=_NO_PROGRESS_REL_TOL, no_progress_max_streak=_NO_PROGRESS_MAX_STREAK,
                   seed=0x5EED0001):
    state = init_simulation(Ntarget, Tinit, Tr_init, edges1, edges2, eos, inv_eos, Ntarget_ic=Ntarget_ic,
                            geometry=geometry, seed=seed)
    times = [0.0]
    Tr_hist = [state.radiation_temperature.copy()]
    T_hist = [state.temperature.copy()]
    while state.time < final_time - 1e-15:
        step_dt = min(dt, final_time - state.time)
        state, info = step(state, Ntarget, Nboundary, Nsource, Nmax, T_boundary, step_dt, edges1, edges2,
                           sigma_a_func, inv_eos, cv, source, reflect=reflect,
                           use_scalar_intensity_Tr=use_scalar_intensity_Tr, conserve_comb_energy=conserve_comb_energy,
                           geometry=geometry, rz_linear_source=rz_linear_source,
                           max_events_per_particle=max_events_per_particle, fastpath_threshold=fastpath_threshold)
        if (state.count - 1) % output_freq == 0 or (final_time - state.time) < 1e-12:
            times.append(info["time"])
            Tr_hist.append(state.radiation_temperature.copy())
            T_hist.append(state.temperature.copy())
    return np.array(times), np.array(Tr_hist), np.array(T_hist)
