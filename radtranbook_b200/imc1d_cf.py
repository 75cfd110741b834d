"""Drop-in for the reference's IMC/IMC1D_CarterForest.py (Carter-Forest IMC, slab and
sphere), on the B200 engine.

Same entry points, argument names, defaults and return values as
IMC/IMC1D_CarterForest.py:1103 (init_simulation), :1151 (step) and :1381 (run_simulation).
Carter-Forest uses the true opacity (no Fleck factor, no effective scatter), emits
a T^4 (1 - e^{-k dt}) / beta V per cell with birth times of density ~ e^{-k t}
(k = c sigma_a beta, beta = 4 a T^3 / cv), and re-emits an absorbed photon isotropically after
a delay ~ Exp(k) if that falls inside the step, else deposits it.
Differences from the reference, all deliberate:
  - Philox random streams keyed by `seed`;
  - the slab fixed source is stratified by cell (counts ceil(N S_c / S), as the sphere's and
    the Fleck-Cummings modules') instead of one categorical cell draw per particle (same
    distribution);
  - an entry at or below the weight floor is left in census instead of deleted
    (IMC/IMC1D_CarterForest.py:320-322 loses its energy), and internal energy is not clamped
    at 1e-10 (:1289), so the ledger closes;
  - info['ledger'] adds the FP64 energy-balance closure.
"""
from __future__ import annotations

import numpy as np

from . import imc1d as _imc1d
from ._gray import GrayState, gray_step, tune  # noqa: F401

__c = 29.98
__a = 0.01372

SimulationState = GrayState


def init_simulation(Ntarget, Tinit, Tr_init, mesh, eos, inv_eos, Ntarget_ic=None, geometry="slab", seed=0x5EED0001,
                    _allreduce=None):
    # the Carter-Forest initial census is the Fleck-Cummings module's (ceil counts per cell)
    return _imc1d.init_simulation(Ntarget, Tinit, Tr_init, mesh, eos, inv_eos, Ntarget_ic=Ntarget_ic,
                                  geometry=geometry, seed=seed, _allreduce=_allreduce)


def step(state, Ntarget, Nboundary, Nsource, NMax, T_boundary, dt, mesh, sigma_a_func, inv_eos, cv, source,
         reflect=(False, False), use_scalar_intensity_Tr=True, conserve_comb_energy=False, geometry="slab",
         event_cap_per_particle=0, fastpath_threshold=0.0, _allreduce=None):
    if geometry not in ("slab", "spherical"):
        raise ValueError(f"Unknown geometry: {geometry}")
    # the reference stops a history once its event count reaches the cap (>=,
    # IMC/IMC1D_CarterForest.py:245-248), i.e. after cap - 1 events; the engine allows
    # max_events events (a cap of 1 is taken as 2: at least one event)
    cap = max(int(event_cap_per_particle) - 1, 1) if event_cap_per_particle > 0 else 0
    return gray_step(state, Ntarget=Ntarget, Nboundary=Nboundary, Nsource=Nsource, Nmax=NMax,
                     T_boundary=T_boundary, dt=dt, sigma_a_func=sigma_a_func, inv_eos=inv_eos, cv=cv, source=source,
                     reflect=reflect, theta=1.0, use_scalar_intensity_Tr=use_scalar_intensity_Tr,
                     conserve_comb_energy=conserve_comb_energy, geometry=geometry, max_events=cap,
                     allreduce=_allreduce, method="cf", cf_fastpath=fastpath_threshold)


def run_simulation(Ntarget, Nboundary, Nsource, NMax, Tinit, Tr_init, T_boundary, dt, mesh, sigma_a_func, eos,
                   inv_eos, cv, source, final_time, reflect=(False, False), output_freq=1,
                   use_scalar_intensity_Tr=True, Ntarget_ic=None, conserve_comb_energy=False, geometry="slab",
                   event_cap_per_particle=0, fastpath_threshold=0.0, seed=0x5EED0001):
    state = init_simulation(Ntarget, Tinit, Tr_init, mesh, eos, inv_eos, Ntarget_ic=Ntarget_ic, geometry=geometry,
                            seed=seed)
    radiation_temperatures = [state.radiation_temperature.copy()]
    temperatures = [state.temperature.copy()]
    time_values = [0.0]
    while state.time < final_time:
        step_dt = min(dt, final_time - state.time)
        state, info = step(state, Ntarget, Nboundary, Nsource, NMax, T_boundary, step_dt, mesh, sigma_a_func,
                           inv_eos, cv, source, reflect=reflect, use_scalar_intensity_Tr=use_scalar_intensity_Tr,
                           conserve_comb_energy=conserve_comb_energy, geometry=geometry,
                           event_cap_per_particle=event_cap_per_particle, fastpath_threshold=fastpath_threshold)
        if state.count % output_freq == 0:
            radiation_temperatures.append(state.radiation_temperature.copy())
            temperatures.append(state.temperature.copy())
            time_values.append(state.time)
    return np.array(time_values), np.array(radiation_temperatures), np.array(temperatures)
