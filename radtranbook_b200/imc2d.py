"""Drop-in for the reference's IMC/IMC2D.py time-step API (geometry 'xy' or 'rz'), on the
B200 engine.

Same entry points, argument names, defaults, return values and info keys as
IMC/IMC2D.py:1514-1588 (init_simulation), :1591-1897 (step), :1900-1984 (run_simulation);
T_boundary is ordered (min-1, max-1, min-2, max-2) = (rmin, rmax, zmin, zmax) in rz.
Differences from the reference, all deliberate:
  - Philox random streams keyed by `seed` (statistical, not bitwise, agreement);
  - no 1e-12 position nudges: the cell index decides the cell and positions are clamped to
    it (FP32 tracking);
  - the weight-based radiation temperature (use_scalar_intensity_Tr=False) is binned with
    the flat index i + nx*j consistently (IMC/IMC2D.py:1809 reshapes it as (nx, ny));
  - info['ledger'] adds the FP64 energy-balance closure (including the comb discrepancy).
"""
from __future__ import annotations

import numpy as np

from ._gray import GrayState, gray_step, init_state, tune  # noqa: F401
from .engine import Engine

__c = 29.98
__a = 0.01372

SimulationState2D = GrayState


def _cell_volumes(edges1, edges2, geometry):
    if geometry == "xy":
        return np.diff(edges1)[:, None] * np.diff(edges2)[None, :]
    if geometry == "rz":
        return np.pi * (edges1[1:] ** 2 - edges1[:-1] ** 2)[:, None] * np.diff(edges2)[None, :]
    raise ValueError(f"Unknown geometry: {geometry}")


def _flat_volumes(edges1, edges2, geometry):
    return np.ascontiguousarray(_cell_volumes(edges1, edges2, geometry).T).reshape(-1)


def init_simulation(Ntarget, Tinit, Tr_init, edges1, edges2, eos, inv_eos, Ntarget_ic=None, geometry="xy",
                    seed=0x5EED0001, _allreduce=None):
    """_allreduce: a torch.distributed module for a particle-partitioned run (the process
    parallelism of IMC/IMC2DMPI.py, radtranbook_b200.partition); every step then takes the
    same one."""
    e1 = np.asarray(edges1, dtype=np.float64)
    e2 = np.asarray(edges2, dtype=np.float64)
    eng = Engine(geometry, e1, e2, _flat_volumes(e1, e2, geometry), seed=seed, capacity=4 * int(Ntarget) + 1024)
    return init_state(eng, 2, (len(e1) - 1, len(e2) - 1), Ntarget, Tinit, Tr_init, eos, inv_eos, Ntarget_ic,
                      dist=_allreduce)


def step(state, Ntarget, Nboundary, Nsource, Nmax, T_boundary, dt, edges1, edges2, sigma_a_func, inv_eos, cv,
         source, reflect=(False, False, False, False), theta=1.0, use_scalar_intensity_Tr=True,
         conserve_comb_energy=False, geometry="xy", rz_linear_source=True, max_events_per_particle=1_000_000,
         boundary_source_func=None, _timing=False, _allreduce=None):
    if geometry not in ("xy", "rz"):
        raise ValueError(f"Unknown geometry: {geometry}")
    return gray_step(state, Ntarget=Ntarget, Nboundary=Nboundary, Nsource=Nsource, Nmax=Nmax,
                     T_boundary=T_boundary, dt=dt, sigma_a_func=sigma_a_func, inv_eos=inv_eos, cv=cv, source=source,
                     reflect=reflect, theta=theta, use_scalar_intensity_Tr=use_scalar_intensity_Tr,
                     conserve_comb_energy=conserve_comb_energy, rz_linear_source=rz_linear_source,
                     max_events=max_events_per_particle, boundary_source_func=boundary_source_func,
                     geometry=geometry, allreduce=_allreduce)


def run_simulation(Ntarget, Nboundary, Nsource, Nmax, Tinit, Tr_init, T_boundary, dt, edges1, edges2, sigma_a_func,
                   eos, inv_eos, cv, source, final_time, reflect=(False, False, False, False), output_freq=1,
                   theta=1.0, use_scalar_intensity_Tr=True, Ntarget_ic=None, conserve_comb_energy=False,
                   geometry="xy", rz_linear_source=True, max_events_per_particle=1_000_000, seed=0x5EED0001):
    state = init_simulation(Ntarget, Tinit, Tr_init, edges1, edges2, eos, inv_eos, Ntarget_ic=Ntarget_ic,
                            geometry=geometry, seed=seed)
    times = [0.0]
    Tr_hist = [state.radiation_temperature.copy()]
    T_hist = [state.temperature.copy()]
    while state.time < final_time - 1e-15:
        step_dt = min(dt, final_time - state.time)
        state, info = step(state, Ntarget, Nboundary, Nsource, Nmax, T_boundary, step_dt, edges1, edges2,
                           sigma_a_func, inv_eos, cv, source, reflect=reflect, theta=theta,
                           use_scalar_intensity_Tr=use_scalar_intensity_Tr, conserve_comb_energy=conserve_comb_energy,
                           geometry=geometry, rz_linear_source=rz_linear_source,
                           max_events_per_particle=max_events_per_particle)
        if (state.count - 1) % output_freq == 0 or (final_time - state.time) < 1e-12:
            times.append(info["time"])
            Tr_hist.append(state.radiation_temperature.copy())
            T_hist.append(state.temperature.copy())
    return np.array(times), np.array(Tr_hist), np.array(T_hist)
