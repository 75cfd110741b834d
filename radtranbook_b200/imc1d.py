"""Drop-in for the reference's IMC/IMC1D.py time-step API, on the B200 engine.

Same entry points, argument names, defaults, return values and info keys as
IMC/IMC1D.py:859-905 (init_simulation), :908-1124 (step) and :1127-1169 (run_simulation).
geometry='slab' or 'spherical'; mesh is the reference's (I, 2) array of cell edges.
Differences from the reference, all deliberate:
  - random numbers are Philox streams keyed by `seed` (reproducible; the reference's are
    not), so runs agree with the reference statistically, not bit for bit;
  - a weight-floor kill deposits its energy in every cell (the reference skips the two edge
    cells, IMC/IMC1D.py:191), and fixed-source birth times are U(0, dt) (the reference
    draws U(0, 1), IMC/IMC1D.py:311);
  - info['ledger'] adds the FP64 energy-balance closure (including the comb discrepancy).
"""
from __future__ import annotations

import numpy as np

from ._gray import GrayState, gray_step, init_state, tune  # noqa: F401
from .engine import Engine

__c = 29.98
__a = 0.01372

SimulationState = GrayState


def _cell_volumes(mesh, geometry):
    if geometry == "slab":
        return mesh[:, 1] - mesh[:, 0]
    if geometry == "spherical":
        return (4.0 / 3.0) * np.pi * (mesh[:, 1] ** 3 - mesh[:, 0] ** 3)
    raise ValueError(f"Unknown geometry: {geometry}")


def _edges(mesh):
    mesh = np.asarray(mesh, dtype=np.float64)
    return np.concatenate([mesh[:, 0], mesh[-1:, 1]])


def init_simulation(Ntarget, Tinit, Tr_init, mesh, eos, inv_eos, Ntarget_ic=None, geometry="slab",
                    T_emit_floor=0.0, seed=0x5EED0001, _allreduce=None):
    """_allreduce: a torch.distributed module for a particle-partitioned run (the process
    parallelism of IMC/IMC1DMPI.py, radtranbook_b200.partition); every step then takes the
    same one."""
    mesh = np.asarray(mesh, dtype=np.float64)
    eng = Engine(geometry, _edges(mesh), np.array([0.0, 1.0]), _cell_volumes(mesh, geometry), seed=seed,
                 capacity=4 * int(Ntarget) + 1024)
    return init_state(eng, 1, (mesh.shape[0],), Ntarget, Tinit, Tr_init, eos, inv_eos, Ntarget_ic, T_emit_floor,
                      dist=_allreduce)


def step(state, Ntarget, Nboundary, Nsource, NMax, T_boundary, dt, mesh, sigma_a_func, inv_eos, cv, source,
         reflect=(False, False), theta=1.0, use_scalar_intensity_Tr=True, conserve_comb_energy=False,
         T_emit_floor=0.0, geometry="slab", _allreduce=None):
    return gray_step(state, Ntarget=Ntarget, Nboundary=Nboundary, Nsource=Nsource, Nmax=NMax,
                     T_boundary=T_boundary, dt=dt, sigma_a_func=sigma_a_func, inv_eos=inv_eos, cv=cv, source=source,
                     reflect=reflect, theta=theta, use_scalar_intensity_Tr=use_scalar_intensity_Tr,
                     conserve_comb_energy=conserve_comb_energy, T_emit_floor=T_emit_floor, geometry=geometry,
                     allreduce=_allreduce)


def run_simulation(Ntarget, Nboundary, Nsource, NMax, Tinit, Tr_init, T_boundary, dt, mesh, sigma_a_func, eos,
                   inv_eos, cv, source, final_time, reflect=(False, False), output_freq=1, theta=1.0,
                   use_scalar_intensity_Tr=True, Ntarget_ic=None, conserve_comb_energy=False, geometry="slab",
                   seed=0x5EED0001):
    state = init_simulation(Ntarget, Tinit, Tr_init, mesh, eos, inv_eos, Ntarget_ic=Ntarget_ic, geometry=geometry,
                            seed=seed)
    radiation_temperatures = [state.radiation_temperature.copy()]
    temperatures = [state.temperature.copy()]
    time_values = [0.0]
    while state.time < final_time:
        step_dt = min(dt, final_time - state.time)
        state, info = step(state, Ntarget, Nboundary, Nsource, NMax, T_boundary, step_dt, mesh, sigma_a_func,
                           inv_eos, cv, source, reflect, theta=theta, use_scalar_intensity_Tr=use_scalar_intensity_Tr,
                           conserve_comb_energy=conserve_comb_energy, geometry=geometry)
        if (state.count - 1) % output_freq == 0 or (info["time"] - final_time) < step_dt:
            radiation_temperatures.append(state.radiation_temperature.copy())
            temperatures.append(state.temperature.copy())
            time_values.append(info["time"])
    return np.array(time_values), np.array(radiation_temperatures), np.array(temperatures)
