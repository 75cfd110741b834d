"""Drop-in for the reference's MG_IMC/MG_IMC1D.py multigroup spherical time-step API, on the
B200 engine.

Same entry points, argument names, defaults, return values and info keys as
MG_IMC/MG_IMC1D.py:850 (init_simulation), :917 (step) and :1312 (run_simulation); `mesh` is
the reference's (I, 2) array of shell radii, `source` is (I,) (placed in group 0, as the
reference does) or (n_groups, I).  Group Planck fractions come from the engine's own
incomplete-Planck-integral series (the reference imports them from the external
`planck_integrals` extension, or splits energy equally across groups without it,
MG_IMC/MG_IMC1D.py:60-94).
Differences from the reference, all deliberate:
  - Philox random streams keyed by `seed`;
  - zero-weight entries are not tracked, and a boundary sphere of radius 0 issues no
    particles (the reference moves zero-weight particles without effect);
  - copies made by the comb carry FP32 weights, so conserve_comb_energy='radiation' leaves a
    per-bin discrepancy at FP32 rounding, booked in info['ledger'];
  - max_events_per_particle is accepted and, as in the reference, not applied;
  - info['ledger'] adds the FP64 energy-balance closure.
"""
from __future__ import annotations

import math
import time as _time

import numpy as np
import torch

from . import _lib
from ._gray import GrayState, _host_copy, _staged, check_partition, face_temperatures
from .engine import A_RAD, C_LIGHT, Engine
from .materials import evaluate, evaluate_groups
from .mg_imc2d import planck_fractions
from .partition import local_count, sum_scalars, sum_tensors, summary_totals, world_of

__c = 29.98
__a = 0.01372


def _volumes(mesh: np.ndarray) -> np.ndarray:
    return (4.0 / 3.0) * np.pi * (mesh[:, 1] ** 3 - mesh[:, 0] ** 3)


class SimulationState1DMG(GrayState):
    """MG_IMC/MG_IMC1D.py:115-137 fields: the bank (weights, mus, times, positions,
    cell_indices, groups), the material arrays, radiation energy and flux by group."""

    def __getattr__(self, name):
        if name == "groups":
            return object.__getattribute__(self, "_engine").bank.view("group").cpu().numpy().astype(np.int32)
        return super().__getattr__(name)


def _census_moments(eng: Engine) -> tuple[torch.Tensor, torch.Tensor]:
    """Per (group, cell) sums over the live census: energy (GJ) and radial flux
    c * sum(w mu) / V (MG_IMC/MG_IMC1D.py:1209-1227), each (G, I)."""
    G, nc = eng.ng, eng.nc
    E = torch.zeros(G * nc, dtype=torch.float64, device=eng.device)
    F = torch.zeros(G * nc, dtype=torch.float64, device=eng.device)
    if eng.bank.size:
        w = eng.bank.view("weight").double()
        live = w > 0
        idx = (eng.bank.view("cell").long() + nc * eng.bank.view("group").long())[live]
        E.index_add_(0, idx, w[live])
        F.index_add_(0, idx, (w * eng.bank.view("dir1").double())[live])
    return E.view(G, nc), C_LIGHT * F.view(G, nc) / eng.vol.view(1, nc)


def _comb_mode(conserve_comb_energy) -> str:
    if conserve_comb_energy is True or conserve_comb_energy == "material":
        return "material"
    if conserve_comb_energy == "radiation":
        return "radiation"
    if conserve_comb_energy is False or conserve_comb_energy in ("none", None):
        return "none"
    raise ValueError(f"conserve_comb_energy: {conserve_comb_energy!r}")


def init_simulation(Ntarget, Tinit, Tr_init, mesh, energy_edges, eos, inv_eos, Ntarget_ic=None, T_emit_floor=0.0,
                    seed=0x5EED0001, _allreduce=None):
    """_allreduce: a torch.distributed module for a particle-partitioned run
    (radtranbook_b200.partition); every step of the state then takes the same one."""
    rank, world = world_of(_allreduce)
    dist = _allreduce if world > 1 else None
    mesh = np.asarray(mesh, dtype=np.float64)
    I = mesh.shape[0]
    G = len(energy_edges) - 1
    edges = np.concatenate([mesh[:, 0], mesh[-1:, 1]])
    eng = Engine("spherical", edges, np.array([0.0, 1.0]), _volumes(mesh), seed=seed, n_groups=G,
                 group_edges=energy_edges, capacity=4 * int(Ntarget) + 1024)
    if world > 1:
        eng.partition(rank, world)
    dev = eng.device
    z = lambda: torch.zeros(I, dtype=torch.float64, device=dev)  # noqa: E731
    state = SimulationState1DMG(eng, 1, (I,), z(), z(), z(), 0.0, 0.0, 0)
    Tg = torch.as_tensor(np.asarray(Tinit, dtype=np.float64), device=dev)
    e = evaluate(eos, Tg, lambda: np.asarray(Tinit, dtype=np.float64), Tg)
    state._e.copy_(e.reshape(-1))
    state._T.copy_(Tg.reshape(-1))
    back = evaluate(inv_eos, state._e, lambda: state._e.cpu().numpy(), Tg)
    assert torch.allclose(back, Tg), "Inverse EOS failed"
    N_ic = Ntarget if Ntarget_ic is None else Ntarget_ic
    tr = torch.as_tensor(np.asarray(Tr_init, dtype=np.float64), device=dev).reshape(-1)
    eng.init_census(tr, local_count(N_ic, rank, world), T_emit_floor)
    rad, _ = _census_moments(eng)
    sum_tensors(dist, [rad])
    state.__dict__["radiation_energy_by_group"] = rad.cpu().numpy().copy()
    state.__dict__["radiation_flux_by_group"] = np.zeros((G, I))
    state.__dict__["radiation_energy_by_group_postcomb"] = None
    state._Tr.copy_(torch.pow(rad.sum(0) / eng.vol / A_RAD, 0.25))
    radiation, internal = eng.energy_totals(state._e)
    radiation = sum_scalars(dist, [radiation], dev)[0]
    state.previous_total_energy = internal + radiation
    state.refresh_host()
    return state


def _budget(state, sig_h, cv_h, T_inner, T_outer, source, energy_edges, dt, theta, Ntarget, fmin, T_emit_floor):
    """Particle budget shared by the sources in proportion to their energies, at least
    fmin * Ntarget for each non-zero one (MG_IMC/MG_IMC1D.py:1000-1040)."""
    eng = state._engine
    e = eng.e1.cpu().numpy()
    vol = eng.vol.cpu().numpy()
    T = state.temperature
    E_in = __a * __c * T_inner ** 4 / 4.0 * dt * 4.0 * math.pi * e[0] ** 2 if T_inner > 0.0 else 0.0
    E_out = __a * __c * T_outer ** 4 / 4.0 * dt * 4.0 * math.pi * e[-1] ** 2 if T_outer > 0.0 else 0.0
    s = np.asarray(source if source is not None else 0.0, dtype=np.float64)
    E_src = float(np.sum(np.maximum(s, 0.0) * (vol if s.ndim == 1 else vol[None, :]) * dt)) if s.ndim else 0.0
    b = planck_fractions(energy_edges, T)
    sP = np.sum(sig_h * b, axis=0)
    f = np.clip(1.0 / (1.0 + theta * (4.0 * __a * T ** 3 / cv_h) * sP * __c * dt), 0.0, 1.0)
    emit = __a * __c * T ** 4 * np.sum(sig_h * f[None, :] * b, axis=0) * dt * vol
    if T_emit_floor > 0.0:
        emit[T < T_emit_floor] = 0.0
    E_emit = float(np.sum(emit))
    E_all = E_in + E_out + E_src + E_emit
    N = int(Ntarget)
    floor = max(1, int(round(fmin * N)))
    if not E_all > 0.0:
        return N, 0, 0, 0
    part = lambda E: max(int(round(N * E / E_all)), floor) if E > 0.0 else 0  # noqa: E731
    return part(E_in), part(E_out), part(E_src), part(E_emit)


def step(state, Ntarget, Nboundary, Nsource, Nmax, T_boundary, dt, mesh, energy_edges, sigma_a_funcs, inv_eos, cv,
         source, reflect=(False, False), theta=1.0, use_scalar_intensity_Tr=True, conserve_comb_energy=True,
         max_events_per_particle=1_000_000, T_emit_floor=0.0, particle_budget_fmin=0.0, Nmax_growth=0,
         Nmax_final=None, _allreduce=None):
    t0 = _time.perf_counter()
    eng: Engine = state._engine
    # particle partition (radtranbook_b200.partition): counts are totals, each rank takes its share
    rank, world = check_partition(eng, _allreduce)
    dist = _allreduce if world > 1 else None
    G, I = eng.ng, eng.nc
    mode = _comb_mode(conserve_comb_energy)
    like = state._T
    host_T = lambda: state.temperature  # noqa: E731
    # host callables' results go up by asynchronous copies from pinned buffers of the state
    sig = evaluate_groups(sigma_a_funcs, like, host_T, like, **_staged(state, "sigma_g", G * I))  # (G, I)
    cvv = evaluate(cv, like, host_T, like, **_staged(state, "cv", I))
    Tb = [T_boundary[q](state.time) if callable(T_boundary[q]) else T_boundary[q] for q in range(2)]
    n_side = None
    if particle_budget_fmin > 0.0:
        n_in, n_out, Nsource, Ntarget = _budget(state, sig.cpu().numpy(), cvv.cpu().numpy(), float(Tb[0]),
                                                float(Tb[1]), source, energy_edges, dt, theta, Ntarget,
                                                particle_budget_fmin, T_emit_floor)
        Nboundary, n_side = 0, [n_in, n_out, 0, 0]
    src = None
    if Nsource > 0 and source is not None:
        s = np.asarray(source, dtype=np.float64)
        if s.ndim == 1:  # gray source: group 0 (MG_IMC/MG_IMC1D.py:690-694)
            s2 = np.zeros((G, I))
            s2[0] = s
            s = s2
        elif s.ndim != 2:
            raise ValueError(f"source shape {s.shape} not supported")
        if s.max() > 0.0:
            src = torch.as_tensor(np.ascontiguousarray(s).reshape(-1), device=eng.device)
    cache = state.__dict__.setdefault("_face_cache", {})
    e1 = eng.e1.cpu().numpy() if "e1" not in cache else cache["e1"]
    cache["e1"] = e1
    faces = face_temperatures(1, "spherical", tuple(Tb), state.time, e1, np.array([0.0, 1.0]), None, eng.device,
                              cache)
    refl = tuple(reflect) + (False,) * (4 - len(reflect))
    t_eval = _time.perf_counter()
    lc = lambda n: local_count(n, rank, world)  # noqa: E731
    eng.transport_async(state._T, sig.reshape(-1).contiguous(), cvv, src, state.count, dt, theta, lc(Ntarget),
                        lc(Nboundary), lc(Nsource), faces, refl, max_events=0, rz_linear_source=False,
                        t_emit_floor=T_emit_floor, n_boundary_side=None if n_side is None else [lc(n) for n in n_side])
    sum_tensors(dist, [eng.dep, eng.si, eng.emitted, eng.boundary_group, eng.escaped_group])
    eng.material_update(state._e, state._Tr)
    nmax_l = lc(Nmax) if Nmax > 0 else (-lc(-Nmax) if Nmax < 0 else 0)
    eng.comb_async(nmax_l, state.count, state._e, per_group=True, conserve_radiation=(mode == "radiation"))
    if mode == "material":
        sum_tensors(dist, [eng.disc])
        state._e.add_(eng.disc.view(G, I).sum(0) / eng.vol)
    Tn = evaluate(inv_eos, state._e, lambda: _host_copy(state._e), like, **_staged(state, "T_new", I))
    state._T.copy_(Tn.reshape(-1))
    copies = state.host_copies()
    ms_src, ms_tr = eng.phase_times()  # waits for the tracking only (the comb still runs)
    try:
        sm = eng.fetch(copies)
    except _lib.ImcError as ex:
        if ex.status == 3:
            raise AssertionError("non-finite or non-positive material state") from ex
        raise
    if not use_scalar_intensity_Tr:
        pre = eng.spare  # the tracked bank before the comb
        w = pre.view("weight").double()
        live = w > 0
        rad_c = torch.zeros(I, dtype=torch.float64, device=eng.device)
        rad_c.index_add_(0, pre.view("cell").long()[live], w[live])
        sum_tensors(dist, [rad_c])
        state._Tr.copy_(torch.pow(rad_c / eng.vol / A_RAD, 0.25))
        state.refresh_host()
    else:
        state.take_host_copies()
    rad_g, flux_g = _census_moments(eng)
    sum_tensors(dist, [rad_g, flux_g])
    internal = float(sm.internal_energy)  # the same material state on every rank
    tot = summary_totals(dist, sm, eng.bank.size, eng.device)  # summed over the ranks of a partition
    rad = tot["rad"]
    comb_disc = tot["comb_before"] - rad
    if mode == "material":
        internal += comb_disc
    boundary_emission = tot["e_side_total"]
    boundary_loss = tot["escaped_total"]
    source_emission = tot["source_emission"]
    n_boundary = int(sum(sm.n_side))
    if dist is not None:
        n_boundary = int(sum_scalars(dist, [float(n_boundary)], eng.device)[0])
    total = internal + rad
    dE = total - state.previous_total_energy
    residual = dE - boundary_emission + boundary_loss - source_emission
    closure = residual + (0.0 if mode == "material" else comb_disc)
    state.__dict__["radiation_energy_by_group"] = rad_g.cpu().numpy().copy()
    state.__dict__["radiation_flux_by_group"] = flux_g.cpu().numpy().copy()
    state.time = state.time + dt
    state.previous_total_energy = total
    state.count += 1
    stats = tot["stats"]
    n_tr = tot["n_bank"]
    ev = int(stats[_lib.STAT_EVENTS])
    t_end = _time.perf_counter()
    info = {
        "time": state.time,
        "temperature": state.temperature.copy(),
        "radiation_temperature": state.radiation_temperature.copy(),
        "radiation_energy_by_group": state.radiation_energy_by_group.copy(),
        "radiation_flux_by_group": state.radiation_flux_by_group.copy(),
        "N_particles": tot["n_particles"],
        "total_energy": total,
        "total_internal_energy": internal,
        "total_radiation_energy": rad,
        "boundary_emission": boundary_emission,
        "N_boundary": n_boundary,
        "boundary_loss": boundary_loss,
        "boundary_loss_by_group": eng.escaped_group.cpu().numpy().copy(),
        "source_emission": source_emission,
        "energy_residual": residual,
        "Nmax_next": (min(Nmax + Nmax_growth, Nmax_final) if Nmax_final is not None else Nmax + Nmax_growth)
        if Nmax_growth > 0 else Nmax,
        "ledger": {"comb_discrepancy": comb_disc, "closure": closure,
                   "relative_closure": closure / max(abs(total), 1e-300),
                   "emission": tot["emission_total"],
                   "weight_floor": 1e-14 * tot["weight_sum"] / max(n_tr, 1)},
        "profiling": {
            "phase_times_s": {
                "sampling": (t_eval - t0) + ms_src * 1e-3,
                "transport": ms_tr * 1e-3,
                "postprocess": max(t_end - t_eval - (ms_src + ms_tr) * 1e-3, 0.0),
                "total": t_end - t0,
            },
            "transport_events": {
                "total": ev,
                "boundary_crossings": int(stats[_lib.STAT_BOUNDARY]),
                "scatter_events": int(stats[_lib.STAT_SCATTER]),
                "census_events": int(stats[_lib.STAT_CENSUS]),
                "weight_floor_kills": int(stats[_lib.STAT_FLOOR]),
                "reflections": int(stats[_lib.STAT_REFLECT]),
                "avg_events_per_particle": ev / max(n_tr, 1),
                "n_particles_transported": n_tr,
            },
        },
    }
    return state, info


def run_simulation(Ntarget, Nboundary, Nsource, Nmax, Tinit, Tr_init, T_boundary, dt, mesh, energy_edges,
                   sigma_a_funcs, eos, inv_eos, cv, source, final_time, reflect=(False, False), output_freq=1,
                   theta=1.0, use_scalar_intensity_Tr=True, Ntarget_ic=None, conserve_comb_energy=True,
                   Nmax_growth=0, Nmax_final=None, seed=0x5EED0001):
    state = init_simulation(Ntarget, Tinit, Tr_init, mesh, energy_edges, eos, inv_eos, Ntarget_ic=Ntarget_ic,
                            seed=seed)
    time_values = [0.0]
    Tr_history = [state.radiation_temperature.copy()]
    T_history = [state.temperature.copy()]
    history = []
    time_tol = max(1e-15, 1e-12 * max(final_time, 1.0))
    while state.time < final_time - time_tol:
        step_dt = min(dt, final_time - state.time)
        state, info = step(state, Ntarget, Nboundary, Nsource, Nmax, T_boundary, step_dt, mesh, energy_edges,
                           sigma_a_funcs, inv_eos, cv, source, reflect, theta=theta,
                           use_scalar_intensity_Tr=use_scalar_intensity_Tr, conserve_comb_energy=conserve_comb_energy,
                           Nmax_growth=Nmax_growth, Nmax_final=Nmax_final)
        Nmax = info["Nmax_next"]
        history.append(info)
        if (state.count - 1) % output_freq == 0:
            time_values.append(info["time"])
            Tr_history.append(state.radiation_temperature.copy())
            T_history.append(state.temperature.copy())
    return np.array(time_values), np.array(Tr_history), np.array(T_history), state, history


def tune(state, grid=None, repeats=2):
    from ._gray import tune as _tune

    return _tune(state, grid=grid, repeats=repeats)
