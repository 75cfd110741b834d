"""Checkpoint and exact restart of drop-in simulation states, in the formats the reference's
drivers write.

  * NPZ, IMC/CrookedPipe2D.py:459-505 (save_checkpoint) and :508-551 (load_checkpoint): the
    same function signatures and keys.  The reference's save reads state.mu / eta / r / z,
    which IMC2D states do not have, so its files carry an empty census; here the census is
    written under the keys it meant (dir1 -> chkpt_mu, dir2 -> chkpt_eta, pos1 -> chkpt_r,
    pos2 -> chkpt_z; 1-D: mus -> chkpt_mu, positions -> chkpt_r), with the cell indices,
    groups, step counter, previous total energy and Philox key added (chkpt_cell_i,
    chkpt_cell_j, chkpt_groups, chkpt_count, chkpt_previous_total_energy, chkpt_philox_seed).
  * pickle payload, MG_IMC/problems/test_marshak_wave_multigroup_powerlaw.py:46-120
    (_serialize_state, save_checkpoint, load_checkpoint; checkpoint_version 1), with
    "philox": {"seed", "step"} added to the payload.

Exact resume: particle fields are FP32 on the device and are stored widened to FP64 (exact
both ways), material fields are FP64, and the Philox key and the step counter (state.count,
the counter word of every draw of a step) are restored, so a resumed run draws the same random
numbers as an uninterrupted one.  The reference's own restart restores NumPy / Python random
states instead (its Numba streams are not restored at all).
"""
from __future__ import annotations

import pickle
import random

import numpy as np
import torch

CHECKPOINT_VERSION = 1


def _is_mg(state) -> bool:
    return state._engine.ng > 1


def serialize_state(state) -> dict:
    """Pickle-safe payload of a drop-in state (the reference's _serialize_state keys for its
    state class: 2-D weights/dir1/dir2/times/pos1/pos2/cell_i/cell_j, 1-D
    weights/mus/times/positions/cell_indices; groups and radiation_energy_by_group when
    multigroup), plus the Philox key."""
    eng = state._engine
    if state._dim == 2:
        keys = ("weights", "dir1", "dir2", "times", "pos1", "pos2", "cell_i", "cell_j")
    else:
        keys = ("weights", "mus", "times", "positions", "cell_indices")
    out = {k: np.asarray(getattr(state, k)) for k in keys}
    out.update(internal_energy=np.array(state.internal_energy), temperature=np.array(state.temperature),
               radiation_temperature=np.array(state.radiation_temperature), time=float(state.time),
               previous_total_energy=float(state.previous_total_energy), count=int(state.count),
               philox_seed=int(eng.seed), geometry=eng.geometry)
    if _is_mg(state):
        out["groups"] = np.asarray(state.groups)
        for k in ("radiation_energy_by_group", "radiation_energy_by_group_postcomb", "radiation_flux_by_group"):
            if k in state.__dict__:
                v = state.__dict__[k]
                out[k] = None if v is None else np.array(v)
    return out


def restore_state(state, data: dict) -> None:
    """Load a payload into a state built by the matching init_simulation (same mesh, groups
    and geometry): census bank, material fields, time, counters and Philox key."""
    eng = state._engine
    if "geometry" in data and data["geometry"] != eng.geometry:
        raise ValueError(f"checkpoint geometry {data['geometry']!r} does not match the state's {eng.geometry!r}")
    w = np.asarray(data["weights"], dtype=np.float64)
    n = len(w)
    z = np.zeros(n)
    if state._dim == 2:
        nx = state._shape[0]
        cell = np.asarray(data["cell_i"], dtype=np.int64) + nx * np.asarray(data["cell_j"], dtype=np.int64)
        d1, d2, p1, p2 = data["dir1"], data["dir2"], data["pos1"], data["pos2"]
    else:
        cell = np.asarray(data["cell_indices"], dtype=np.int64)
        d1, d2, p1, p2 = data["mus"], z, data["positions"], z
    if n and (cell.min() < 0 or cell.max() >= eng.nc):
        raise ValueError("checkpoint census has cells outside the mesh")
    groups = data.get("groups") if _is_mg(state) else None
    eng.bank.load(w, d1, d2, data["times"], p1, p2, cell, groups)
    eng._census_dev_valid = False
    dev = eng.device
    for name, t in (("internal_energy", state._e), ("temperature", state._T), ("radiation_temperature", state._Tr)):
        t.copy_(state.flat(torch.as_tensor(np.asarray(data[name], dtype=np.float64), device=dev)))
    state.time = float(data["time"])
    state.previous_total_energy = float(data["previous_total_energy"])
    state.count = int(data["count"])
    if data.get("philox_seed") is not None:
        eng.seed = int(data["philox_seed"]) & 0xFFFFFFFFFFFFFFFF
    for k in ("radiation_energy_by_group", "radiation_energy_by_group_postcomb", "radiation_flux_by_group"):
        if k in data:
            state.__dict__[k] = None if data[k] is None else np.array(data[k])
    state.refresh_host()


# ------------------------------------------------------------------ pickle payload
def save_checkpoint(path, state, step_count, cumulative_residual, history, metadata) -> None:
    """MG_IMC/problems/test_marshak_wave_multigroup_powerlaw.py:97-107 payload, with the
    Philox key and step counter."""
    payload = {
        "checkpoint_version": CHECKPOINT_VERSION,
        "state": serialize_state(state),
        "step_count": int(step_count),
        "cumulative_residual": float(cumulative_residual),
        "history": history,
        "metadata": metadata,
        "philox": {"seed": int(state._engine.seed), "step": int(state.count)},
        "np_random_state": np.random.get_state(),
        "py_random_state": random.getstate(),
    }
    with open(path, "wb") as f:
        pickle.dump(payload, f, protocol=pickle.HIGHEST_PROTOCOL)


def load_checkpoint(path) -> dict:
    """Load and validate a payload (MG_IMC/problems/test_marshak_wave_multigroup_powerlaw.py:110-120);
    restore it into a state with restore_state(state, payload["state"])."""
    with open(path, "rb") as f:
        payload = pickle.load(f)
    version = payload.get("checkpoint_version", None)
    if version != CHECKPOINT_VERSION:
        raise ValueError(f"Unsupported checkpoint version: {version} (expected {CHECKPOINT_VERSION})")
    return payload


# ------------------------------------------------------------------ NPZ (crooked pipe driver)
def save_checkpoint_npz(state, step_count, times, fiducial_data, fiducial_data_rad, output_times_saved, current_dt,
                        filename, method="fc", fastpath_threshold=0.0, no_progress_rel_tol=1e-12,
                        no_progress_max_streak=8, profile_phase_totals_s=None, profile_event_totals=None,
                        profile_transported_particles_total=0, profile_step_count=0) -> None:
    """IMC/CrookedPipe2D.py:459-505 with the census written (see the module docstring)."""
    fiducial_labels = list(fiducial_data.keys())
    fiducial_temps = np.array([fiducial_data[lbl] for lbl in fiducial_labels])
    fiducial_temps_rad = np.array([fiducial_data_rad[lbl] for lbl in fiducial_labels])
    if profile_phase_totals_s is None:
        profile_phase_totals_s = np.zeros(4, dtype=np.float64)
    if profile_event_totals is None:
        profile_event_totals = np.zeros(8, dtype=np.int64)
    s = serialize_state(state)
    if state._dim == 2:
        mu, eta, r, z, ci, cj = s["dir1"], s["dir2"], s["pos1"], s["pos2"], s["cell_i"], s["cell_j"]
    else:
        mu, r, ci = s["mus"], s["positions"], s["cell_indices"]
        eta, z, cj = np.array([]), np.array([]), np.zeros(len(ci), dtype=np.int64)
    extra = {"chkpt_groups": s["groups"]} if "groups" in s else {}
    np.savez(
        filename,
        chkpt_temperature=s["temperature"], chkpt_radiation_temperature=s["radiation_temperature"],
        chkpt_internal_energy=s["internal_energy"],
        chkpt_weights=s["weights"], chkpt_mu=mu, chkpt_eta=eta, chkpt_particle_times=s["times"], chkpt_r=r, chkpt_z=z,
        chkpt_time=np.float64(state.time), chkpt_current_dt=np.float64(current_dt),
        chkpt_step_count=np.int64(step_count),
        chkpt_times=np.array(times, dtype=np.float64),
        chkpt_output_saved=np.array(sorted(output_times_saved), dtype=np.float64),
        chkpt_fiducial_labels=np.array(fiducial_labels, dtype=object),
        chkpt_fiducial_temps=fiducial_temps, chkpt_fiducial_temps_rad=fiducial_temps_rad,
        chkpt_method=np.array(method, dtype=object), chkpt_fastpath_threshold=np.float64(fastpath_threshold),
        chkpt_no_progress_rel_tol=np.float64(no_progress_rel_tol),
        chkpt_no_progress_max_streak=np.int64(no_progress_max_streak),
        chkpt_profile_phase_totals_s=np.array(profile_phase_totals_s, dtype=np.float64),
        chkpt_profile_event_totals=np.array(profile_event_totals, dtype=np.int64),
        chkpt_profile_transported_particles_total=np.int64(profile_transported_particles_total),
        chkpt_profile_step_count=np.int64(profile_step_count),
        # restart fields the reference file lacks
        chkpt_cell_i=np.asarray(ci, dtype=np.int64), chkpt_cell_j=np.asarray(cj, dtype=np.int64),
        chkpt_count=np.int64(state.count), chkpt_previous_total_energy=np.float64(state.previous_total_energy),
        chkpt_philox_seed=np.uint64(state._engine.seed), chkpt_geometry=np.array(state._engine.geometry, dtype=object),
        **extra,
    )


def load_checkpoint_npz(filename, state, fiducial_points):
    """IMC/CrookedPipe2D.py:508-551: restores the state in place and returns (step_count, times,
    fiducial_data, fiducial_data_rad, output_times_saved, current_dt, metadata).  A file without
    cell indices (one the reference wrote) has its census located from the positions; without
    chkpt_count / chkpt_previous_total_energy the step counter is step_count and the energy is
    recomputed from the restored state."""
    del fiducial_points  # the labels are stored in the file, as in the reference
    ck = np.load(filename, allow_pickle=True)
    eng = state._engine
    w = ck["chkpt_weights"]
    n = len(w)
    data = {
        "weights": w, "times": ck["chkpt_particle_times"] if n else np.zeros(0),
        "internal_energy": ck["chkpt_internal_energy"], "temperature": ck["chkpt_temperature"],
        "radiation_temperature": ck["chkpt_radiation_temperature"], "time": float(ck["chkpt_time"]),
        "previous_total_energy": float(ck["chkpt_previous_total_energy"]) if "chkpt_previous_total_energy" in ck
        else 0.0,
        "count": int(ck["chkpt_count"]) if "chkpt_count" in ck else int(ck["chkpt_step_count"]),
        "philox_seed": int(ck["chkpt_philox_seed"]) if "chkpt_philox_seed" in ck else None,
    }
    e1, e2 = eng.e1.cpu().numpy(), eng.e2.cpu().numpy()

    def locate(x, e):
        return np.clip(np.searchsorted(e, x, side="right") - 1, 0, len(e) - 2)

    if state._dim == 2:
        data.update(dir1=ck["chkpt_mu"], dir2=ck["chkpt_eta"], pos1=ck["chkpt_r"], pos2=ck["chkpt_z"])
        if "chkpt_cell_i" in ck:
            data.update(cell_i=ck["chkpt_cell_i"], cell_j=ck["chkpt_cell_j"])
        else:
            data.update(cell_i=locate(ck["chkpt_r"], e1), cell_j=locate(ck["chkpt_z"], e2))
    else:
        data.update(mus=ck["chkpt_mu"], positions=ck["chkpt_r"])
        data["cell_indices"] = ck["chkpt_cell_i"] if "chkpt_cell_i" in ck else locate(ck["chkpt_r"], e1)
    if "chkpt_groups" in ck:
        data["groups"] = ck["chkpt_groups"]
    restore_state(state, data)
    if "chkpt_previous_total_energy" not in ck:
        rad, internal = eng.energy_totals(state._e)
        state.previous_total_energy = internal + rad
    step_count = int(ck["chkpt_step_count"])
    current_dt = float(ck["chkpt_current_dt"])
    times = list(ck["chkpt_times"])
    output_times_saved = set(float(v) for v in ck["chkpt_output_saved"])
    fiducial_data, fiducial_data_rad = {}, {}
    for idx, lbl in enumerate(ck["chkpt_fiducial_labels"]):
        fiducial_data[str(lbl)] = list(ck["chkpt_fiducial_temps"][idx])
        fiducial_data_rad[str(lbl)] = list(ck["chkpt_fiducial_temps_rad"][idx])
    get = lambda k, d: ck[k] if k in ck else d  # noqa: E731
    metadata = {
        "method": str(get("chkpt_method", "fc")),
        "fastpath_threshold": float(get("chkpt_fastpath_threshold", 0.0)),
        "no_progress_rel_tol": float(get("chkpt_no_progress_rel_tol", 1e-12)),
        "no_progress_max_streak": int(get("chkpt_no_progress_max_streak", 8)),
        "profile_phase_totals_s": np.asarray(get("chkpt_profile_phase_totals_s", np.zeros(4)), dtype=np.float64),
        "profile_event_totals": np.asarray(get("chkpt_profile_event_totals", np.zeros(8)), dtype=np.int64),
        "profile_transported_particles_total": int(get("chkpt_profile_transported_particles_total", 0)),
        "profile_step_count": int(get("chkpt_profile_step_count", 0)),
    }
    return step_count, times, fiducial_data, fiducial_data_rad, output_times_saved, current_dt, metadata
