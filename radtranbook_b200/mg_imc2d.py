"""Drop-in for the reference's MG_IMC/MG_IMC2D.py multigroup time-step API (geometry 'xy'
or 'rz'; a 1-D slab is 'xy' with one cell in y), on the B200 engine.

Same entry points, argument names, defaults, return values and info keys as
MG_IMC/MG_IMC2D.py:1409 (init_simulation), :1635 (step) and :2125 (run_simulation).
Group Planck fractions come from the engine's own incomplete-Planck-integral series (the
reference imports them from an external `planck_integrals` extension, or splits energy
equally across groups without it, MG_IMC/MG_IMC2D.py:60-94).
Differences from the reference, all deliberate:
  - Philox random streams keyed by `seed`;
  - right/top face sources start inside the last cell (the reference places them at index
    nx / ny, where they are lost at once, MG_IMC/MG_IMC2D.py:424-441 with :840-852);
  - a reflection at the -x (-r) face puts the particle back in cell 0 (the reference keeps
    index -1 and loses it on the next event, MG_IMC/MG_IMC2D.py:916-919);
  - material emission removes from each cell its nominal emission energy scaled so the total
    equals the issued particle energy exactly (FP32 weights);
  - info['ledger'] adds the FP64 energy-balance closure.
"""
from __future__ import annotations

import time as _time

import numpy as np
import torch

from . import _lib
from ._gray import GrayState, _host_copy, _law, _same, _staged, check_partition, face_temperatures
from .partition import local_count, sum_scalars, sum_tensors, summary_totals, world_of
from .engine import A_RAD, C_LIGHT, Engine
from .materials import evaluate, evaluate_groups

__c = 29.98
__a = 0.01372


def _cell_volumes(edges1, edges2, geometry):
    if geometry == "xy":
        return np.diff(edges1)[:, None] * np.diff(edges2)[None, :]
    if geometry == "rz":
        return np.pi * (edges1[1:] ** 2 - edges1[:-1] ** 2)[:, None] * np.diff(edges2)[None, :]
    raise ValueError(f"Unknown geometry: {geometry}")


def planck_fractions(energy_edges, T) -> np.ndarray:
    """Normalised group fractions b*_g(T) on the host, shape (G,) + T.shape (used for the
    particle-budget estimate of Ntotal); the device computes the same series per cell."""
    e = np.asarray(energy_edges, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)

    def F(x):
        x = np.asarray(x, dtype=np.float64)
        out = np.zeros_like(x)
        c = 15.0 / np.pi ** 4
        small = (x > 0) & (x < 1.0)
        xs = x[small]
        B = [1.0, -0.5, 1 / 6, 0, -1 / 30, 0, 1 / 42, 0, -1 / 30, 0, 5 / 66, 0, -691 / 2730, 0, 7 / 6, 0,
             -3617 / 510, 0, 43867 / 798, 0, -174611 / 330]
        acc = np.zeros_like(xs)
        fact = 1.0
        for n in range(21):
            if n > 0:
                fact *= n
            if B[n]:
                acc += B[n] * xs ** (n + 3) / ((n + 3) * fact)
        out[small] = c * acc
        big = x >= 1.0
        out[big] = 1.0 - c * tail(x[big])
        return out

    def tail(x):
        t = np.zeros_like(x)
        for k in range(42, 0, -1):
            ik = 1.0 / k
            t += np.exp(-k * x) * ik * (x ** 3 + ik * (3 * x ** 2 + ik * (6 * x + ik * 6)))
        return t

    def frac(x0, x1):
        # above x = 1 as a difference of tails (1 - F cancels to 0 deep in the Wien tail)
        x0, x1 = np.broadcast_arrays(np.asarray(x0, dtype=np.float64), np.asarray(x1, dtype=np.float64))
        hi = x0 >= 1.0
        out = F(x1) - F(x0)
        out[hi] = 15.0 / np.pi ** 4 * (tail(x0[hi]) - tail(x1[hi]))
        return out

    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        Tpos = np.where(T > 0, T, 1.0)
        f = np.stack([frac(e[g] / Tpos, e[g + 1] / Tpos) for g in range(len(e) - 1)])
    f = np.clip(f, 0.0, None)
    tot = f.sum(axis=0)
    return np.where(tot > 0, f / np.where(tot > 0, tot, 1.0), 0.0)


class SimulationState2DMG(GrayState):
    """Multigroup state: the gray fields plus groups and radiation energy by group."""

    _PARTICLE_2D = dict(GrayState._PARTICLE_2D)

    def __getattr__(self, name):
        if name == "groups":
            return object.__getattribute__(self, "_engine").bank.view("group").cpu().numpy().astype(np.int32)
        return super().__getattr__(name)


def init_simulation(Ntarget, Tinit, Tr_init, edges1, edges2, energy_edges, eos, inv_eos, Ntarget_ic=None,
                    T_emit_floor=0.0, geometry="xy", seed=0x5EED0001, _allreduce=None):
    """_allreduce: a torch.distributed module for a particle-partitioned run
    (radtranbook_b200.partition); every step of the state then takes the same one."""
    rank, world = world_of(_allreduce)
    dist = _allreduce if world > 1 else None
    e1 = np.asarray(edges1, dtype=np.float64)
    e2 = np.asarray(edges2, dtype=np.float64)
    G = len(energy_edges) - 1
    vol = _cell_volumes(e1, e2, geometry)
    eng = Engine(geometry, e1, e2, np.ascontiguousarray(vol.T).reshape(-1), seed=seed, n_groups=G,
                 group_edges=energy_edges, capacity=4 * int(Ntarget) + 1024)
    if world > 1:
        eng.partition(rank, world)
    dev = eng.device
    nx, ny = len(e1) - 1, len(e2) - 1
    state = SimulationState2DMG(eng, 2, (nx, ny), torch.zeros(eng.nc, dtype=torch.float64, device=dev),
                                torch.zeros(eng.nc, dtype=torch.float64, device=dev),
                                torch.zeros(eng.nc, dtype=torch.float64, device=dev), 0.0, 0.0, 0)
    Tg = torch.as_tensor(np.asarray(Tinit, dtype=np.float64), device=dev)
    e = evaluate(eos, Tg, lambda: np.asarray(Tinit, dtype=np.float64), Tg)
    state._e.copy_(state.flat(e))
    state._T.copy_(state.flat(Tg))
    back = evaluate(inv_eos, state.grid(state._e), lambda: state.grid(state._e).cpu().numpy(), Tg)
    assert torch.allclose(back, Tg), "Inverse EOS failed"
    N_ic = Ntarget if Ntarget_ic is None else Ntarget_ic
    tr = state.flat(torch.as_tensor(np.asarray(Tr_init, dtype=np.float64), device=dev))
    eng.init_census(tr, local_count(N_ic, rank, world), T_emit_floor)
    rad = _rad_by_group(eng)
    sum_tensors(dist, [rad])
    state.__dict__["radiation_energy_by_group"] = rad.view(G, ny, nx).transpose(1, 2).cpu().numpy().copy()
    state.__dict__["radiation_energy_by_group_postcomb"] = None
    state._Tr.copy_(torch.pow(rad.sum(0) / A_RAD, 0.25))
    radiation, internal = eng.energy_totals(state._e)
    radiation = sum_scalars(dist, [radiation], dev)[0]
    state.previous_total_energy = internal + radiation
    state.refresh_host()
    return state


def _rad_by_group(eng: Engine) -> torch.Tensor:
    """Census radiation energy density by (group, cell) from the bank's weights, (G, nc)."""
    G, nc = eng.ng, eng.nc
    acc = torch.zeros(G * nc, dtype=torch.float64, device=eng.device)
    if eng.bank.size:
        w = eng.bank.view("weight").double()
        live = w > 0
        idx = (eng.bank.view("cell").long() + nc * eng.bank.view("group").long())[live]
        acc.index_add_(0, idx, w[live])
    return acc.view(G, nc) / eng.vol.view(1, nc)


def _report_buffers(state, eng: Engine, n: int) -> dict:
    """The step's pinned host buffer of n reported doubles (imc_mg_report_fields layout,
    GrayState.host_buffer) and its parts: the radiation energy by group before and after the
    comb, e / T / Tr (the state's host mirrors read them), the boundary and escaped energy by
    group."""
    G, nc = eng.ng, eng.nc
    buf = state.host_buffer(n)
    o = 2 * G * nc + 3 * nc
    object.__setattr__(state, "_hpin", buf[2 * G * nc:o])  # e, T, Tr for take_host_copies
    return {"all": buf, "pre": buf[:G * nc], "post": buf[G * nc:2 * G * nc], "bnd": buf[o:o + G],
            "esc": buf[o + G:o + 2 * G]}


def _report_early(state, eng: Engine) -> tuple:
    """Gather the report's sections that are final before the comb (all but the post-comb
    energies) and copy them into this step's host buffer on the engine's side stream, after
    the work the current stream holds (the material update), so both run beside the comb.
    Returns (the side stream's event after the copies, the buffer's parts)."""
    G, nc = eng.ng, eng.nc
    hb = _report_buffers(state, eng, eng.report_buffer().numel())
    side = eng.side_stream()
    side.wait_stream(torch.cuda.current_stream(eng.device))
    with torch.cuda.stream(side):
        eng.mg_report_fields(state._e, state._T, state._Tr, sections="early")
        hb["pre"].copy_(eng.report_dev[:G * nc], non_blocking=True)
        hb["all"][2 * G * nc:].copy_(eng.report_dev[2 * G * nc:], non_blocking=True)
    done = torch.cuda.Event()
    done.record(side)
    return done, hb


def _law_buffers(state, eng: Engine, sigma: torch.Tensor) -> tuple:
    """The (opacity [g][c], heat capacity [c]) pair the material law kernel writes this step:
    of two pairs, the one the step is not reading."""
    nb = state.__dict__.get("_law_buf")
    if nb is None or nb[0].numel() != eng.ng * eng.nc:
        nb = (torch.empty(eng.ng * eng.nc, dtype=torch.float64, device=eng.device),
              torch.empty(eng.nc, dtype=torch.float64, device=eng.device),
              torch.empty(eng.ng * eng.nc, dtype=torch.float64, device=eng.device),
              torch.empty(eng.nc, dtype=torch.float64, device=eng.device))
        object.__setattr__(state, "_law_buf", nb)
    return nb[:2] if sigma.data_ptr() != nb[0].data_ptr() else nb[2:]


def _boundary_energy_estimate(geometry, e1, e2, Tb, dt, bsf) -> float:
    """Analytic boundary emission for the Ntotal split (MG_IMC/MG_IMC2D.py:1546-1632)."""
    E = 0.0
    names = ("left", "right", "bottom", "top") if geometry == "xy" else ("rmin", "rmax", "zmin", "zmax")
    for q, side in enumerate(names):
        if q < 2:
            centers, widths = 0.5 * (e2[:-1] + e2[1:]), np.diff(e2)
            X = e1[0] if q == 0 else e1[-1]
            area = widths if geometry == "xy" else 2.0 * np.pi * X * widths
            Ts = np.array([bsf(X, c, side) for c in centers]) if bsf is not None else np.full(len(centers), Tb[q])
        else:
            centers = 0.5 * (e1[:-1] + e1[1:])
            Y = e2[0] if q == 2 else e2[-1]
            area = np.diff(e1) if geometry == "xy" else np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)
            Ts = np.array([bsf(c, Y, side) for c in centers]) if bsf is not None else np.full(len(centers), Tb[q])
        Ts = np.where(Ts > 0, Ts, 0.0)
        E += float(np.sum(__a * __c * Ts ** 4 / 4.0 * area * dt))
    return E


def step(state, Ntarget, Nboundary, Nsource, Nmax, T_boundary, dt, edges1, edges2, energy_edges, sigma_a_funcs,
         inv_eos, cv, source, reflect=(False, False, False, False), theta=1.0, use_scalar_intensity_Tr=True,
         conserve_comb_energy=False, geometry="xy", max_events_per_particle=1_000_000, boundary_source_func=None,
         emission_fractions=None, Ntotal=0, Ntotal_T_floor=0.0, particle_budget_fmin=0.1, T_emit_floor=0.0,
         Nmax_growth=0, Nmax_final=None, _timing=False, _allreduce=None):
    if geometry not in ("xy", "rz"):
        raise ValueError(f"Unknown geometry: {geometry}")
    t_step_start = _time.perf_counter()
    eng: Engine = state._engine
    # particle partition (radtranbook_b200.partition): counts are totals, each rank takes its share
    rank, world = check_partition(eng, _allreduce)
    dist = _allreduce if world > 1 else None
    G, nc = eng.ng, eng.nc
    like = state.grid(state._T)
    host_T = lambda: state.temperature  # noqa: E731
    # a material the device evaluates itself (LinearEOS, Constant cv, GroupPowerLawOpacity):
    # the material update, inverse EOS and next step's opacities are one kernel at the step's end
    law = _law(state, sigma_a_funcs, cv, inv_eos) if not conserve_comb_energy else None
    if law is not None and len(sigma_a_funcs) != G:
        raise ValueError(f"{len(sigma_a_funcs)} opacity groups for a {G}-group state")
    nxt = state.__dict__.get("_law_next")
    if law is not None and nxt is not None and _same(nxt[0], (sigma_a_funcs, cv)):
        sig, cvv = nxt[1].view(G, nc), nxt[2]  # evaluated on the device at the end of the last step
    else:
        # host callables' results go up by asynchronous copies from pinned buffers of the state
        sig = evaluate_groups(sigma_a_funcs, like, host_T, like,
                              **_staged(state, "sigma_g", G * nc)).transpose(1, 2).reshape(G, -1)  # (G, nc)
        cvv = state.flat(evaluate(cv, like, host_T, like, **_staged(state, "cv", nc)))
    if emission_fractions is not None:
        eng.emission_fractions = torch.as_tensor(np.asarray(emission_fractions, dtype=np.float64), device=eng.device)
    else:
        eng.emission_fractions = None
    src = None
    if Nsource > 0 and source is not None:
        s = np.asarray(source, dtype=np.float64)
        if s.ndim == 0:
            s = np.broadcast_to(s, like.shape)
        if s.ndim == 2:  # gray source goes to the lowest group (MG_IMC/MG_IMC2D.py:1111-1118)
            s3 = np.zeros((G,) + s.shape)
            s3[0] = s
            s = s3
        if s.max() > 0:
            src = torch.stack([state.flat(torch.as_tensor(s[g], device=eng.device)) for g in range(G)]).reshape(-1)
    e1, e2 = np.asarray(edges1, dtype=np.float64), np.asarray(edges2, dtype=np.float64)
    E_bc_est = E_mat_est = float("nan")
    if Ntotal > 0:
        Tb = [T_boundary[q](state.time) if callable(T_boundary[q]) else T_boundary[q] for q in range(4)]
        E_bc_est = _boundary_energy_estimate(geometry, e1, e2, Tb, dt, boundary_source_func)
        T = state.temperature
        sig_h = sig.view(G, *reversed(like.shape)).transpose(1, 2).cpu().numpy()
        b = planck_fractions(energy_edges, T)
        sP = np.sum(sig_h * b, axis=0)
        beta = 4.0 * __a * T ** 3 / np.broadcast_to(np.asarray(cv(T) if not getattr(cv, "_imc_device", False)
                                                                 else state.grid(cvv).cpu().numpy()), T.shape)
        f = np.clip(1.0 / (1.0 + theta * beta * sP * __c * dt), 0.0, 1.0)
        vol = _cell_volumes(e1, e2, geometry)
        ce = np.sum(sig_h * f * b, axis=0) * __a * __c * T ** 4 * dt * vol
        if Ntotal_T_floor > 0.0:
            ce = np.where(T > Ntotal_T_floor, ce, 0.0)
        E_mat_est = float(np.sum(ce))
        tot = E_bc_est + E_mat_est
        frac_bc = E_bc_est / tot if tot > 0 else 0.5
        fmin = float(np.clip(particle_budget_fmin, 0.0, 0.5))
        frac_bc = float(np.clip(frac_bc, fmin, 1.0 - fmin))
        Nboundary = int(round(Ntotal * frac_bc))
        Ntarget = Ntotal - Nboundary
    cache = state.__dict__.setdefault("_face_cache", {})
    faces = face_temperatures(2, geometry, T_boundary, state.time, e1, e2, boundary_source_func, eng.device, cache)
    refl = tuple(reflect) + (False,) * (4 - len(reflect))
    t_eval = _time.perf_counter()
    nt_l, nb_l, ns_l = (local_count(n, rank, world) for n in (Ntarget, Nboundary, Nsource))
    nmax_l = local_count(Nmax, rank, world) if Nmax > 0 else Nmax
    if Nmax_final is not None and Nmax_growth > 0:  # size the banks once for the whole schedule
        eng.reserve(local_count(max(int(Nmax_final), Nmax), rank, world), nt_l + 4 * nb_l + ns_l)
    eng.transport_async(state._T, sig.reshape(-1).contiguous(), cvv, src, state.count, dt, theta, nt_l, nb_l, ns_l,
                        faces, refl, max_events=max_events_per_particle, rz_linear_source=False,
                        t_emit_floor=T_emit_floor)
    sum_tensors(dist, [eng.dep, eng.si, eng.emitted, eng.boundary_group, eng.escaped_group])
    if law is not None:
        sig_next, cv_next = _law_buffers(state, eng, sig)
        eng.material_update_law(state._e, state._Tr, state._T, law[0], sig_next, cv_next)
        state.__dict__["_law_next"] = ((sigma_a_funcs, cv), sig_next, cv_next)
    else:
        state.__dict__.pop("_law_next", None)
        eng.material_update(state._e, state._Tr)
    # with the device law (and no comb discrepancy booked into e) every reported field but the
    # post-comb energies is final now: gathered and copied to the host beside the comb
    early = _report_early(state, eng) if law is not None and not conserve_comb_energy else None
    # the comb is queued next (the host prepares the by-group fields while it runs); it also
    # writes the energy after it per (group, cell) bin: the post-comb radiation energy by
    # group without a pass over the new census
    eng.comb_async(nmax_l, state.count, state._e, per_group=True, write_after=True)
    nx, ny = state._shape

    def to_grid3(x):  # device (G, nc) in flat cell order -> (G, nx, ny) C order, flattened
        return x.reshape(G, ny, nx).transpose(1, 2).reshape(-1)

    sum_tensors(dist, [eng.comb_after])
    if conserve_comb_energy:
        sum_tensors(dist, [eng.disc])
        state._e.add_(eng.disc.view(G, nc).sum(0) / eng.vol)
    if law is None:
        Tn = evaluate(inv_eos, state.grid(state._e), lambda: _host_copy(state.grid(state._e)), like,
                      **_staged(state, "T_new", nc))
        state._T.copy_(state.flat(Tn))
    # every reported field in the reference's layout in one device buffer (one kernel), then
    # one copy into a fresh pinned buffer that the host arrays view
    if early is None:
        hb = _report_buffers(state, eng, eng.mg_report_fields(state._e, state._T, state._Tr))
        copies = [(eng.report_dev, hb["all"])]
    else:
        hb = early[1]
        eng.mg_report_fields(None, None, None, sections="post")
        copies = [(eng.report_dev[G * nc:2 * G * nc], hb["post"])]
    ms_src, ms_tr = eng.phase_times()  # waits for the tracking only (the comb still runs)
    try:
        sm = eng.fetch(copies)
    except _lib.ImcError as ex:
        if ex.status == 3:
            raise AssertionError("non-finite or non-positive material state") from ex
        raise
    if early is not None:
        early[0].synchronize()  # done long before the comb
    if not use_scalar_intensity_Tr:
        pre = eng.spare
        acc = torch.zeros(G * nc, dtype=torch.float64, device=eng.device)
        w = pre.view("weight").double()
        live = w > 0
        acc.index_add_(0, (pre.view("cell").long() + nc * pre.view("group").long())[live], w[live])
        sum_tensors(dist, [acc])
        rad_pre = acc.view(G, nc) / eng.vol.view(1, nc)
        state._Tr.copy_(torch.pow(rad_pre.sum(0) / A_RAD, 0.25))
        state.refresh_host()
        hb["pre"].copy_(to_grid3(rad_pre))
        eTT = []
    else:
        eTT = state.take_host_copies(publish=False)
    # the comb ran again after an overflow (on any rank): rebuild from the new census
    if sum_scalars(dist, [float(eng.comb_repeated)], eng.device)[0] > 0:
        post = _rad_by_group(eng)
        sum_tensors(dist, [post])
        hb["post"].copy_(to_grid3(post))
    internal = float(sm.internal_energy)  # the same material state on every rank
    tot = summary_totals(dist, sm, eng.bank.size, eng.device)  # summed over the ranks of a partition
    rad = tot["rad"]
    comb_disc = tot["comb_before"] - rad
    if conserve_comb_energy:
        internal += comb_disc
    boundary_emission = tot["e_side_total"]
    boundary_loss = tot["escaped_total"]
    source_emission = tot["source_emission"]
    total = internal + rad
    dE = total - state.previous_total_energy
    residual = dE - boundary_emission + boundary_loss - source_emission
    closure = residual + (0.0 if conserve_comb_energy else comb_disc)
    state.time = state.time + dt
    state.previous_total_energy = total
    state.count += 1

    def grid3(h):  # this step's pinned host buffer, already (G, nx, ny): the array views it
        return h.numpy().reshape(G, nx, ny)

    rad_group_pre, rad_group_post, bnd_group, esc_group, *eTT = state.publish(
        [grid3(hb["pre"]), grid3(hb["post"]), hb["bnd"].numpy(), hb["esc"].numpy()] + eTT)
    if eTT:
        state.set_host_mirrors(eTT)
    _lib.TRANSFER["d2h"] += 8 * (2 * G * nc + 2 * G)
    state.__dict__["radiation_energy_by_group"] = rad_group_pre
    state.__dict__["radiation_energy_by_group_postcomb"] = rad_group_post
    stats = tot["stats"]
    t_end = _time.perf_counter()
    n_tr = tot["n_bank"]
    ev = int(stats[_lib.STAT_EVENTS])
    info = {
        "time": state.time,
        "temperature": state.temperature,
        "radiation_temperature": state.radiation_temperature,
        "radiation_energy_by_group": rad_group_pre,
        "radiation_energy_by_group_postcomb": rad_group_post,
        "N_particles": tot["n_particles"],
        "N_boundary": Nboundary,
        "N_target": Ntarget,
        "particle_budget_fmin": float(np.clip(particle_budget_fmin, 0.0, 0.5)),
        "E_boundary_est": E_bc_est,
        "E_material_est": E_mat_est,
        "total_energy": total,
        "total_internal_energy": internal,
        "total_radiation_energy": rad,
        "boundary_emission": boundary_emission,
        "boundary_emission_by_group": bnd_group,
        "boundary_emission_by_side": tot["e_side"],
        "boundary_loss": boundary_loss,
        "boundary_outgoing": boundary_loss,
        "boundary_outgoing_by_group": esc_group,
        "boundary_outgoing_by_side": tot["escaped"],
        "source_emission": source_emission,
        "incoming_energy_total": boundary_emission + source_emission,
        "outgoing_energy_total": boundary_loss,
        "dE_system": dE,
        "energy_expected_dE": boundary_emission + source_emission - boundary_loss,
        "energy_residual": residual,
        "energy_loss": residual,
        "Nmax_next": (min(Nmax + Nmax_growth, Nmax_final) if Nmax_final is not None else Nmax + Nmax_growth)
        if Nmax_growth > 0 else Nmax,
        "ledger": {"comb_discrepancy": comb_disc, "closure": closure,
                   "relative_closure": closure / max(abs(total), 1e-300),
                   "emission": tot["emission_total"],
                   "weight_floor": 1e-10 * tot["weight_sum"] / max(n_tr, 1)},
        "profiling": {
            "phase_times_s": {
                "sampling": (t_eval - t_step_start) + ms_src * 1e-3,
                "transport": ms_tr * 1e-3,
                "postprocess": max(t_end - t_eval - (ms_src + ms_tr) * 1e-3, 0.0),
                "total": t_end - t_step_start,
            },
            "transport_events": {
                "total": ev,
                "boundary_crossings": int(stats[_lib.STAT_BOUNDARY]),
                "absorption_continue_events": int(stats[_lib.STAT_SCATTER]),
                "census_events": int(stats[_lib.STAT_CENSUS]),
                "absorption_capture_events": 0,
                "weight_floor_kills": int(stats[_lib.STAT_FLOOR]),
                "reflections": int(stats[_lib.STAT_REFLECT]),
                "event_cap_hits": int(stats[_lib.STAT_CAP]),
                "avg_events_per_particle": ev / max(n_tr, 1),
                "n_particles_transported": n_tr,
            },
        },
    }
    return state, info


def run_simulation(Ntarget, Nboundary, Nsource, Nmax, Tinit, Tr_init, T_boundary, dt, edges1, edges2, energy_edges,
                   sigma_a_funcs, eos, inv_eos, cv, source, final_time, reflect=(False, False, False, False),
                   output_freq=1, theta=1.0, use_scalar_intensity_Tr=True, Ntarget_ic=None,
                   conserve_comb_energy=False, geometry="xy", max_events_per_particle=1_000_000,
                   emission_fractions=None, T_emit_floor=0.0, Nmax_growth=0, Nmax_final=None, seed=0x5EED0001):
    """The time loop of MG_IMC/MG_IMC2D.py:2125-2259: steps of min(dt, time left) until
    final_time (within max(1e-15, 1e-12 max(final_time, 1))); every output_freq-th step and the
    last one append the step's info, with 'cumulative_energy_residual' and
    'net_boundary_energy' added, to the history.  Returns (history, state)."""
    state = init_simulation(Ntarget, Tinit, Tr_init, edges1, edges2, energy_edges, eos, inv_eos,
                            Ntarget_ic=Ntarget_ic, T_emit_floor=T_emit_floor, geometry=geometry, seed=seed)
    history = []
    t = 0.0
    step_count = 0
    cumulative_residual = 0.0
    time_tol = max(1e-15, 1e-12 * max(final_time, 1.0))
    while t < final_time - time_tol:
        step_dt = min(dt, final_time - t)
        if step_dt <= time_tol:
            break
        state, info = step(state, Ntarget, Nboundary, Nsource, Nmax, T_boundary, step_dt, edges1, edges2,
                           energy_edges, sigma_a_funcs, inv_eos, cv, source, reflect=reflect, theta=theta,
                           use_scalar_intensity_Tr=use_scalar_intensity_Tr, conserve_comb_energy=conserve_comb_energy,
                           geometry=geometry, max_events_per_particle=max_events_per_particle,
                           emission_fractions=emission_fractions, T_emit_floor=T_emit_floor,
                           Nmax_growth=Nmax_growth, Nmax_final=Nmax_final)
        t = state.time
        Nmax = info["Nmax_next"]
        step_count += 1
        cumulative_residual += info["energy_residual"]
        if step_count % output_freq == 0 or (final_time - t) < time_tol:
            info["cumulative_energy_residual"] = cumulative_residual
            info["net_boundary_energy"] = info["boundary_emission"] - info["boundary_outgoing"]
            for k in ("radiation_energy_by_group", "radiation_energy_by_group_postcomb", "temperature",
                      "radiation_temperature"):
                info[k] = np.array(info[k])  # a kept record holds ordinary memory, not a pinned step buffer
            history.append(info)
    return history, state


def tune(state, grid=None, repeats=2):
    from ._gray import tune as _tune

    return _tune(state, grid=grid, repeats=repeats)
