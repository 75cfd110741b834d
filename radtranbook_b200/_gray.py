"""Shared core of the gray drop-in step (IMC1D / IMC2D signatures).

One call of :func:`gray_step` is one reference time step (IMC/IMC1D.py:908-1124,
IMC/IMC2D.py:1591-1897): material callables are evaluated on the temperature field, the
device engine plans and samples the sources, tracks the bank to census, updates the
material energy, combs the census, and the energy ledger is closed in FP64.
"""
from __future__ import annotations

import time as _time
import weakref

import numpy as np
import torch

from . import _lib
from .engine import A_RAD, C_LIGHT, Engine
from .materials import evaluate, is_device
from .partition import local_count, sum_tensors, summary_totals, world_of


class GrayState:
    """Device-resident state with the reference's field names available as NumPy arrays.

    Material fields (internal_energy, temperature, radiation_temperature) are mirrored to the
    host after every step (O(cells)); particle fields are copied from the device bank when
    read (O(particles), only for drivers that inspect or checkpoint the census).
    """

    _PARTICLE_1D = {"weights": "weight", "mus": "dir1", "times": "time", "positions": "pos1"}
    _PARTICLE_2D = {"weights": "weight", "dir1": "dir1", "dir2": "dir2", "times": "time", "pos1": "pos1", "pos2": "pos2"}

    def __init__(self, engine: Engine, dim: int, shape: tuple, e: torch.Tensor, T: torch.Tensor, Tr: torch.Tensor,
                 time: float, previous_total_energy: float, count: int = 0):
        object.__setattr__(self, "_engine", engine)
        object.__setattr__(self, "_dim", dim)
        object.__setattr__(self, "_shape", shape)
        object.__setattr__(self, "_e", e)
        object.__setattr__(self, "_T", T)
        object.__setattr__(self, "_Tr", Tr)
        object.__setattr__(self, "_host", {})
        self.time = time
        self.previous_total_energy = previous_total_energy
        self.count = count

    # ---- layout helpers: flat c = i + nx*j <-> reference (nx, ny) ----
    def grid(self, flat: torch.Tensor) -> torch.Tensor:
        if self._dim == 1:
            return flat
        nx, ny = self._shape
        return flat.view(ny, nx).t()

    def flat(self, grid: torch.Tensor) -> torch.Tensor:
        if self._dim == 1:
            return grid.reshape(-1).contiguous()
        return grid.t().contiguous().view(-1)

    # ---- the step's host arrays ----
    # A step's reported arrays view a pinned buffer that the step's one device-to-host copy
    # filled: a fresh buffer from torch's caching pinned allocator each step, so no host copy
    # is made, and a buffer returns to the cache once nothing views it.  A caller that keeps
    # the arrays of every step (a list of info dicts) would make the allocator pin new memory
    # each step; once the arrays of a step are still alive two steps later (the caller's
    # current info holds the previous step's), the state switches to one buffer of its own,
    # overwritten each step, and returns copies.
    def host_buffer(self, n: int) -> torch.Tensor:
        """Pinned buffer of n doubles for this step's reported arrays."""
        if not self.__dict__.get("_host_copy_mode"):
            return torch.empty(n, dtype=torch.float64, pin_memory=True)
        own = self.__dict__.get("_host_own")
        if own is None or own.numel() < n:
            own = torch.empty(n, dtype=torch.float64, pin_memory=True)
            object.__setattr__(self, "_host_own", own)
        return own[:n]

    def publish(self, arrays: list) -> list:
        """The arrays this step returns (views of host_buffer): copies in copy mode; else the
        views, with weak references kept to see whether the caller keeps them."""
        if self.__dict__.get("_host_copy_mode"):
            return [np.array(a) for a in arrays]
        refs = self.__dict__.setdefault("_host_refs", [])
        refs.append([weakref.ref(a) for a in arrays])
        if len(refs) > 2 and any(r() is not None for r in refs.pop(0)):
            object.__setattr__(self, "_host_copy_mode", True)
        return arrays

    def host_copies(self):
        """(device, pinned host) pair for the end-of-step copy of e, T and Tr: the three fields
        stacked on the device in the reference's layout ((nx, ny) in 2-D), one copy into the
        step's host buffer."""
        src = torch.stack([self.grid(self._e), self.grid(self._T), self.grid(self._Tr)]).reshape(-1)
        pin = self.host_buffer(src.numel())
        object.__setattr__(self, "_hpin", pin)
        return [(src, pin)]

    def host_copies_early(self) -> "torch.cuda.Event":
        """Queue the copy of host_copies() on a side stream of the engine, after the work the
        current stream holds so far (the material update), so that it runs beside the work
        queued next (the comb).  Returns the side stream's event after the copy: the caller
        synchronises the host on it before reading the buffer and before the step returns
        (nothing that changes e, T or Tr is queued before then)."""
        eng = self._engine
        side = eng.side_stream()
        main = torch.cuda.current_stream(eng.device)
        side.wait_stream(main)
        with torch.cuda.stream(side):
            for d, h in self.host_copies():
                h.copy_(d, non_blocking=True)
        done = torch.cuda.Event()
        done.record(side)
        return done

    def take_host_copies(self, publish: bool = True) -> list:
        """Host mirrors of e, T and Tr from the buffer filled by the last fetch (no device
        access); publish=False leaves publishing them (with other arrays) to the caller, which
        then sets the mirrors.  Returns the three arrays."""
        nc = self._engine.nc
        a = self._hpin.numpy()
        shape = (nc,) if self._dim == 1 else tuple(self._shape)
        arrs = [a[:nc].reshape(shape), a[nc:2 * nc].reshape(shape), a[2 * nc:].reshape(shape)]
        _lib.TRANSFER["d2h"] += 3 * 8 * nc
        if publish:
            arrs = self.publish(arrs)
            self.set_host_mirrors(arrs)
        return arrs

    def set_host_mirrors(self, arrs: list) -> None:
        h = self._host
        h["internal_energy"], h["temperature"], h["radiation_temperature"] = arrs

    def refresh_host(self) -> None:
        h = self._host
        h["internal_energy"] = self.grid(self._e).cpu().numpy().copy()
        h["temperature"] = self.grid(self._T).cpu().numpy().copy()
        h["radiation_temperature"] = self.grid(self._Tr).cpu().numpy().copy()
        _lib.TRANSFER["d2h"] += 3 * 8 * self._engine.nc

    def __getattr__(self, name):
        host = object.__getattribute__(self, "_host")
        if name in ("internal_energy", "temperature", "radiation_temperature"):
            if name not in host:
                self.refresh_host()
            return host[name]
        pmap = self._PARTICLE_1D if self._dim == 1 else self._PARTICLE_2D
        bank = object.__getattribute__(self, "_engine").bank
        if name in pmap:
            return bank.view(pmap[name]).double().cpu().numpy()
        if name in ("cell_indices", "cell_i", "cell_j"):
            c = bank.view("cell").long().cpu().numpy()
            nx = self._shape[0]
            if name == "cell_indices" or name == "cell_i":
                return c % nx if self._dim == 2 else c
            return c // nx
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in ("internal_energy", "temperature"):
            t = torch.as_tensor(np.asarray(value, dtype=np.float64), device=self._engine.device)
            (self._e if name == "internal_energy" else self._T).copy_(self.flat(t))
            self._host.pop(name, None)
            self.__dict__.pop("_law_next", None)  # the next step's opacity follows a new T
            self.__dict__.pop("_host_next", None)
            return
        object.__setattr__(self, name, value)


def _pinned(state, key: str, n: int) -> torch.Tensor:
    """A pinned host buffer of n doubles kept on the state (allocated once)."""
    bufs = state.__dict__.get("_pinned")
    if bufs is None:
        bufs = {}
        object.__setattr__(state, "_pinned", bufs)
    if key not in bufs or bufs[key].numel() != n:
        bufs[key] = torch.empty(n, dtype=torch.float64, pin_memory=True)
    return bufs[key]


def _staged(state, key: str, n: int) -> dict:
    """A pinned host buffer and its device twin (n doubles each) kept on the state: the
    stage / stage_dev pair of materials.evaluate, so a host callable's result reaches the
    device without a device allocation per step."""
    devs = state.__dict__.get("_stage_dev")
    if devs is None:
        devs = {}
        object.__setattr__(state, "_stage_dev", devs)
    if key not in devs or devs[key].numel() != n:
        devs[key] = torch.empty(n, dtype=torch.float64, device=state._engine.device)
    return {"stage": _pinned(state, key, n), "stage_dev": devs[key]}


def _same(key, objs: tuple) -> bool:
    """Whether a cached value was made for these objects: identity, not equality.  The cache
    holds the objects themselves, so a freed callable's id cannot be reused while it lives."""
    return key is not None and len(key) == len(objs) and all(a is b for a, b in zip(key, objs))


def _upload_flat(state, values, stage: torch.Tensor, dev: torch.Tensor) -> torch.Tensor:
    """Copy a field given in the reference's layout ((nx, ny) in 2-D, or a scalar) to `dev`
    in the engine's flat cell order c = i + nx*j: the reordering is done on the host, into
    the pinned `stage`, so the asynchronous upload lands in place (no device transpose and
    no device allocation).  Returns the first nc entries of dev."""
    n = state._engine.nc
    host = stage[:n].numpy()
    v = np.asarray(values, dtype=np.float64)
    if state._dim == 1:
        np.copyto(host, np.broadcast_to(v, (n,)))
    else:
        nx, ny = state._shape
        np.copyto(host.reshape(ny, nx), np.broadcast_to(v, (nx, ny)).T)
    _lib.TRANSFER["h2d"] += n * 8
    out = dev[:n]
    out.copy_(stage[:n], non_blocking=True)
    return out


def _field_flat(state, fn, like: torch.Tensor, host_fn, key: str) -> torch.Tensor:
    """A material callable on the temperature field, as a flat device field.  A device
    callable runs on `like`; a host callable on host_fn()'s array, its result uploaded from
    the state's pinned stage (refilled only next step, after this step's synchronisation)."""
    if is_device(fn):
        return state.flat(evaluate(fn, like, host_fn, like))
    st = _staged(state, key, state._engine.nc)
    return _upload_flat(state, fn(host_fn()), st["stage"], st["stage_dev"])


def _host_copy(t: torch.Tensor) -> np.ndarray:
    a = t.cpu().numpy()
    _lib.TRANSFER["d2h"] += a.nbytes
    return a


def check_partition(eng: Engine, dist) -> tuple[int, int]:
    """(rank, world) of a partitioned step; the state must have been initialised for it."""
    if dist is None and eng.world == 1:
        return 0, 1
    rank, world = world_of(dist)
    if (eng.rank, eng.world) != (rank, world):
        raise ValueError("the state was initialised for rank %d of %d, the step runs as rank %d of %d "
                         "(pass the same _allreduce to init_simulation)" % (eng.rank, eng.world, rank, world))
    return rank, world


def face_temperatures(dim: int, geometry: str, T_boundary, time_now: float, e1: np.ndarray, e2: np.ndarray,
                      boundary_source_func, device, cache: dict) -> list:
    """Per-face-cell boundary temperatures for the four sides (None = no source).

    1-D: sides 0/1 = left/right (one face cell).  2-D: T_boundary order (min-1, max-1,
    min-2, max-2) as IMC/IMC2D.py:1617-1620; with boundary_source_func the temperature of
    each face cell is the callable at its centre (IMC/IMC2D.py:183-191, 353-396).
    """
    out = [None, None, None, None]
    nsides = 2 if dim == 1 else 4
    names = {"xy": ("left", "right", "bottom", "top"), "rz": ("rmin", "rmax", "zmin", "zmax")}
    for q in range(nsides):
        Tb = T_boundary[q] if q < len(T_boundary) else 0.0
        Tb = Tb(time_now) if callable(Tb) else Tb
        if dim == 2 and boundary_source_func is not None:
            key = ("func", id(boundary_source_func), q)
            if key not in cache:
                side = names[geometry][q]
                if q < 2:
                    X = e1[0] if q == 0 else e1[-1]
                    centers = 0.5 * (e2[:-1] + e2[1:])
                    vals = np.array([boundary_source_func(X, c, side) for c in centers], dtype=np.float64)
                else:
                    Y = e2[0] if q == 2 else e2[-1]
                    centers = 0.5 * (e1[:-1] + e1[1:])
                    vals = np.array([boundary_source_func(c, Y, side) for c in centers], dtype=np.float64)
                cache[key] = torch.as_tensor(vals, device=device) if np.any(vals > 0) else None
            out[q] = cache[key]
            continue
        if Tb is None or not (float(Tb) > 0.0):
            continue
        n = 1 if dim == 1 else (len(e2) - 1 if q < 2 else len(e1) - 1)
        key = ("T", q, float(Tb), n)
        if key not in cache:
            cache[key] = torch.full((n,), float(Tb), dtype=torch.float64, device=device)
        out[q] = cache[key]
    return out


def gray_step(state: GrayState, *, Ntarget, Nboundary, Nsource, Nmax, T_boundary, dt, sigma_a_func, inv_eos, cv,
              source, reflect, theta, use_scalar_intensity_Tr, conserve_comb_energy, T_emit_floor=0.0,
              rz_linear_source=True, max_events=0, boundary_source_func=None, geometry="slab",
              allreduce=None, method="fc", cf_fastpath=0.0):
    """One time step (method 'fc' Fleck-Cummings, 'cf' Carter-Forest).  With device material
    callables the host synchronises once, at the end (sizes, energies and statistics come
    back in one device summary).

    allreduce: a torch.distributed module for a particle-partitioned step (the process
    parallelism of IMC/IMC1DMPI.py and IMC/IMC2DMPI.py, radtranbook_b200.partition): Ntarget,
    Nboundary, Nsource and Nmax are totals, each rank tracks its share with its own Philox id
    range and 1/world of the source energy, the per-cell deposition, intensity and emission
    are summed over the ranks before the material update (so every rank holds the same
    material state), each rank combs its census to its share of Nmax, and the ledger terms
    are summed.  The state must come from init_simulation with the same allreduce."""
    t_step_start = _time.perf_counter()
    eng: Engine = state._engine
    rank, world = check_partition(eng, allreduce)
    dist = allreduce if world > 1 else None
    if world > 1:
        Ntarget, Nboundary, Nsource = (local_count(n, rank, world) for n in (Ntarget, Nboundary, Nsource))
        Nmax = local_count(Nmax, rank, world) if Nmax > 0 else Nmax
    dim = state._dim
    like = None  # the reference-layout view of T, for host callables only
    host_T = lambda: state.temperature  # noqa: E731
    # a material the device evaluates itself (LinearEOS, Constant, PowerLawOpacity): the
    # material update, inverse EOS and next step's opacity are one kernel at the step's end
    law = _law(state, sigma_a_func, cv, inv_eos) if not conserve_comb_energy else None
    nxt = state.__dict__.get("_law_next")
    hn = state.__dict__.pop("_host_next", None)
    if law is not None and nxt is not None and _same(nxt[0], (sigma_a_func, cv)):
        sigma, cvv = nxt[1], nxt[2]  # evaluated on the device at the end of the last step
    elif law is None and hn is not None and _same(hn[0], (sigma_a_func, cv)) and hn[1] == state.count:
        sigma, cvv = hn[2], hn[3]  # host callables evaluated at this T while the last comb ran
    else:
        # host callables' results go up by asynchronous copies from pinned buffers of the state
        # (refilled only next step, after this step's end-of-step synchronisation)
        like = state.grid(state._T)
        sigma = _field_flat(state, sigma_a_func, like, host_T, "sigma")
        cvv = _field_flat(state, cv, like, host_T, "cv")
    src = None
    if Nsource > 0 and source is not None:
        src_t = source.double() if isinstance(source, torch.Tensor) else torch.as_tensor(
            np.asarray(source, dtype=np.float64))
        if float(src_t.max()) > 0:
            src = state.flat(src_t.to(eng.device))
    cache = state.__dict__.setdefault("_face_cache", {})
    if "edges" not in cache:
        cache["edges"] = (eng.e1.cpu().numpy(), eng.e2.cpu().numpy())
    faces = face_temperatures(dim, geometry, T_boundary, state.time, cache["edges"][0], cache["edges"][1],
                              boundary_source_func, eng.device, cache)
    refl = tuple(reflect) + (False,) * (4 - len(reflect))
    t_eval = _time.perf_counter()
    eng.transport_async(state._T, sigma, cvv, src, state.count, dt, theta, Ntarget, Nboundary, Nsource, faces,
                        refl, max_events=max_events, rz_linear_source=rz_linear_source, t_emit_floor=T_emit_floor,
                        method=_lib.METHOD_CARTER_FOREST if method == "cf" else _lib.METHOD_FLECK_CUMMINGS,
                        cf_fastpath=cf_fastpath)
    # partition: the per-cell tallies of all ranks (the step's only data exchange)
    sum_tensors(dist, [eng.dep, eng.si, eng.emitted])

    # material update: e += dep - emitted/V ; Tr from the path-length intensity.  The comb
    # does not need T: with a host inv_eos (and the comb discrepancy not booked into e), e is
    # copied out before the comb is queued, so the host evaluation overlaps the comb.
    if law is not None:
        nb = state.__dict__.get("_law_buf")
        if nb is None or nb[0].numel() != eng.nc:
            nb = tuple(torch.empty(eng.nc, dtype=torch.float64, device=eng.device) for _ in range(4))
            object.__setattr__(state, "_law_buf", nb)
        # two buffer pairs: the step reads one pair (its sigma, cv) while it writes the other
        pair = nb[:2] if sigma.data_ptr() != nb[0].data_ptr() else nb[2:]
        eng.material_update_law(state._e, state._Tr, state._T, law[0], pair[0], pair[1])
        state.__dict__["_law_next"] = ((sigma_a_func, cv), pair[0], pair[1])
    else:
        state.__dict__.pop("_law_next", None)
        eng.material_update(state._e, state._Tr)
    # e and Tr are final now (no comb discrepancy booked into e), and so is T with the device
    # law: their copy to the host runs on a side stream beside the comb.  A host inv_eos then
    # evaluates T from that copy of e while the comb runs.
    host_inv = law is None and not conserve_comb_energy and not is_device(inv_eos)
    early = state.host_copies_early() if (law is not None and not conserve_comb_energy) or host_inv else None
    t_up = None
    eng.comb_async(Nmax, state.count, state._e)
    if conserve_comb_energy:
        sum_tensors(dist, [eng.disc])
        state._e.add_(eng.disc[: eng.nc] / eng.vol)
    if law is None and like is None:
        like = state.grid(state._T)
    if law is not None:
        pass  # T = e / cv came with the material update
    elif host_inv:
        # the early copy holds e, (the old) T and Tr in the reference's layout: T = inv_eos(e)
        # replaces the T slot (the host mirror this step returns) and goes up to the device on
        # the side stream (nothing queued on the current stream reads T before the step ends)
        early.synchronize()
        n = eng.nc
        shape = (n,) if state._dim == 1 else tuple(state._shape)
        hp = state._hpin.numpy()
        Tn = np.asarray(inv_eos(hp[:n].reshape(shape)), dtype=np.float64)
        np.copyto(hp[n:2 * n].reshape(shape), np.broadcast_to(Tn, shape))
        side = eng.side_stream()
        with torch.cuda.stream(side):
            _upload_flat(state, Tn, _pinned(state, "T_new", n), state._T)
            if not is_device(sigma_a_func) and not is_device(cv):
                # the next step's opacity and heat capacity at this T (the host mirror it
                # returns), while the comb runs; the next step takes them if it passes the same
                # callables and nothing has set T since (this step's own inputs are read)
                T_ref = hp[n:2 * n].reshape(shape)
                st_s, st_c = _staged(state, "sigma", n), _staged(state, "cv", n)
                sig_n = _upload_flat(state, sigma_a_func(T_ref), st_s["stage"], st_s["stage_dev"])
                cv_n = _upload_flat(state, cv(T_ref), st_c["stage"], st_c["stage_dev"])
                state.__dict__["_host_next"] = ((sigma_a_func, cv), state.count + 1, sig_n, cv_n)
        t_up = torch.cuda.Event()
        t_up.record(side)
    else:
        Tn = evaluate(inv_eos, state.grid(state._e), lambda: _host_copy(state.grid(state._e)), like)
        state._T.copy_(state.flat(Tn))
    copies = state.host_copies() if early is None else ()
    # the phase times wait for the tracking only: read while the comb still runs on the device
    ms_src, ms_tr = eng.phase_times()
    try:
        sm = eng.fetch(copies)
    except _lib.ImcError as ex:
        if ex.status == 3:
            raise AssertionError("Fleck factor out of bounds / non-positive temperature in material state") from ex
        raise
    if early is not None:
        early.synchronize()  # done long before the comb
    if t_up is not None:
        t_up.synchronize()
    t_post = _time.perf_counter()
    pre_comb = eng.spare  # the tracked (pre-comb) bank after the swap
    if not use_scalar_intensity_Tr:
        live = pre_comb.view("weight") > 0
        rad_c = torch.zeros(eng.nc, dtype=torch.float64, device=eng.device)
        rad_c.index_add_(0, pre_comb.view("cell")[live].long(), pre_comb.view("weight")[live].double())
        sum_tensors(dist, [rad_c])
        state._Tr.copy_(torch.pow(rad_c / eng.vol / A_RAD, 0.25))
    internal = float(sm.internal_energy)  # the same material state on every rank
    # ledger terms and counts (summed over the ranks of a partition)
    tot = summary_totals(dist, sm, eng.bank.size, eng.device)
    rad, stats = tot["rad"], tot["stats"]
    comb_disc = tot["comb_before"] - rad
    boundary_emission, boundary_loss = tot["e_side_total"], tot["escaped_total"]
    source_emission, emission_total, weight_sum = tot["source_emission"], tot["emission_total"], tot["weight_sum"]
    n_particles, n_tr = tot["n_particles"], tot["n_bank"]
    if conserve_comb_energy:
        internal += comb_disc
    if not use_scalar_intensity_Tr:
        state.refresh_host()
    else:
        state.take_host_copies()
    total = internal + rad
    energy_loss = total - state.previous_total_energy - boundary_emission + boundary_loss - source_emission
    closure = energy_loss + (0.0 if conserve_comb_energy else comb_disc)
    state.time = state.time + dt
    state.previous_total_energy = total
    state.count += 1
    t_end = _time.perf_counter()

    n_tr = int(n_tr)
    ev = int(stats[_lib.STAT_EVENTS])
    info = {
        "time": state.time,
        "radiation_temperature": state.radiation_temperature,
        "temperature": state.temperature,
        "N_particles": int(n_particles),
        "total_energy": total,
        "total_internal_energy": internal,
        "total_radiation_energy": rad,
        "boundary_emission": boundary_emission,
        "boundary_loss": boundary_loss,
        "source_emission": source_emission,
        "energy_loss": energy_loss,
        "ledger": {
            "comb_discrepancy": comb_disc,
            "closure": closure,
            "relative_closure": closure / max(abs(total), 1e-300),
            "emission": emission_total,
            "weight_floor": 1e-10 * weight_sum / max(n_tr, 1),
        },
        "profiling": {
            "phase_times_s": {
                "sampling": (t_eval - t_step_start) + ms_src * 1e-3,
                "transport": ms_tr * 1e-3,
                "postprocess": max(t_end - t_step_start - (t_eval - t_step_start) - (ms_src + ms_tr) * 1e-3, 0.0),
                "total": t_end - t_step_start,
            },
            "transport_events": {
                "total": ev,
                "boundary_crossings": int(stats[_lib.STAT_BOUNDARY]),
                "census_events": int(stats[_lib.STAT_CENSUS]),
                "weight_floor_kills": int(stats[_lib.STAT_FLOOR]),
                "reflections": int(stats[_lib.STAT_REFLECT]),
                "escapes": int(stats[_lib.STAT_ESCAPE]),
                "avg_events_per_particle": ev / max(n_tr, 1),
                "n_particles_transported": n_tr,
            },
        },
    }
    te = info["profiling"]["transport_events"]
    if method == "cf":
        # IMC/IMC1D_CarterForest.py:1359-1372 and IMC/IMC2D_CarterForest.py:1141-1152 keys
        te["absorption_continue_events"] = int(stats[_lib.STAT_SCATTER])
        te["absorption_capture_events"] = int(stats[_lib.STAT_CAPTURE])
        te["event_cap_hits"] = int(stats[_lib.STAT_CAP])
    elif dim == 1:
        te["scatter_events"] = int(stats[_lib.STAT_SCATTER])
    else:
        te["absorption_continue_events"] = int(stats[_lib.STAT_SCATTER])
        te["absorption_capture_events"] = int(stats[_lib.STAT_CAPTURE])
        te["event_cap_hits"] = int(stats[_lib.STAT_CAP])
    return state, info


def _law(state, sigma_a_func, cv, inv_eos):
    """The device material law of these callables (cached on the state), or None."""
    key = (sigma_a_func, cv, inv_eos)
    cache = state.__dict__.get("_law_cache")
    if cache is None or not _same(cache[0], key):
        from .materials import material_law

        cache = (key, material_law(sigma_a_func, cv, inv_eos, state.flat, state._engine.device))
        object.__setattr__(state, "_law_cache", cache)
    return cache[1]


def tune(state: GrayState, grid: dict | None = None, repeats: int = 2) -> dict:
    """Autotune the tracking launch shape on the state's census: the last step's transport
    (sources, counts, step index) at the state's current temperature.  With a device-evaluated
    material law the opacity and heat capacity are the law's at that temperature, i.e. the
    next step's own inputs.  With other callables they are the last step's, evaluated at its
    start temperature, which the material update has since replaced: where the opacity
    depends on T, the replay's Fleck factor then differs from any real step's (a cell that
    heated keeps its cold opacity next to its new T^3), and so does its number of events.
    Call after at least one step.  Installs the best shape on the engine."""
    from .autotune import tune_tracking

    eng = state._engine
    if eng._last_transport is None:
        raise RuntimeError("tune() needs one completed step to replay")
    args, kwargs = eng._last_transport
    nxt = state.__dict__.get("_law_next")
    if nxt is not None:  # (T, sigma, cv) consistent: the next step's material inputs
        args = (state._T, nxt[1].reshape(-1), nxt[2]) + tuple(args[3:])
    return tune_tracking(eng, args, kwargs, grid=grid, repeats=repeats)


def init_state(engine: Engine, dim: int, shape: tuple, Ntarget, Tinit, Tr_init, eos, inv_eos, Ntarget_ic,
               T_emit_floor=0.0, dist=None) -> GrayState:
    """State at t = 0 with the equilibrium initial census.  dist: a torch.distributed module
    for a particle-partitioned run (each rank holds its share of the initial census, with
    1/world of its energy; radiation temperature and energy from the summed census)."""
    from .partition import local_count, sum_scalars, sum_tensors, world_of

    rank, world = world_of(dist)
    if world > 1:
        engine.partition(rank, world)
    dist = dist if world > 1 else None
    dev = engine.device
    Tg = torch.as_tensor(np.asarray(Tinit, dtype=np.float64), device=dev)
    Trg = torch.as_tensor(np.asarray(Tr_init, dtype=np.float64), device=dev)
    state = GrayState(engine, dim, shape, torch.zeros(engine.nc, dtype=torch.float64, device=dev),
                      torch.zeros(engine.nc, dtype=torch.float64, device=dev),
                      torch.zeros(engine.nc, dtype=torch.float64, device=dev), 0.0, 0.0, 0)
    e = evaluate(eos, Tg, lambda: np.asarray(Tinit, dtype=np.float64), Tg)
    state._e.copy_(state.flat(e))
    state._T.copy_(state.flat(Tg))
    back = evaluate(inv_eos, state.grid(state._e), lambda: state.grid(state._e).cpu().numpy(), Tg)
    assert torch.allclose(back, Tg), "Inverse EOS failed"
    N_ic = Ntarget if Ntarget_ic is None else Ntarget_ic
    engine.init_census(state.flat(Trg), local_count(N_ic, rank, world), T_emit_floor)
    rad_cell = torch.zeros(engine.nc, dtype=torch.float64, device=dev)
    if engine.bank.size:
        rad_cell.index_add_(0, engine.bank.view("cell").long(), engine.bank.view("weight").double())
    sum_tensors(dist, [rad_cell])
    state._Tr.copy_(torch.pow(rad_cell / engine.vol / A_RAD, 0.25))
    rad, internal = engine.energy_totals(state._e)
    rad = sum_scalars(dist, [rad], dev)[0]
    state.previous_total_energy = internal + rad
    state.refresh_host()
    return state
