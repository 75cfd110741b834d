"""Device-resident time loop: the reference drivers' step loops (IMC/CrookedPipe2D.py:887-1007:
adaptive dt, output-time hitting, fiducial history; the run_simulation loops of IMC/IMC1D.py,
IMC/IMC2D.py and the Carter-Forest modules) run as one captured CUDA graph replayed for every
step, with no host synchronisation between steps.

The drivers' dt schedule depends only on (dt_initial, growth factor, dt_max, output times), not
on the solution, so it is computed on the host first (adaptive_schedule) and written to device
memory.  A two-step graph is captured once (its two steps alternate the double-buffered bank):
a prologue reads this step's dt and Philox step counter from the schedule into device
scalars that every kernel reads at run time (imc_step_params.step_dev / dt_dev,
imc_comb_async_dev), then the step itself (device material callables, sources, tracking,
material update, comb), then an epilogue copies the step summary, the fiducial temperatures
and (at output steps) the temperature fields into device history buffers.  The graph is
replayed n/2 times (a one-step graph finishes an odd count); one synchronisation at the end
brings the histories back, and the FP64 energy ledger of every step is rebuilt from the
stored summaries exactly as the eager step builds it.

Multigroup states (mg_imc2d; MG_IMC/problems/crooked_pipe_multigroup_imc.py's loop) take a
list of per-group opacity callables, comb per (group, cell) and may grow Nmax every step
(Nmax_growth up to Nmax_final, read by the comb from a device schedule); the loop also keeps
the radiation energy by group (path-length estimate, MG_IMC2D's radiation_energy_by_group)
at the fiducial cells every step and over the mesh at output steps.

Requirements: gray (imc1d, imc2d, imc1d_cf, imc2d_cf) or 2-D multigroup states, device
material callables, fixed particle counts (no Ntotal split: it needs host estimates),
time-independent boundary temperatures (the graph holds fixed face tables), and a census
bound: the comb's output is capped at census_margin * max Nmax (+ slack); a step that would
exceed it is flagged (its census is emptied, so nothing is written out of bounds) and run()
raises.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._gray import _law, _same, face_temperatures
from .engine import C_LIGHT
from .materials import GroupedOpacity, evaluate, evaluate_groups, is_device


def adaptive_schedule(t0: float, output_times, dt_initial: float, dt_max: float, growth: float, saved=()):
    """The time steps of IMC/CrookedPipe2D.py:887-1007 from time t0: dt grows by `growth` up to
    dt_max, except after a step cut short to land on an output time.  Returns
    ([(dt, output_time or None), ...], the dt the next step would start from)."""
    t_final = max(output_times) if len(output_times) else 10.0
    saved = set(float(x) for x in saved)
    time, current, steps = float(t0), float(dt_initial), []
    while time < t_final - 1e-12:
        step_dt = min(current, t_final - time)
        hit = False
        for tout in output_times:
            if tout not in saved and time < tout < time + step_dt:
                step_dt = tout - time
                hit = True
                break
        time = time + step_dt
        out = None
        for tout in output_times:
            if tout not in saved and abs(time - tout) < 1e-9:
                saved.add(tout)
                out = tout
                break
        steps.append((step_dt, out))
        if not hit:
            current = min(current * growth, dt_max)
    return steps, current


def _no_host():
    raise RuntimeError("the device loop needs device material callables (radtranbook_b200.materials)")


class DeviceLoop:
    """Run many drop-in steps of one state as a replayed CUDA graph (see the module
    docstring).  The keyword arguments are those of the drop-in step (IMC2D.step and
    MG_IMC2D.step names; sigma_a_func is the list of per-group callables for a multigroup
    state); fiducial_cells: reference-layout cell indices ((i, j) in 2-D, i in 1-D) whose T and
    Tr are recorded after every step."""

    def __init__(self, state, *, Ntarget, Nboundary, Nsource, Nmax, T_boundary, sigma_a_func, inv_eos, cv,
                 source=None, reflect=(False, False, False, False), theta=1.0, conserve_comb_energy=False,
                 rz_linear_source=True, max_events=0, boundary_source_func=None, geometry="xy", method="fc",
                 cf_fastpath=0.0, T_emit_floor=0.0, fiducial_cells=(), census_margin=1.25, Nmax_growth=0,
                 Nmax_final=None):
        self.state = state
        eng = state._engine
        self.eng = eng
        dev = eng.device
        self.mg = eng.ng > 1
        funcs = (sigma_a_func if isinstance(sigma_a_func, GroupedOpacity) else list(sigma_a_func)) if self.mg \
            else [sigma_a_func]
        if self.mg and (len(funcs) != eng.ng or state._dim != 2):
            raise ValueError("a multigroup device loop needs a 2-D state and one opacity callable per group")
        for f in (*funcs, inv_eos, cv):
            if not is_device(f):
                _no_host()
        if any(callable(t) for t in T_boundary):
            raise ValueError("the device loop needs time-independent boundary temperatures")
        if int(Nmax) <= 0:
            raise ValueError("the device loop combs to Nmax > 0 every step")
        self.sigma_funcs = funcs
        self.nmax = (int(Nmax), int(Nmax_growth), int(Nmax_final) if Nmax_final is not None else None)
        self.nmax_top = max(int(Nmax), int(Nmax_final)) if (Nmax_growth and Nmax_final is not None) else int(Nmax)
        if Nmax_growth and Nmax_final is None:
            raise ValueError("Nmax_growth needs Nmax_final (the census bound)")
        if self.mg:
            rz_linear_source = False  # MG_IMC2D samples emission uniformly in the cell
        self.kw = dict(Ntarget=int(Ntarget), Nboundary=int(Nboundary), Nsource=int(Nsource), Nmax=int(Nmax),
                       theta=float(theta), max_events=int(max_events), rz_linear_source=bool(rz_linear_source),
                       method=_lib.METHOD_CARTER_FOREST if method == "cf" else _lib.METHOD_FLECK_CUMMINGS,
                       cf_fastpath=float(cf_fastpath), T_emit_floor=float(T_emit_floor))
        self.sigma_a_func, self.inv_eos, self.cv = sigma_a_func, inv_eos, cv
        self.conserve = bool(conserve_comb_energy)
        # a device-evaluated material law (LinearEOS, Constant cv, PowerLawOpacity / Constant /
        # GroupPowerLawOpacity): the material update kernel writes T and the next step's opacity
        # and cv into one buffer pair, which the next step's plan reads (nothing later in a step
        # reads them, so one pair serves every step of the graph)
        self.law = _law(state, sigma_a_func, cv, inv_eos) if not self.conserve else None
        self.law_key = (sigma_a_func, cv)
        if self.law is not None:
            self.law_sigma = torch.empty(eng.ng * eng.nc, dtype=torch.float64, device=dev)
            self.law_cv = torch.empty(eng.nc, dtype=torch.float64, device=dev)
        self.refl = tuple(reflect) + (False,) * (4 - len(reflect))
        self.src = None
        if Nsource > 0 and source is not None:
            s = torch.as_tensor(np.asarray(source, dtype=np.float64), device=dev)
            if float(s.max()) > 0:
                self.src = state.flat(s).contiguous()
        e1, e2 = eng.e1.cpu().numpy(), eng.e2.cpu().numpy()
        self.faces = face_temperatures(state._dim, geometry, T_boundary, state.time, e1, e2, boundary_source_func,
                                       dev, {})
        if state._dim == 2:
            nx = state._shape[0]
            fid = [int(i) + nx * int(j) for i, j in fiducial_cells]
        else:
            fid = [int(i) for i in fiducial_cells]
        self.fid = torch.as_tensor(np.asarray(fid, dtype=np.int64), device=dev)
        self.cap_census = int(census_margin * self.nmax_top) + 2 * eng.nc * eng.ng + 4096
        self.step_dev = torch.zeros(1, dtype=torch.int32, device=dev)
        self.dt_dev = torch.zeros(1, dtype=torch.float64, device=dev)
        self.nmax_dev = torch.zeros(1, dtype=torch.int64, device=dev)
        self.k_done = 0  # steps run so far (the Nmax schedule continues across run() calls)
        if self.mg:
            self.rad_last = torch.zeros(eng.ng * eng.nc, dtype=torch.float64, device=dev)
        self.k_dev = torch.zeros(1, dtype=torch.int64, device=dev)
        self._cap = (0, -1)   # (steps, outputs) the history buffers hold
        self._graphs = {}     # (id of the bank holding the census, steps per graph) -> graph

    # ------------------------------------------------------------------ one captured step
    def _enqueue_step(self) -> None:
        st, eng, kw = self.state, self.eng, self.kw
        # prologue: this step's dt and Philox step counter
        torch.index_select(self.dt_sched, 0, self.k_dev, out=self.dt_dev)
        torch.index_select(self.step_sched, 0, self.k_dev, out=self.step_dev)
        torch.index_select(self.nmax_sched, 0, self.k_dev, out=self.nmax_dev)
        like = st.grid(st._T)
        if self.law is not None:
            sigma, cvv = self.law_sigma, self.law_cv
        else:
            sigma, cvv = self._materials(like)
        # the host-side step and dt are placeholders: the kernels read step_dev / dt_dev
        eng.transport_async(st._T, sigma, cvv, self.src, 0, 1.0, kw["theta"], kw["Ntarget"], kw["Nboundary"],
                            kw["Nsource"], self.faces, self.refl, max_events=kw["max_events"],
                            rz_linear_source=kw["rz_linear_source"], t_emit_floor=kw["T_emit_floor"],
                            method=kw["method"], cf_fastpath=kw["cf_fastpath"], step_dev=self.step_dev,
                            dt_dev=self.dt_dev)
        if self.law is not None:
            eng.material_update_law(st._e, st._Tr, st._T, self.law[0], self.law_sigma, self.law_cv)
        else:
            eng.material_update(st._e, st._Tr)
        if self.mg:
            self.rad_last.copy_(eng.si)
            if self.fid.numel():
                at_fid = eng.si.view(eng.ng, eng.nc).index_select(1, self.fid)
                self.hist_Eg.index_copy_(0, self.k_dev, at_fid.view(1, -1))
        eng.comb_async(self.nmax_top, 0, st._e, per_group=self.mg, step_dev=self.step_dev,
                       out_capacity=self.cap_census, n_max_dev=self.nmax_dev)
        if self.conserve:
            st._e.add_((eng.disc.view(eng.ng, eng.nc).sum(0) if self.mg else eng.disc[: eng.nc]) / eng.vol)
        if self.law is None:
            Tn = evaluate(self.inv_eos, st.grid(st._e), _no_host, like)
            st._T.copy_(st.flat(Tn))
        # epilogue: summary, fiducial temperatures, output snapshots
        self.hist_sum.index_copy_(0, self.k_dev, eng.summary_dev.view(1, -1))
        if self.fid.numel():
            self.hist_T.index_copy_(0, self.k_dev, st._T.index_select(0, self.fid).view(1, -1))
            self.hist_Tr.index_copy_(0, self.k_dev, st._Tr.index_select(0, self.fid).view(1, -1))
        slot = torch.index_select(self.out_slot, 0, self.k_dev)
        self.snap_T.index_copy_(0, slot, st._T.view(1, -1))
        self.snap_Tr.index_copy_(0, slot, st._Tr.view(1, -1))
        if self.mg:
            self.snap_Eg.index_copy_(0, slot, self.rad_last.view(1, -1))
        self.k_dev.add_(1)
        # the comb wrote the next census into the spare bank: swap (sizes stay upper bounds)
        eng.spare.size = self.cap_census
        eng.bank, eng.spare = eng.spare, eng.bank
        eng._census_dev_valid = True

    def _materials(self, like) -> tuple:
        """Opacity ([g][c] flat) and heat capacity of the material callables at the state's T."""
        st = self.state
        sigma = evaluate_groups(self.sigma_funcs, like, _no_host, like).transpose(1, 2).reshape(-1) \
            if self.mg else st.flat(evaluate(self.sigma_funcs[0], like, _no_host, like))
        return sigma, st.flat(evaluate(self.cv, like, _no_host, like))

    def _graph(self, n: int) -> torch.cuda.CUDAGraph:
        """The n-step graph starting from the bank that holds the census now (captured once;
        a graph reads fixed bank pointers, so each starting bank has its own)."""
        key = (id(self.eng.bank), n)
        if key not in self._graphs:
            g = torch.cuda.CUDAGraph()
            order = (self.eng.bank, self.eng.spare)
            with torch.cuda.graph(g):
                for _ in range(n):
                    self._enqueue_step()
            self.eng.bank, self.eng.spare = order  # capturing ran nothing: restore the host view
            self._graphs[key] = g
        return self._graphs[key]

    def _buffers(self, n: int, n_out: int) -> None:
        """History buffers for n steps and n_out snapshots (reallocated, and the graphs that
        point at them dropped, only when they grow)."""
        if n <= self._cap[0] and n_out <= self._cap[1]:
            return
        n, n_out = max(n, self._cap[0]), max(n_out, self._cap[1], 0)
        dev = self.eng.device
        self.dt_sched = torch.zeros(n, dtype=torch.float64, device=dev)
        self.step_sched = torch.zeros(n, dtype=torch.int32, device=dev)
        self.nmax_sched = torch.zeros(n, dtype=torch.int64, device=dev)
        self.out_slot = torch.full((n,), n_out, dtype=torch.int64, device=dev)
        self.hist_sum = torch.zeros((n, ctypes.sizeof(_lib.ImcStepSummary)), dtype=torch.uint8, device=dev)
        nf = max(int(self.fid.numel()), 1)
        self.hist_T = torch.zeros((n, nf), dtype=torch.float64, device=dev)
        self.hist_Tr = torch.zeros((n, nf), dtype=torch.float64, device=dev)
        self.snap_T = torch.zeros((n_out + 1, self.eng.nc), dtype=torch.float64, device=dev)
        self.snap_Tr = torch.zeros_like(self.snap_T)
        if self.mg:
            ncg = self.eng.ng * self.eng.nc
            self.hist_Eg = torch.zeros((n, self.eng.ng * nf), dtype=torch.float64, device=dev)
            self.snap_Eg = torch.zeros((n_out + 1, ncg), dtype=torch.float64, device=dev)
        self._cap = (n, n_out)
        self._graphs = {}

    # ------------------------------------------------------------------ run
    def run(self, dts, output_steps=None) -> dict:
        """Advance by len(dts) steps of the given lengths.  output_steps: {step index: label}
        whose T / Tr fields are kept.  Returns per-step times, fiducial histories, snapshots and
        per-step ledger figures (as the drop-in step's info)."""
        st, eng = self.state, self.eng
        dev = eng.device
        n = len(dts)
        if n == 0:
            return {"times": [], "steps": []}
        if eng.bank.size > self.cap_census:
            raise ValueError("census larger than the device loop's bound: raise census_margin")
        outs = dict(output_steps or {})
        labels = list(outs.values())
        self._buffers(n, len(labels))
        self.dt_sched[:n].copy_(torch.as_tensor(np.asarray(dts, dtype=np.float64)))
        self.step_sched[:n].copy_(torch.arange(st.count, st.count + n, dtype=torch.int32))
        self.nmax_sched[:n].copy_(torch.as_tensor(self._nmax_schedule(n), dtype=torch.int64))
        slots = np.full(n, self._cap[1], dtype=np.int64)  # the last row collects non-output steps
        for q, k in enumerate(outs):
            slots[int(k)] = q
        self.out_slot[:n].copy_(torch.as_tensor(slots))
        # size everything for the census bound before capture (no allocation in the graph)
        bound = int(eng.lib.imc_source_bound(ctypes.byref(eng.cmesh), ctypes.byref(eng._params(
            0, 1.0, 1.0, self.kw["Ntarget"], self.kw["Nboundary"], self.kw["Nsource"], self.faces, self.refl, 0,
            self.kw["rz_linear_source"], 0.0))))
        for b in (eng.bank, eng.spare):
            b.ensure(self.cap_census + bound)
        eng._ws(max(eng.bank.capacity, eng.spare.capacity))
        # evaluate the material callables once outside the capture (they may build device
        # tables on first use, which a capture cannot do)
        like = st.grid(st._T)
        if self.mg:
            evaluate_groups(self.sigma_funcs, like, _no_host, like)
        for f in self.sigma_funcs:
            evaluate(f, like, _no_host, like)
        evaluate(self.cv, like, _no_host, like)
        evaluate(self.inv_eos, st.grid(st._e), _no_host, like)
        if self.law is not None:  # the first step's opacity: the eager step's law output, else the callables
            nxt = st.__dict__.get("_law_next")
            if nxt is not None and _same(nxt[0], self.law_key):
                self.law_sigma.copy_(nxt[1].reshape(-1))
                self.law_cv.copy_(nxt[2])
            else:
                sigma, cvv = self._materials(like)
                self.law_sigma.copy_(sigma)
                self.law_cv.copy_(cvv)
        eng._set_census_count(eng.bank.size)
        eng.bank.size = eng.spare.size = self.cap_census
        g2 = self._graph(2) if n >= 2 else None
        g1 = self._graph(1) if n % 2 else None
        self.k_dev.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n // 2):
            g2.replay()
        if g1 is not None:
            g1.replay()
            eng.bank, eng.spare = eng.spare, eng.bank
        e1.record()
        torch.cuda.current_stream().synchronize()
        st.__dict__.pop("_host_next", None)  # the loop's steps changed T
        if self.law is not None:  # an eager step after the loop continues from the loop's law output
            st.__dict__["_law_next"] = (self.law_key, self.law_sigma, self.law_cv)
        else:
            st.__dict__.pop("_law_next", None)
        out = self._finish(dts, outs, labels)
        out["device_ms"] = e0.elapsed_time(e1)
        return out

    def _nmax_schedule(self, n: int) -> list:
        """Comb targets of the next n steps (MG_IMC2D 'Nmax_next': + Nmax_growth per step, capped
        at Nmax_final)."""
        n0, growth, final = self.nmax
        out = [n0 + (self.k_done + k) * growth if growth else n0 for k in range(n)]
        return [min(x, final) for x in out] if (growth and final is not None) else out

    def _finish(self, dts, outs, labels) -> dict:
        st, eng = self.state, self.eng
        raw = self.hist_sum.cpu().numpy()
        steps, times = [], []
        prev = st.previous_total_energy
        worst = 0.0
        for k, dt in enumerate(dts):
            sm = _lib.ImcStepSummary.from_buffer_copy(raw[k].tobytes())
            if sm.flags & _lib.FLAG_BOUNDS:
                raise _lib.ImcError("device loop: bounds check", 9)
            if sm.flags & _lib.FLAG_COMB_OVERFLOW:
                raise _lib.ImcError("device loop: census above census_margin * Nmax", _lib.BANK_OVERFLOW)
            if sm.flags & _lib.FLAG_NONFINITE:
                raise _lib.ImcError("device loop", 3)
            if sm.flags & _lib.FLAG_EVENT_CAP:
                raise _lib.ImcError("device loop", 2)
            internal, rad = float(sm.internal_energy), float(sm.comb_after)
            comb_disc = float(sm.comb_before) - rad
            if self.conserve:
                internal += comb_disc
            total = internal + rad
            be, bl, se = float(sum(sm.e_side)), float(sum(sm.escaped)), float(sm.source_emission)
            loss = total - prev - be + bl - se
            closure = loss + (0.0 if self.conserve else comb_disc)
            worst = max(worst, abs(closure) / max(abs(total), 1e-300))
            st.time = st.time + dt
            times.append(st.time)
            steps.append({"time": st.time, "dt": dt, "N_particles": int(sm.n_out), "total_energy": total,
                          "total_internal_energy": internal, "total_radiation_energy": rad,
                          "boundary_emission": be, "boundary_loss": bl, "source_emission": se, "energy_loss": loss,
                          "ledger": {"comb_discrepancy": comb_disc, "closure": closure,
                                     "relative_closure": closure / max(abs(total), 1e-300)},
                          "transport_events": {"total": int(sm.stats[_lib.STAT_EVENTS]),
                                               "n_particles_transported": int(sm.n_bank)}})
            prev = total
        st.count += len(dts)
        self.k_done += len(dts)
        st.previous_total_energy = prev
        eng.bank.size = int(steps[-1]["N_particles"])
        eng.spare.size = 0
        eng._census_dev_valid = True
        st.refresh_host()
        n = len(dts)
        fid_T = self.hist_T[:n].cpu().numpy()[:, : int(self.fid.numel())]
        fid_Tr = self.hist_Tr[:n].cpu().numpy()[:, : int(self.fid.numel())]
        snaps = {}
        sT, sTr = self.snap_T.cpu(), self.snap_Tr.cpu()
        for q, label in enumerate(labels):
            snaps[label] = (st.grid(sT[q]).numpy().copy(), st.grid(sTr[q]).numpy().copy())
        out = {"times": times, "steps": steps, "fiducial_T": fid_T, "fiducial_Tr": fid_Tr, "snapshots": snaps,
               "max_relative_closure": worst}
        if self.mg:
            G, nf = eng.ng, int(self.fid.numel())
            nx, ny = st._shape

            def grid3(x):  # (G * nc) -> (G, nx, ny), energy density (si / c)
                return (x.view(G, ny, nx).transpose(1, 2) / C_LIGHT).cpu().numpy().copy()

            out["fiducial_Erad_by_group"] = self.hist_Eg[:n].cpu().numpy().reshape(n, G, -1)[:, :, :nf] / C_LIGHT
            sE = self.snap_Eg
            out["snapshots_Erad_by_group"] = {label: grid3(sE[q]) for q, label in enumerate(labels)}
            st.__dict__["radiation_energy_by_group"] = grid3(self.rad_last)
            st.__dict__["radiation_energy_by_group_postcomb"] = None
            out["Nmax_next"] = self._nmax_schedule(1)[0]
        return out


def crooked_pipe_run(state, problem: dict, output_times, dt_initial=0.001, dt_max=10.0, growth=1.1,
                     fiducial_points=None, method="fc", census_margin=1.25):
    """The time loop of IMC/CrookedPipe2D.py:887-1007 on the device: adaptive dt that lands on
    the output times, fiducial histories and output snapshots.  problem: a
    radtranbook_b200.problems.crooked_pipe dict (device callables); state: its imc2d /
    imc2d_cf state.  Returns (times, fiducial_data, fiducial_data_rad, snapshots, result)."""
    e1, e2 = problem["edges1"], problem["edges2"]
    rc, zc = 0.5 * (e1[:-1] + e1[1:]), 0.5 * (e2[:-1] + e2[1:])
    pts = fiducial_points if fiducial_points is not None else problem["fiducials"]
    cells = {lbl: (int(np.argmin(np.abs(rc - r))), int(np.argmin(np.abs(zc - z)))) for lbl, (r, z) in pts.items()}
    sched, _ = adaptive_schedule(state.time, list(output_times), dt_initial, dt_max, growth)
    loop = DeviceLoop(state, Ntarget=problem["Ntarget"], Nboundary=problem["Nboundary"], Nsource=0,
                      Nmax=problem["Nmax"], T_boundary=problem["T_boundary"], sigma_a_func=problem["sigma_dev"],
                      inv_eos=problem["inv_eos_dev"], cv=problem["cv_dev"], source=problem["source"],
                      reflect=problem["reflect"], geometry="rz", max_events=1_000_000,
                      boundary_source_func=problem["boundary_source_func"], method=method,
                      fiducial_cells=list(cells.values()), census_margin=census_margin)
    outputs = {k: tout for k, (_, tout) in enumerate(sched) if tout is not None}
    T0, Tr0 = state.temperature.copy(), state.radiation_temperature.copy()
    t_start = state.time
    res = loop.run([dt for dt, _ in sched], outputs)
    times = [t_start] + res["times"]
    fid, fid_rad = {}, {}
    for q, (lbl, (i, j)) in enumerate(cells.items()):
        fid[lbl] = [float(T0[i, j])] + list(res["fiducial_T"][:, q])
        fid_rad[lbl] = [float(Tr0[i, j])] + list(res["fiducial_Tr"][:, q])
    return times, fid, fid_rad, res["snapshots"], res


def mg_crooked_pipe_run(state, problem: dict, output_times, fiducial_points=None, census_margin=1.25):
    """The time loop of MG_IMC/problems/crooked_pipe_multigroup_imc.py on the device: dt from
    the problem's dt_initial growing by dt_growth to dt_max and landing on the output times,
    Nmax growing by Nmax_growth per step to Nmax_final, fiducial T / Tr / radiation spectra every
    step, and T, Tr and the radiation energy by group at the output times.  problem: a
    radtranbook_b200.problems.mg_crooked_pipe dict; state: its mg_imc2d state.  Returns
    (times, fiducial_data, fiducial_data_rad, snapshots, result); snapshots[t] = (T, Tr, Erad_g)."""
    e1, e2 = problem["edges1"], problem["edges2"]
    rc, zc = 0.5 * (e1[:-1] + e1[1:]), 0.5 * (e2[:-1] + e2[1:])
    pts = fiducial_points if fiducial_points is not None else problem["fiducials"]
    cells = {lbl: (int(np.argmin(np.abs(rc - r))), int(np.argmin(np.abs(zc - z)))) for lbl, (r, z) in pts.items()}
    sched, _ = adaptive_schedule(state.time, list(output_times), problem["dt_initial"], problem["dt_max"],
                                 problem["dt_growth"])
    loop = DeviceLoop(state, Ntarget=problem["Ntarget"], Nboundary=problem["Nboundary"], Nsource=0,
                      Nmax=problem["Nmax"], T_boundary=problem["T_boundary"], sigma_a_func=problem["sigma_dev"],
                      inv_eos=problem["inv_eos_dev"], cv=problem["cv_dev"], reflect=problem["reflect"],
                      geometry="rz", max_events=1_000_000, boundary_source_func=problem["boundary_source_func"],
                      T_emit_floor=problem["T_emit_floor"], fiducial_cells=list(cells.values()),
                      census_margin=census_margin, Nmax_growth=problem["Nmax_growth"],
                      Nmax_final=problem["Nmax_final"])
    outputs = {k: tout for k, (_, tout) in enumerate(sched) if tout is not None}
    T0, Tr0 = state.temperature.copy(), state.radiation_temperature.copy()
    t_start = state.time
    res = loop.run([dt for dt, _ in sched], outputs)
    times = [t_start] + res["times"]
    fid, fid_rad = {}, {}
    for q, (lbl, (i, j)) in enumerate(cells.items()):
        fid[lbl] = [float(T0[i, j])] + list(res["fiducial_T"][:, q])
        fid_rad[lbl] = [float(Tr0[i, j])] + list(res["fiducial_Tr"][:, q])
    snaps = {t: (T, Tr, res["snapshots_Erad_by_group"][t]) for t, (T, Tr) in res["snapshots"].items()}
    return times, fid, fid_rad, snaps, res
