"""Device engine: owns the particle banks, tallies and workspace of one IMC problem on one
GPU and drives the C ABI of libimcb200.so on the current torch stream.

All memory is allocated here, through torch (the library itself never allocates).  Banks
are double-buffered: tracking runs in place on the active bank; the comb writes the other
bank, and the two swap.  A call that reports IMC_ERR_BANK_OVERFLOW is retried after the
bank grows; the library guarantees nothing was modified in that case.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import (ImcBank, ImcCombReport, ImcMaterial, ImcMesh, ImcStepParams, ImcStepReport, ImcStepSummary,
                   ImcTallies)

A_RAD = 0.01372
C_LIGHT = 29.98


# the current stream's raw handle without building a torch Stream object (which costs a few
# microseconds of the host time a step leaves the device idle); the public call otherwise
_RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _comb_flags(per_group: bool, conserve_radiation: bool) -> int:
    return (_lib.COMB_PER_GROUP if per_group else 0) | (_lib.COMB_CONSERVE_RADIATION if conserve_radiation else 0)


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("radtranbook_b200 needs a CUDA device (B200, sm_100a); none is available")
    return torch.device("cuda", torch.cuda.current_device())


class Bank:
    """Structure-of-arrays particle bank in device memory."""

    FIELDS_F = ("pos1", "pos2", "dir1", "dir2", "weight", "time")
    FIELDS_I = ("cell", "group")

    def __init__(self, capacity: int, device: torch.device, multigroup: bool = False):
        self.device = device
        self.multigroup = multigroup
        self.size = 0
        self.capacity = 0
        self._alloc(max(int(capacity), 1024))

    def _alloc(self, cap: int) -> None:
        old = {k: getattr(self, k, None) for k in self.FIELDS_F + self.FIELDS_I}
        for k in self.FIELDS_F:
            setattr(self, k, torch.empty(cap, dtype=torch.float32, device=self.device))
        self.cell = torch.empty(cap, dtype=torch.int32, device=self.device)
        self.group = torch.empty(cap, dtype=torch.int32, device=self.device) if self.multigroup else None
        if self.size:
            for k in self.FIELDS_F + ("cell",) + (("group",) if self.multigroup else ()):
                getattr(self, k)[: self.size].copy_(old[k][: self.size])
        self.capacity = cap

    def ensure(self, cap: int) -> None:
        if cap > self.capacity:
            self._alloc(int(cap * 1.25) + 1024)

    def c(self) -> ImcBank:
        return ImcBank(_ptr(self.pos1), _ptr(self.pos2), _ptr(self.dir1), _ptr(self.dir2), _ptr(self.weight),
                       _ptr(self.time), _ptr(self.cell), _ptr(self.group), self.size, self.capacity)

    def view(self, name: str) -> torch.Tensor:
        return getattr(self, name)[: self.size]

    def load(self, weight, dir1, dir2, time, pos1, pos2, cell, group=None) -> None:
        n = len(weight)
        self.size = 0
        self.ensure(n)
        for k, v in (("weight", weight), ("dir1", dir1), ("dir2", dir2), ("time", time),
                     ("pos1", pos1), ("pos2", pos2)):
            getattr(self, k)[:n].copy_(torch.as_tensor(np.asarray(v, dtype=np.float32)))
        self.cell[:n].copy_(torch.as_tensor(np.asarray(cell, dtype=np.int32)))
        if self.multigroup:
            self.group[:n].copy_(torch.as_tensor(np.asarray(group if group is not None else np.zeros(n), dtype=np.int32)))
        self.size = n


@dataclass
class StepResult:
    report: ImcStepReport
    comb: ImcCombReport | None = None
    stats: np.ndarray = field(default_factory=lambda: np.zeros(_lib.STAT_N, dtype=np.int64))
    escaped: np.ndarray = field(default_factory=lambda: np.zeros(4))


class Engine:
    """One IMC mesh on one device.  Cell arrays are flat, c = i + nx*j (float64)."""

    def __init__(self, geometry: str, edges1, edges2, volumes, seed: int = 0x5EED0001, n_groups: int = 1,
                 capacity: int = 1 << 16, device: torch.device | None = None, group_edges=None):
        self.lib = _lib.load()
        self.device = device or require_cuda()
        if geometry not in _lib.GEOM:
            raise ValueError(f"Unknown geometry: {geometry}")
        self.geometry = geometry
        self.gcode = _lib.GEOM[geometry]
        e1 = np.asarray(edges1, dtype=np.float64)
        e2 = np.asarray(edges2, dtype=np.float64)
        self.nx, self.ny = len(e1) - 1, len(e2) - 1
        self.nc = self.nx * self.ny
        self.ng = n_groups
        self.rank, self.world = 0, 1
        self.seed = seed
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.e1 = torch.as_tensor(e1, **f64)
        self.e2 = torch.as_tensor(e2, **f64)
        self.vol = torch.as_tensor(np.asarray(volumes, dtype=np.float64).reshape(-1), **f64)
        if self.vol.numel() != self.nc:
            raise ValueError("volumes must have nx*ny entries")
        self.gedges = None
        if n_groups > 1:
            if group_edges is None or len(group_edges) != n_groups + 1:
                raise ValueError("multigroup needs n_groups + 1 group edges")
            self.gedges = torch.as_tensor(np.asarray(group_edges, dtype=np.float64), **f64)
        self.cmesh = ImcMesh(self.gcode, self.nx, self.ny, n_groups, _ptr(self.e1), _ptr(self.e2), _ptr(self.vol),
                             _ptr(self.gedges))
        self.escaped_group = torch.zeros(n_groups, **f64) if n_groups > 1 else None
        self.boundary_group = torch.zeros(n_groups, **f64) if n_groups > 1 else None
        self.emission_fractions = None  # optional device tensor [g]
        ncg = self.nc * n_groups
        self.dep = torch.zeros(ncg, **f64)
        self.si = torch.zeros(ncg, **f64)
        self.emitted = torch.zeros(self.nc, **f64)
        self.sigma_a = torch.zeros(ncg, **f64)
        self.sigma_s = torch.zeros(ncg, **f64)
        self.escaped = torch.zeros(4 + n_groups, **f64)
        self.stats = torch.zeros(_lib.STAT_N, dtype=torch.int64, device=dev)
        # comb discrepancy per bin, then (IMC_COMB_WRITE_AFTER) the energy after the comb per bin
        self._disc2 = torch.zeros(2 * ncg, **f64)
        self.disc, self.comb_after = self._disc2[:ncg], self._disc2[ncg:]
        self.ctal = ImcTallies(_ptr(self.dep), _ptr(self.si), _ptr(self.emitted), _ptr(self.sigma_a),
                               _ptr(self.sigma_s), _ptr(self.escaped), _ptr(self.stats),
                               _ptr(self.escaped_group), _ptr(self.boundary_group))
        # device step summary (sizes, energies, statistics) and its pinned host copy; the
        # asynchronous step writes its statistics and escaped energy straight into it
        nsum = ctypes.sizeof(ImcStepSummary)
        self.summary_dev = torch.zeros(nsum, dtype=torch.uint8, device=dev)
        self.summary_host = torch.zeros(nsum, dtype=torch.uint8, pin_memory=True)
        self.summary = ImcStepSummary.from_address(self.summary_host.data_ptr())
        base = self.summary_dev.data_ptr()
        self.ctal_async = ImcTallies(_ptr(self.dep), _ptr(self.si), _ptr(self.emitted), _ptr(self.sigma_a),
                                     _ptr(self.sigma_s), base + ImcStepSummary.escaped.offset,
                                     base + ImcStepSummary.stats.offset, _ptr(self.escaped_group),
                                     _ptr(self.boundary_group))
        self._census_dev_valid = False
        self._upper = 0
        mg = n_groups > 1
        self.bank = Bank(capacity, dev, mg)
        self.spare = Bank(capacity, dev, mg)
        self.ws = torch.empty(0, dtype=torch.uint8, device=dev)
        self._ws_need = (None, 0)  # (capacity, event form) -> workspace bytes, of the last query
        self.launch = dict(block_size=256, blocks_per_sm=4, chunk=512, smem_cells=0)
        self._last_transport = None
        # particle partition over ranks (radtranbook_b200.partition): this rank's Philox id
        # offset and share of the source energy; its comb and initial census use comb_seed
        self.id_base = 0
        self.energy_share = 1.0
        # the asynchronous step's tracking sums the census per comb bin (cells, or (group, cell)
        # on a multigroup mesh) and the comb that follows uses those sums
        self.fuse_census = True
        self._census_bins = 0

    @property
    def seed(self) -> int:
        return self._seed

    @seed.setter
    def seed(self, value: int) -> None:
        self._seed = int(value) & 0xFFFFFFFFFFFFFFFF

    @property
    def comb_seed(self) -> int:
        """Philox key of the comb and the initial census: the seed, or on rank r > 0 of a
        partition a per-rank key derived from it."""
        from .partition import rank_key

        return rank_key(self._seed, getattr(self, "rank", 0))

    ic_seed = comb_seed

    def partition(self, rank: int, world: int) -> None:
        """Make this engine rank `rank` of a `world`-rank particle partition: its sources and
        tracking draw Philox ids from rank * (2^32 // world), it issues 1/world of every source
        energy, and its comb and initial census use a per-rank key."""
        from .partition import id_base

        if not (0 <= rank < world):
            raise ValueError("rank must be in [0, world)")
        self.rank, self.world = int(rank), int(world)
        self.id_base = id_base(rank, world)
        self.energy_share = 1.0 / world

    # ------------------------------------------------------------------ helpers
    def _stream(self) -> int:
        if _RAW_STREAM is not None:
            idx = self.device.index
            return _RAW_STREAM(torch.cuda.current_device() if idx is None else idx)
        return torch.cuda.current_stream(self.device).cuda_stream

    def _ws(self, capacity: int) -> tuple[int, int]:
        key = (int(capacity), bool(self.launch.get("event_based")))
        if self._ws_need[0] == key:
            need = self._ws_need[1]
        else:
            size = self.lib.imc_workspace_bytes_event if key[1] else self.lib.imc_workspace_bytes
            need = int(size(ctypes.byref(self.cmesh), key[0]))
            self._ws_need = (key, need)
        if self.ws.numel() < need:
            self.ws = torch.empty(int(need * 1.25) + 4096, dtype=torch.uint8, device=self.device)
        return self.ws.data_ptr(), self.ws.numel()

    def reserve(self, census: int, sources: int = 0) -> None:
        """Size the bank and the spare bank for a census of up to `census` entries (a comb
        target) plus `sources` new entries a step, so that a growing comb target reallocates
        nothing (each bank otherwise grows by 1.25x when it runs out)."""
        cap = int(1.15 * census) + 2 * self.nc * self.ng + 4096 + int(sources)
        self.bank.ensure(cap)
        self.spare.ensure(cap)

    def _call_bank(self, name: str, fn, bank: Bank, grow_from, *args):
        """Call fn(cbank, ...); on bank overflow grow `bank` and retry once."""
        for _ in range(2):
            cb = bank.c()
            st = fn(cb, *args)
            if st == _lib.BANK_OVERFLOW:
                bank.ensure(int(grow_from()))
                continue
            _lib.check(name, st)
            return cb
        raise _lib.ImcError(name, _lib.BANK_OVERFLOW)

    # ------------------------------------------------------------------ phases
    def init_census(self, tr_flat: torch.Tensor, n_target: int, t_emit_floor: float = 0.0) -> int:
        tr_flat = tr_flat.to(self.device, torch.float64).contiguous()
        # upper bound: ceil adds at most one per cell (2-D also at least one per cell)
        self.bank.size = 0
        self.bank.ensure(int(n_target) + 2 * self.nc + 16)
        wsp, wsn = self._ws(self.bank.capacity)
        n_out = ctypes.c_int64(0)
        cb = self.bank.c()
        st = self.lib.imc_init_census(ctypes.byref(self.cmesh), _ptr(tr_flat), int(n_target), float(t_emit_floor),
                                      self.ic_seed, ctypes.byref(cb), wsp, wsn, ctypes.byref(n_out), self._stream())
        _lib.check("imc_init_census", st)
        self.bank.size = int(cb.size)
        if self.energy_share != 1.0 and self.bank.size:
            self.bank.weight[: self.bank.size].mul_(self.energy_share)  # this rank's share of the energy
        self._census_dev_valid = False
        return self.bank.size

    def transport(self, T: torch.Tensor, sigma: torch.Tensor, cv: torch.Tensor, source: torch.Tensor | None,
                  step: int, dt: float, theta: float, n_target: int, n_boundary: int, n_source: int,
                  face_T: list, reflect, max_events: int = 0, rz_linear_source: bool = True,
                  t_emit_floor: float = 0.0, method: int = 0, cf_fastpath: float = 0.0) -> StepResult:
        mat = ImcMaterial(_ptr(T), _ptr(sigma), _ptr(cv), _ptr(source))
        par = self._params(step, dt, theta, n_target, n_boundary, n_source, face_T, reflect, max_events,
                           rz_linear_source, t_emit_floor, method=method, cf_fastpath=cf_fastpath)
        rep = ImcStepReport()
        # sources add at most n_target + n_source + ncell (ceil) + 4 * n_boundary entries
        self.bank.ensure(self.bank.size + int(n_target) + int(n_source) + 2 * self.nc + 4 * int(n_boundary) + 16)

        def run(cb):
            wsp, wsn = self._ws(self.bank.capacity)
            return self.lib.imc_step_transport(ctypes.byref(self.cmesh), ctypes.byref(mat), ctypes.byref(par),
                                               ctypes.byref(cb), ctypes.byref(self.ctal), wsp, wsn,
                                               ctypes.byref(rep), self._stream())

        cb = self._call_bank("imc_step_transport", run, self.bank, lambda: rep.required_capacity)
        self.bank.size = int(cb.size)
        self._census_dev_valid = False
        res = StepResult(report=rep)
        return res

    def material_update(self, e: torch.Tensor, tr: torch.Tensor) -> None:
        _lib.check("imc_material_update", self.lib.imc_material_update(
            ctypes.byref(self.cmesh), ctypes.byref(self.ctal), _ptr(e), _ptr(tr), self._stream()))

    def material_update_law(self, e, tr, T, law, sigma_next, cv_next) -> None:
        """material_update, then T = e / cv and the next step's opacity and heat capacity of a
        device-evaluated material law (imc_material_update_law), in one kernel."""
        _lib.check("imc_material_update_law", self.lib.imc_material_update_law(
            ctypes.byref(self.cmesh), ctypes.byref(self.ctal), ctypes.byref(law), _ptr(e), _ptr(tr), _ptr(T),
            _ptr(sigma_next), _ptr(cv_next), self._stream()))

    def comb(self, n_max: int, step: int, per_group: bool = False, conserve_radiation: bool = False) -> ImcCombReport:
        """Comb the bank (n_max > 0: to n_max; 0: drop dead entries only; < 0: to |n_max| once
        at least |n_max| entries are alive)."""
        rep = ImcCombReport()
        src = self.bank
        dst = self.spare
        dst.size = 0
        # n_max <= 0 keeps at most every input entry (a threshold comb makes <= the live count)
        dst.ensure((int(n_max) if n_max > 0 else src.size) + 2 * self.nc * self.ng + 1024)
        flags = _comb_flags(per_group, conserve_radiation)
        cin = src.c()

        def run(cb):
            wsp, wsn = self._ws(max(src.size, 1))
            return self.lib.imc_comb(ctypes.byref(self.cmesh), ctypes.byref(cin), ctypes.byref(cb), int(n_max),
                                     self.comb_seed, int(step) & 0xFFFFFFFF, flags, _ptr(self.disc), wsp, wsn,
                                     ctypes.byref(rep), self._stream())

        cb = self._call_bank("imc_comb", run, dst, lambda: rep.required_capacity)
        dst.size = int(cb.size)
        self.bank, self.spare = dst, src
        self._census_dev_valid = False
        return rep

    def energy_totals(self, e: torch.Tensor) -> tuple[float, float]:
        rad = ctypes.c_double(0.0)
        internal = ctypes.c_double(0.0)
        wsp, wsn = self._ws(max(self.bank.capacity, 1))
        cb = self.bank.c()
        _lib.check("imc_energy_totals", self.lib.imc_energy_totals(
            ctypes.byref(self.cmesh), ctypes.byref(cb), _ptr(e), ctypes.byref(rad), ctypes.byref(internal),
            wsp, wsn, self._stream()))
        return rad.value, internal.value

    def host_stats(self) -> tuple[np.ndarray, np.ndarray]:
        return self.stats.cpu().numpy(), self.escaped.cpu().numpy()

    # ------------------------------------------------------------------ asynchronous step
    # One step = transport_async -> material_update -> (caller's inv_eos) -> comb_async ->
    # fetch(): a single device->host copy of the summary and one stream synchronisation.
    def _params(self, step, dt, theta, n_target, n_boundary, n_source, face_T, reflect, max_events,
                rz_linear_source, t_emit_floor, n_boundary_side=None, method=0, cf_fastpath=0.0,
                step_dev=None, dt_dev=None) -> ImcStepParams:
        par = ImcStepParams()
        par.seed = self.seed
        par.step = int(step) & 0xFFFFFFFF
        for q in range(4):
            par.reflect[q] = int(bool(reflect[q])) if q < len(reflect) else 0
            par.face_T[q] = _ptr(face_T[q]) if q < len(face_T) and face_T[q] is not None else None
        par.dt, par.theta = float(dt), float(theta)
        par.n_target, par.n_boundary, par.n_source = int(n_target), int(n_boundary), int(n_source)
        par.max_events = int(max_events)
        par.rz_linear_source = int(bool(rz_linear_source))
        par.t_emit_floor = float(t_emit_floor)
        par.block_size = int(self.launch["block_size"])
        par.blocks_per_sm = int(self.launch["blocks_per_sm"])
        par.chunk = int(self.launch["chunk"])
        # bit 0: shared-memory cell table; block tallies in shared memory: bit 1 on, bit 2 off
        # (launch["smem_tally"] 1 / 0; absent or None: the library's default)
        st = self.launch.get("smem_tally")
        par.reserved = int(bool(self.launch.get("smem_cells", 0))) | (2 if st == 1 else 4 if st == 0 else 0)
        # bit 3: the event-by-event form of the tracking (launch["event_based"] = 1)
        if self.launch.get("event_based"):
            par.reserved |= 8
        # bit 4: prefetched refills (launch["prefetch"] = 1)
        if self.launch.get("prefetch"):
            par.reserved |= 16
        par.emission_fractions = _ptr(self.emission_fractions)
        for q, n in enumerate(n_boundary_side or ()):
            par.n_boundary_side[q] = int(n)
        par.method = int(method)
        par.cf_fastpath = float(cf_fastpath)
        par.step_dev = _ptr(step_dev)
        par.dt_dev = _ptr(dt_dev)
        par.id_base = int(self.id_base)
        par.energy_share = float(self.energy_share)
        return par

    def _set_census_count(self, n: int) -> None:
        self.summary_dev[:8].copy_(torch.tensor([int(n)], dtype=torch.int64).view(torch.uint8))
        self._census_dev_valid = True

    def transport_async(self, T, sigma, cv, source, step, dt, theta, n_target, n_boundary, n_source, face_T,
                        reflect, max_events=0, rz_linear_source=True, t_emit_floor=0.0, n_boundary_side=None,
                        method=0, cf_fastpath=0.0, step_dev=None, dt_dev=None) -> int:
        """Sources + tracking without a host synchronisation.  Returns the host upper bound
        of the tracked bank size (the true size is in the device summary).  step_dev / dt_dev:
        device scalars (int32 / float64) the kernels read the step counter and dt from, for a
        captured step replayed with new values."""
        if not self._census_dev_valid:
            self._set_census_count(self.bank.size)
        self._last_transport = ((T, sigma, cv, source, step, dt, theta, n_target, n_boundary, n_source, face_T,
                                 reflect), dict(max_events=max_events, rz_linear_source=rz_linear_source,
                                                t_emit_floor=t_emit_floor, n_boundary_side=n_boundary_side,
                                                method=method, cf_fastpath=cf_fastpath))
        self._mat = ImcMaterial(_ptr(T), _ptr(sigma), _ptr(cv), _ptr(source))
        self._par = self._params(step, dt, theta, n_target, n_boundary, n_source, face_T, reflect, max_events,
                                 rz_linear_source, t_emit_floor, n_boundary_side, method, cf_fastpath,
                                 step_dev, dt_dev)
        self._census_bins = 0
        if self.fuse_census and not self.launch.get("event_based"):
            self._census_bins = _lib.CENSUS_BY_GROUP_CELL if self.ng > 1 else _lib.CENSUS_BY_CELL
        self._par.census_bins = self._census_bins
        bound = int(self.lib.imc_source_bound(ctypes.byref(self.cmesh), ctypes.byref(self._par)))
        self.bank.ensure(self.bank.size + bound)
        wsp, wsn = self._ws(self.bank.capacity)
        cb = self.bank.c()
        st = self.lib.imc_step_transport_async(ctypes.byref(self.cmesh), ctypes.byref(self._mat),
                                               ctypes.byref(self._par), ctypes.byref(cb),
                                               ctypes.byref(self.ctal_async), wsp, wsn, self.summary_dev.data_ptr(),
                                               self._stream())
        _lib.check("imc_step_transport_async", st)
        self._upper = self.bank.size + bound
        return self._upper

    def comb_async(self, n_max: int, step: int, e: torch.Tensor | None, per_group: bool = False,
                   conserve_radiation: bool = False, step_dev: torch.Tensor | None = None,
                   out_capacity: int | None = None, n_max_dev: torch.Tensor | None = None,
                   write_after: bool = False) -> None:
        """Queue the comb (n_max semantics as comb()); fetch() completes it.  step_dev: device
        step counter (graph replay); n_max_dev: device int64 comb target read when the comb runs
        (with step_dev; n_max > 0 then sizes the spare bank); out_capacity: cap the combed census
        below the spare bank's capacity (a larger one is flagged as an overflow and the census
        is emptied); write_after: the energy after the comb per bin goes to comb_after."""
        self.spare.size = 0
        want = int(1.15 * n_max) if n_max > 0 else self._upper
        self.spare.ensure(want + 2 * self.nc * self.ng + 4096)
        if n_max_dev is not None and (step_dev is None or n_max <= 0):
            raise ValueError("n_max_dev needs step_dev and n_max > 0")
        flags = _comb_flags(per_group, conserve_radiation) | (_lib.COMB_WRITE_AFTER if write_after else 0)
        want_bins = _lib.CENSUS_BY_GROUP_CELL if per_group else _lib.CENSUS_BY_CELL
        if self._census_bins and self._census_bins == want_bins:
            flags |= _lib.COMB_CENSUS_READY  # the tracking of this bank summed its census
        self._census_bins = 0
        self._comb_args = (int(n_max), int(step), e, flags, step_dev, out_capacity, n_max_dev)
        self._launch_comb()

    def _launch_comb(self) -> None:
        n_max, step, e, flags, step_dev, out_capacity, n_max_dev = self._comb_args
        cin = self.bank.c()
        cin.size = self._upper
        cout = self.spare.c()
        if out_capacity is not None:
            cout.capacity = min(int(out_capacity), cout.capacity)
        wsp, wsn = self._ws(max(self._upper, self.bank.capacity))
        if step_dev is not None:
            st = self.lib.imc_comb_async_dev(ctypes.byref(self.cmesh), ctypes.byref(cin), ctypes.byref(cout), n_max,
                                             None if n_max_dev is None else n_max_dev.data_ptr(), self.comb_seed,
                                             step_dev.data_ptr(), flags, _ptr(self.disc), _ptr(e),
                                             wsp, wsn, self.summary_dev.data_ptr(), self._stream())
            _lib.check("imc_comb_async_dev", st)
            return
        st = self.lib.imc_comb_async(ctypes.byref(self.cmesh), ctypes.byref(cin), ctypes.byref(cout), n_max,
                                     self.comb_seed, step & 0xFFFFFFFF, flags, _ptr(self.disc), _ptr(e),
                                     wsp, wsn, self.summary_dev.data_ptr(), self._stream())
        _lib.check("imc_comb_async", st)

    def census_energy_async(self, out: torch.Tensor, per_group: bool = True) -> None:
        """Queue, after comb_async, the energy per bin ((group, cell), or cell) of the comb's
        output (the next census) into out; the entry count is read on the device.  A comb that
        fetch() has to repeat (overflow) makes this stale: fetch() then sets comb_repeated."""
        cb = self.spare.c()
        cb.size = cb.capacity
        off = ImcStepSummary.n_out.offset
        st = self.lib.imc_bank_energy_by_bin(ctypes.byref(self.cmesh), ctypes.byref(cb),
                                            self.summary_dev.data_ptr() + off, int(bool(per_group)), _ptr(out),
                                            self._stream())
        _lib.check("imc_bank_energy_by_bin", st)

    def side_stream(self) -> torch.cuda.Stream:
        """A second stream of the engine's device (created once): device-to-host copies of
        fields that are final before the comb run on it beside the comb."""
        side = self.__dict__.get("_side_stream")
        if side is None:
            side = torch.cuda.Stream(device=self.device)
            self.__dict__["_side_stream"] = side
        return side

    def report_buffer(self) -> torch.Tensor:
        """self.report_dev, (2G + 3) nc + 2G doubles (allocated once)."""
        n = (2 * self.ng + 3) * self.nc + 2 * self.ng
        if getattr(self, "report_dev", None) is None or self.report_dev.numel() != n:
            self.report_dev = torch.empty(n, dtype=torch.float64, device=self.device)
        return self.report_dev

    def mg_report_fields(self, e: torch.Tensor, T: torch.Tensor, Tr: torch.Tensor, sections: str = "all") -> int:
        """Queue imc_mg_report_fields into self.report_dev (2-D multigroup): the radiation
        energy by group before (si / c) and after the comb (comb_after / V), e, T, Tr and the
        boundary / escaped energy by group, in the reference's array order.  sections: "all";
        "early" (all but the post-comb energies, which are final only after the comb); "post"
        (those alone).  Returns the buffer's length in doubles."""
        n = self.report_buffer().numel()
        early, post = sections in ("all", "early"), sections in ("all", "post")
        _lib.check("imc_mg_report_fields", self.lib.imc_mg_report_fields(
            ctypes.byref(self.cmesh), _ptr(self.si) if early else None, _ptr(self.comb_after) if post else None,
            _ptr(e) if early else None, _ptr(T) if early else None, _ptr(Tr) if early else None,
            _ptr(self.boundary_group) if early else None, _ptr(self.escaped_group) if early else None,
            _ptr(self.report_dev), self._stream()))
        return n

    def fetch(self, host_copies=()) -> ImcStepSummary:
        """Copy the summary (and any (device, pinned host) pairs) to the host and synchronise.
        A comb overflow is handled by growing the output bank and combing again (the input
        bank is untouched by the comb)."""
        stream = torch.cuda.current_stream(self.device)
        for d, h in host_copies:
            h.copy_(d, non_blocking=True)
        self.summary_host.copy_(self.summary_dev, non_blocking=True)
        stream.synchronize()
        _lib.TRANSFER["d2h"] += self.summary_host.numel()
        sm = self.summary
        self.comb_repeated = False
        if sm.flags & _lib.FLAG_BOUNDS:
            raise _lib.ImcError("bounds check", 9)
        if sm.flags & _lib.FLAG_NONFINITE:
            raise _lib.ImcError("imc_step_transport_async", 3)
        if sm.flags & _lib.FLAG_EVENT_CAP:
            raise _lib.ImcError("imc_step_transport_async", 2)
        if sm.flags & _lib.FLAG_COMB_OVERFLOW:
            self.spare.ensure(int(sm.n_out * 1.1) + 1024)
            off = ImcStepSummary.flags.offset
            self.summary_dev[off:off + 4].zero_()
            self._launch_comb()
            self.comb_repeated = True
            self.summary_host.copy_(self.summary_dev, non_blocking=True)
            stream.synchronize()
            if sm.flags & _lib.FLAG_COMB_OVERFLOW:
                raise _lib.ImcError("imc_comb_async", 1)
        self.spare.size = int(sm.n_out)
        self.bank.size = int(sm.n_bank)
        self.bank, self.spare = self.spare, self.bank
        self._census_dev_valid = True  # the comb wrote n_census = n_out
        return sm

    def phase_times(self) -> tuple[float, float]:
        a, b = ctypes.c_float(0), ctypes.c_float(0)
        if self.lib.imc_phase_times(ctypes.byref(a), ctypes.byref(b)) != 0:
            return 0.0, 0.0
        return a.value, b.value
