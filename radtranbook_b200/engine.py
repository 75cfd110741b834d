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
from ._lib import ImcBank, ImcCombReport, ImcMaterial, ImcMesh, ImcStepParams, ImcStepReport, ImcTallies

A_RAD = 0.01372
C_LIGHT = 29.98


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


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
                 capacity: int = 1 << 16, device: torch.device | None = None):
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
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.e1 = torch.as_tensor(e1, **f64)
        self.e2 = torch.as_tensor(e2, **f64)
        self.vol = torch.as_tensor(np.asarray(volumes, dtype=np.float64).reshape(-1), **f64)
        if self.vol.numel() != self.nc:
            raise ValueError("volumes must have nx*ny entries")
        self.cmesh = ImcMesh(self.gcode, self.nx, self.ny, n_groups, _ptr(self.e1), _ptr(self.e2), _ptr(self.vol), None)
        ncg = self.nc * n_groups
        self.dep = torch.zeros(ncg, **f64)
        self.si = torch.zeros(ncg, **f64)
        self.emitted = torch.zeros(self.nc, **f64)
        self.sigma_a = torch.zeros(ncg, **f64)
        self.sigma_s = torch.zeros(ncg, **f64)
        self.escaped = torch.zeros(4 + n_groups, **f64)
        self.stats = torch.zeros(_lib.STAT_N, dtype=torch.int64, device=dev)
        self.disc = torch.zeros(ncg, **f64)
        self.ctal = ImcTallies(_ptr(self.dep), _ptr(self.si), _ptr(self.emitted), _ptr(self.sigma_a),
                               _ptr(self.sigma_s), _ptr(self.escaped), _ptr(self.stats))
        mg = n_groups > 1
        self.bank = Bank(capacity, dev, mg)
        self.spare = Bank(capacity, dev, mg)
        self.ws = torch.empty(0, dtype=torch.uint8, device=dev)
        self.launch = dict(block_size=0, blocks_per_sm=0, chunk=0)

    # ------------------------------------------------------------------ helpers
    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def _ws(self, capacity: int) -> tuple[int, int]:
        need = int(self.lib.imc_workspace_bytes(ctypes.byref(self.cmesh), int(capacity)))
        if self.ws.numel() < need:
            self.ws = torch.empty(int(need * 1.25) + 4096, dtype=torch.uint8, device=self.device)
        return self.ws.data_ptr(), self.ws.numel()

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
                                      self.seed, ctypes.byref(cb), wsp, wsn, ctypes.byref(n_out), self._stream())
        _lib.check("imc_init_census", st)
        self.bank.size = int(cb.size)
        return self.bank.size

    def transport(self, T: torch.Tensor, sigma: torch.Tensor, cv: torch.Tensor, source: torch.Tensor | None,
                  step: int, dt: float, theta: float, n_target: int, n_boundary: int, n_source: int,
                  face_T: list, reflect, max_events: int = 0, rz_linear_source: bool = True,
                  t_emit_floor: float = 0.0) -> StepResult:
        mat = ImcMaterial(_ptr(T), _ptr(sigma), _ptr(cv), _ptr(source))
        faces = [None if f is None else _ptr(f) for f in face_T]
        par = ImcStepParams()
        par.seed = self.seed
        par.step = int(step) & 0xFFFFFFFF
        for q in range(4):
            par.reflect[q] = int(bool(reflect[q])) if q < len(reflect) else 0
            par.face_T[q] = faces[q] if q < len(faces) else None
        par.dt, par.theta = float(dt), float(theta)
        par.n_target, par.n_boundary, par.n_source = int(n_target), int(n_boundary), int(n_source)
        par.max_events = int(max_events)
        par.rz_linear_source = int(bool(rz_linear_source))
        par.t_emit_floor = float(t_emit_floor)
        par.block_size = int(self.launch["block_size"])
        par.blocks_per_sm = int(self.launch["blocks_per_sm"])
        par.chunk = int(self.launch["chunk"])
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
        res = StepResult(report=rep)
        return res

    def material_update(self, e: torch.Tensor, tr: torch.Tensor) -> None:
        _lib.check("imc_material_update", self.lib.imc_material_update(
            ctypes.byref(self.cmesh), ctypes.byref(self.ctal), _ptr(e), _ptr(tr), self._stream()))

    def comb(self, n_max: int, step: int, per_group: bool = False) -> ImcCombReport:
        rep = ImcCombReport()
        src = self.bank
        dst = self.spare
        dst.size = 0
        dst.ensure(int(n_max) + 2 * self.nc * self.ng + 1024)
        cin = src.c()

        def run(cb):
            wsp, wsn = self._ws(max(src.size, 1))
            return self.lib.imc_comb(ctypes.byref(self.cmesh), ctypes.byref(cin), ctypes.byref(cb), int(n_max),
                                     self.seed, int(step) & 0xFFFFFFFF, int(per_group), _ptr(self.disc), wsp, wsn,
                                     ctypes.byref(rep), self._stream())

        cb = self._call_bank("imc_comb", run, dst, lambda: rep.required_capacity)
        dst.size = int(cb.size)
        self.bank, self.spare = dst, src
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
