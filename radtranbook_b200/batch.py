"""Many independent 1-D gray slab problems in one set of launches (the batched form).

The reference advances one problem per call (IMC/IMC1D.py:908 step); a batch of
independent problems is a host loop over instances.  Here every phase of a time step runs
once for the whole batch: per-instance planning kernels (one block per instance), one
source-fill launch, one persistent tracking kernel whose work queue spans every instance's
histories (uneven instances share the GPU instead of each draining it alone), the fused
material + Fleck update, the comb, and a per-instance FP64 energy ledger.  A step reads
all its counts from device memory, so it is captured once in a CUDA graph and replayed.

Instance k uses its own Philox key and draws, in the same bank order, the numbers a
single-problem run (radtranbook_b200.imc1d with seed=key) draws, so each instance
reproduces that run; `run_plain` runs the same batch that way, one instance after the
other, as the baseline form.

Material model per instance: sigma_a = A T^p (p = -3 below), e = cv T.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .engine import require_cuda
from .rng import philox4x32_10, u01 as _u01

TAG_INSTANCE = 0x70000000  # Philox stream of per-instance keys and parameters


# --------------------------------------------------------------------------- problem
@dataclass
class BatchSpec:
    """K independent slab problems.  Per-instance arrays have length K."""
    n_cells: np.ndarray          # int
    length: np.ndarray           # cm
    n_target: np.ndarray         # emission particles per step
    n_boundary: np.ndarray       # boundary particles per step (left face)
    n_max: np.ndarray            # comb target
    opacity_a: np.ndarray        # sigma_a = A T^p
    opacity_p: np.ndarray
    cv: np.ndarray               # GJ/(cm^3 keV)
    face_T: np.ndarray           # (K, 2) keV, <= 0: no source
    reflect: np.ndarray          # (K,) bit mask
    seed: np.ndarray             # (K,) uint64 Philox keys
    T0: float = 0.001
    Tr0: float = 0.001
    dt: float = 0.01
    theta: float = 1.0
    edges: list = field(default_factory=list)

    @property
    def K(self) -> int:
        return len(self.n_cells)

    def __post_init__(self):
        if not self.edges:
            self.edges = [np.linspace(0.0, float(L), int(n) + 1) for n, L in zip(self.n_cells, self.length)]


def uneven_slab_batch(n_inst: int = 256, master_seed: int = 0xB200, particle_scale: float = 1.0,
                      dt: float = 0.01) -> BatchSpec:
    """The uneven 256-instance Marshak-wave batch: per instance, from its own Philox stream
    under the master key, cells ~ U{50..800}, length ~ U[0.05, 1] cm, particles per step
    N = 10^U[4, 6] (times particle_scale; half emission, half boundary), NMax = 4 N,
    sigma_a = A T^-3 with A = 10^U[1, 3], cv ~ U[0.05, 1], left-face T ~ U[0.3, 2] keV,
    vacuum faces, T0 = Tr0 = 0.001 keV."""
    K = int(n_inst)
    ks = np.arange(K, dtype=np.uint64)
    z = np.zeros(K, dtype=np.uint64)
    keys = philox4x32_10(np.stack([ks, z, z, z + TAG_INSTANCE], 1), master_seed).astype(np.uint64)
    seeds = keys[:, 0] | (keys[:, 1] << np.uint64(32))
    a = _u01(philox4x32_10(np.stack([ks, z + 1, z, z + TAG_INSTANCE], 1), master_seed))
    b = _u01(philox4x32_10(np.stack([ks, z + 2, z, z + TAG_INSTANCE], 1), master_seed))
    n_cells = 50 + np.minimum((a[:, 0] * 751).astype(np.int64), 750)
    length = 0.05 + 0.95 * a[:, 1]
    N = np.maximum(np.round(10.0 ** (4.0 + 2.0 * a[:, 2]) * particle_scale).astype(np.int64), 2)
    A = 10.0 ** (1.0 + 2.0 * a[:, 3])
    cv = 0.05 + 0.95 * b[:, 0]
    Tb = 0.3 + 1.7 * b[:, 1]
    n_boundary = N // 2
    n_target = N - n_boundary
    face = np.stack([Tb, np.zeros(K)], 1)
    return BatchSpec(n_cells=n_cells, length=length, n_target=n_target, n_boundary=n_boundary, n_max=4 * N,
                     opacity_a=A, opacity_p=np.full(K, -3.0), cv=cv, face_T=face, reflect=np.zeros(K, np.int32),
                     seed=seeds, dt=dt)


def slot_plan(spec: BatchSpec) -> tuple[np.ndarray, np.ndarray, int]:
    """Bank slots per instance: the largest census the comb may leave (NMax + cells + a
    margin of many standard deviations of the comb's copy count) next to one step's new
    particles.  Returns (slot_off[K+1], new_max[K], total new bound)."""
    sides = (np.asarray(spec.face_T) > 0).sum(1)
    new_max = sides * spec.n_boundary + spec.n_target + spec.n_cells
    census = spec.n_max + spec.n_cells + np.ceil(6.0 * np.sqrt(spec.n_max + new_max)).astype(np.int64) + 64
    census = np.maximum(census, spec.n_target + spec.n_cells)
    slots = census + new_max
    off = np.concatenate([[0], np.cumsum(slots)]).astype(np.int64)
    return off, new_max.astype(np.int64), int(new_max.sum())


# --------------------------------------------------------------------------- engine
# form: 1 work units (a block takes chunk x warps entries of one instance at a time and keeps
# its cell table and tallies in shared memory), 2 the entry queue (warps take entries of any
# instance; for many small instances), 3 work units whose lanes prefetch their next history's
# bank record into shared memory; the engine's default follows the particles per instance
DEFAULT_LAUNCH = {"block_size": 256, "blocks_per_sm": 4, "chunk": 1024, "refill_min": 1, "form": 0}
UNITS_MIN_PARTICLES = 20_000  # mean particles per instance from which work units are the default


class BatchEngine:
    """Device state of a batch and its step (eager or as a replayed CUDA graph)."""

    def __init__(self, spec: BatchSpec, device: torch.device | None = None):
        self.spec = spec
        self.device = device or require_cuda()
        self.lib = _lib.load()
        dev = self.device
        K = spec.K
        i64 = dict(dtype=torch.int64, device=dev)
        f64 = dict(dtype=torch.float64, device=dev)
        cell_off = np.concatenate([[0], np.cumsum(spec.n_cells)]).astype(np.int32)
        self.cell_off_h = cell_off
        self.n_cells = int(cell_off[-1])
        slot_off, new_max, max_new = slot_plan(spec)
        self.slot_off_h = slot_off
        self.n_slots = int(slot_off[-1])
        if self.n_slots >= 2 ** 31:
            raise ValueError("batch needs more than 2^31 bank slots")
        t = lambda x, **kw: torch.as_tensor(np.ascontiguousarray(x), **kw)  # noqa: E731
        self.d = {
            "cell_off": t(cell_off, dtype=torch.int32, device=dev),
            "edges": t(np.concatenate(spec.edges), **f64),
            "slot_off": t(slot_off, **i64),
            "seed": t(np.asarray(spec.seed, dtype=np.uint64).view(np.int64), **i64),
            "n_target": t(np.asarray(spec.n_target, np.int64), **i64),
            "n_boundary": t(np.asarray(spec.n_boundary, np.int64), **i64),
            "n_max": t(np.asarray(spec.n_max, np.int64), **i64),
            "face_T": t(np.asarray(spec.face_T, np.float64).reshape(-1), **f64),
            "reflect": t(np.asarray(spec.reflect, np.int32), dtype=torch.int32, device=dev),
            "opacity_a": t(np.asarray(spec.opacity_a, np.float64), **f64),
            "opacity_p": t(np.asarray(spec.opacity_p, np.float64), **f64),
            "cv": t(np.asarray(spec.cv, np.float64), **f64),
        }
        p = lambda name: self.d[name].data_ptr()  # noqa: E731
        self.cb = _lib.ImcBatch(K, self.n_cells, self.n_slots, max_new, float(spec.dt), float(spec.theta),
                                p("cell_off"), p("edges"), p("slot_off"), p("seed"), p("n_target"), p("n_boundary"),
                                p("n_max"), p("face_T"), p("reflect"), p("opacity_a"), p("opacity_p"), p("cv"),
                                int(np.max(spec.n_cells)))
        ns = self.n_slots
        self.banks = []
        for _ in range(2):
            self.banks.append({
                "pos1": torch.zeros(ns, dtype=torch.float32, device=dev),
                "dir1": torch.zeros(ns, dtype=torch.float32, device=dev),
                "weight": torch.zeros(ns, dtype=torch.float32, device=dev),
                "time": torch.zeros(ns, dtype=torch.float32, device=dev),
                "cell": torch.zeros(ns, dtype=torch.int32, device=dev),
            })
        nc = self.n_cells
        self.s = {
            "sel": torch.zeros(1, dtype=torch.int32, device=dev),
            "step": torch.zeros(1, dtype=torch.int32, device=dev),
            "n_census": torch.zeros(K, **i64),
            "T": torch.zeros(nc, **f64), "e": torch.zeros(nc, **f64), "tr": torch.zeros(nc, **f64),
            "dep": torch.zeros(nc, **f64), "si": torch.zeros(nc, **f64), "emitted": torch.zeros(nc, **f64),
            "ledger": torch.zeros(K * _lib.BL_N, **f64),
            "stats": torch.zeros(_lib.STAT_N, **i64),
            "flags": torch.zeros(1, dtype=torch.int32, device=dev),
        }
        banks_c = (_lib.ImcBank * 2)()
        for q, b in enumerate(self.banks):
            banks_c[q] = _lib.ImcBank(b["pos1"].data_ptr(), None, b["dir1"].data_ptr(), None, b["weight"].data_ptr(),
                                      b["time"].data_ptr(), b["cell"].data_ptr(), None, 0, ns)
        sp = lambda name: self.s[name].data_ptr()  # noqa: E731
        self.cs = _lib.ImcBatchState(banks_c, sp("sel"), sp("step"), sp("n_census"), sp("T"), sp("e"), sp("tr"),
                                     sp("dep"), sp("si"), sp("emitted"), sp("ledger"), sp("stats"), sp("flags"))
        self.ws = torch.empty(int(self.lib.imc_batch_workspace_bytes(ctypes.byref(self.cb))), dtype=torch.uint8,
                              device=dev)
        self.launch = dict(DEFAULT_LAUNCH)
        mean_particles = float(np.mean(spec.n_target + spec.n_boundary))
        self.launch["form"] = 1 if mean_particles >= UNITS_MIN_PARTICLES else 2
        self.graph = None
        self._graph_launch = None

    # ------------------------------------------------------------------ steps
    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def init(self) -> None:
        T0 = torch.full((self.n_cells,), float(self.spec.T0), dtype=torch.float64, device=self.device)
        Tr0 = torch.full((self.n_cells,), float(self.spec.Tr0), dtype=torch.float64, device=self.device)
        _lib.check("imc_batch_init", self.lib.imc_batch_init(ctypes.byref(self.cb), ctypes.byref(self.cs),
                                                             T0.data_ptr(), Tr0.data_ptr(), self.ws.data_ptr(),
                                                             self.ws.numel(), self._stream()))

    def _launch_c(self) -> _lib.ImcBatchLaunch:
        L = self.launch
        return _lib.ImcBatchLaunch(int(L["block_size"]), int(L["blocks_per_sm"]), int(L["chunk"]),
                                   int(L["refill_min"]), int(L.get("form", 0)))

    def step_eager(self) -> None:
        """Enqueue one step of every instance (no synchronisation)."""
        lc = self._launch_c()
        _lib.check("imc_batch_step", self.lib.imc_batch_step(ctypes.byref(self.cb), ctypes.byref(self.cs),
                                                             ctypes.byref(lc), self.ws.data_ptr(), self.ws.numel(),
                                                             self._stream()))

    def capture(self) -> None:
        """Capture one step in a CUDA graph (with the current launch shape)."""
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step_eager()
        self.graph = g
        self._graph_launch = dict(self.launch)

    def step(self, n: int = 1, graph: bool = True) -> None:
        """Enqueue n steps; with graph=True each is one replay of the captured step."""
        if graph and (self.graph is None or self._graph_launch != self.launch):
            self.capture()
        for _ in range(n):
            if graph:
                self.graph.replay()
            else:
                self.step_eager()

    # ------------------------------------------------------------------ results
    def check(self) -> None:
        torch.cuda.synchronize(self.device)
        f = int(self.s["flags"].item())
        if f & 4:
            raise _lib.ImcError("imc_batch_step (a bank slot range overflowed)", _lib.BANK_OVERFLOW)
        if f & 2:
            raise AssertionError("non-finite or non-positive material state in the batch")
        if f & 1:
            raise _lib.ImcError("imc_batch_step (events-per-history safety cap)", 2)

    def ledger(self) -> np.ndarray:
        return self.s["ledger"].view(self.spec.K, _lib.BL_N).cpu().numpy()

    def field(self, name: str) -> list[np.ndarray]:
        x = self.s[name].cpu().numpy()
        return [x[self.cell_off_h[k]:self.cell_off_h[k + 1]].copy() for k in range(self.spec.K)]

    def steps_done(self) -> int:
        return int(self.s["step"].item())

    def total_events(self) -> int:
        return int(self.s["stats"][_lib.STAT_EVENTS].item())

    def census_sizes(self) -> np.ndarray:
        return self.s["n_census"].cpu().numpy()

    # ------------------------------------------------------------------ tuning
    def _snapshot(self) -> dict:
        sel = int(self.s["sel"].item())
        snap = {"bank": {k: v.clone() for k, v in self.banks[sel].items()}, "sel": sel,
                "s": {k: v.clone() for k, v in self.s.items()}, "ws": self.ws.clone()}
        return snap

    def _restore(self, snap: dict) -> None:
        for k, v in snap["bank"].items():
            self.banks[snap["sel"]][k].copy_(v)
        for k, v in snap["s"].items():
            self.s[k].copy_(v)
        self.ws.copy_(snap["ws"])


TUNE_GRID = {
    "block_size": (128, 256),
    "blocks_per_sm": (4, 8),
    "chunk": (256, 1024, 4096),
    "refill_min": (1, 4, 16),
    "form": (1, 2),  # form 3 (prefetched refills) measured slower; selectable, not tuned
}


def tune(engine: BatchEngine, grid: dict | None = None, repeats: int = 1) -> dict:
    """Choose the tracking launch shape (block size, blocks per SM, work-queue ticket
    size = the bank tile a warp takes, refill cadence = how many idle lanes a warp
    collects before it compacts them, and the form: work units or the entry queue) by timing
    whole eager steps of the batch from its current state (restored before every trial, so
    each trial is the same work)."""
    import itertools

    g = dict(TUNE_GRID if grid is None else grid)
    keys = list(g)
    snap = engine._snapshot()
    results = []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for vals in itertools.product(*(g[k] for k in keys)):
        cand = dict(zip(keys, vals))
        engine.launch.update(cand)
        best = float("inf")
        for _ in range(repeats):
            engine._restore(snap)
            torch.cuda.synchronize(engine.device)
            e0.record()
            engine.step_eager()
            e1.record()
            torch.cuda.synchronize(engine.device)
            best = min(best, e0.elapsed_time(e1))
        results.append((best, cand))
    engine._restore(snap)
    torch.cuda.synchronize(engine.device)
    results.sort(key=lambda r: r[0])
    engine.launch.update(results[0][1])
    return {"best": results[0][1], "best_ms": results[0][0], "worst_ms": results[-1][0],
            "trials": [(round(t, 4), c) for t, c in results]}


# --------------------------------------------------------------------------- plain form
def run_plain(spec: BatchSpec, steps: int, instances=None, launch: dict | None = None) -> dict:
    """The same batch through the single-problem drop-in (radtranbook_b200.imc1d), one
    instance after the other; device material callables, so each step synchronises the
    host once.  Returns per-instance final T, ledger closures, total events and each step's
    wall time (step_s[k][s], seconds; the step ends with its synchronisation)."""
    from . import imc1d
    from .materials import Constant, PowerLawOpacity, device_callable

    out = {"T": [], "Tr": [], "max_rel_closure": [], "events": 0, "step_s": []}
    ks = range(spec.K) if instances is None else instances
    for k in ks:
        nc = int(spec.n_cells[k])
        e = spec.edges[k]
        mesh = np.stack([e[:-1], e[1:]], 1)
        cvk = float(spec.cv[k])
        eos = device_callable(lambda T, cvk=cvk: cvk * T)
        inv_eos = device_callable(lambda en, cvk=cvk: en / cvk)
        sigma = PowerLawOpacity(float(spec.opacity_a[k]), -float(spec.opacity_p[k]))
        cv = Constant(cvk)
        st = imc1d.init_simulation(int(spec.n_target[k]), np.full(nc, spec.T0), np.full(nc, spec.Tr0), mesh, eos,
                                   inv_eos, seed=int(spec.seed[k]))
        if launch:
            st._engine.launch.update(launch)
        worst = 0.0
        refl = (bool(spec.reflect[k] & 1), bool(spec.reflect[k] & 2))
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            st, info = imc1d.step(st, int(spec.n_target[k]), int(spec.n_boundary[k]), 0, int(spec.n_max[k]),
                                  (float(spec.face_T[k][0]), float(spec.face_T[k][1])), spec.dt, mesh, sigma,
                                  inv_eos, cv, np.zeros(nc), reflect=refl, theta=spec.theta)
            times.append(time.perf_counter() - t0)
            worst = max(worst, abs(info["ledger"]["relative_closure"]))
            out["events"] += info["profiling"]["transport_events"]["total"]
        out["step_s"].append(times)
        out["T"].append(st.temperature.copy())
        out["Tr"].append(st.radiation_temperature.copy())
        out["max_rel_closure"].append(worst)
    return out


def run_batch(spec: BatchSpec, steps: int, graph: bool = True, autotune: bool = False) -> dict:
    """Initialise, optionally tune on the first step's state, run `steps` steps; returns
    per-instance final T, ledger and timing."""
    eng = BatchEngine(spec)
    eng.init()
    tuned = tune(eng) if autotune else None
    torch.cuda.synchronize(eng.device)
    t0 = time.perf_counter()
    eng.step(steps, graph=graph)
    eng.check()
    dt = time.perf_counter() - t0
    return {"engine": eng, "T": eng.field("T"), "ledger": eng.ledger(), "seconds": dt, "tuned": tuned,
            "events": eng.total_events()}


def instance_events_per_second(events: int, seconds: float) -> float:
    return events / seconds if seconds > 0 else math.nan
