"""Benchmark: IMC track segments per second on the 2-D RZ crooked-pipe time step.

One "step" is one full implicit Monte Carlo time step of the 60x210 crooked pipe
(2e6 source particles per step, census combed to 6.67e6): Fleck factor, boundary and
emission sources, tracking of the whole bank to census, material update, comb.

  value   track segments/s with the whole step on the device (device material callables),
          inputs resident in HBM; timed with CUDA events on the launching stream.
  e2e     the same metric through the drop-in API (radtranbook_b200.imc2d.step) with the
          reference driver's NumPy material callables: host evaluation of sigma / cv /
          inv_eos and the host copies of T, Tr, e every step are inside the timed region.
  roofline  tracking kernel: algorithmic bytes = 72 B per 2-D segment (one 36-byte particle
          record loaded and stored per segment) x segments / kernel time (CUDA events in the
          library around the tracking launch), against the measured HBM copy bandwidth.
  cpu_baseline  the FP64 CPU oracle (a C++ port of the reference step, OpenMP over all host
          threads) on a reduced-particle sample of the same problem.

--impl reference runs that CPU port as the reference arm.  With --gpus N > 1 (torchrun), the
problem carries N times the one-GPU particle counts and the step is particle-partitioned over
the ranks (radtranbook_b200.partition: each rank tracks its share with its own Philox id range
and 1/N of the source energy; the per-cell tallies are summed with one NCCL all-reduce per
step), so the work per GPU is the one-GPU workload's ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "IMC track-segments/s and FOM=1/(rel.var*time) on 1 B200: plain vs batched/adjoint"
UNIT = "track-segments/s"
B_SEG_2D = 72  # bytes per 2-D gray segment: 36-byte record loaded + stored
B_SEG_2D_MG = 80  # 2-D multigroup: the 36-byte record plus the group index, loaded + stored
B_SEG_1D = 56  # 1-D gray: a 28-byte record loaded + stored
# DRAM bytes and warp instructions of the tracking kernel per segment on this workload, from
# one full-size launch under ncu (dram__bytes_read.sum + dram__bytes_write.sum = 402.25 MB,
# smsp__inst_executed.sum = 1.520 G, for 67.18 M segments); the histories stay in registers
# across their events, and the kernel is bound by instruction issue.
DRAM_B_PER_SEG_MEASURED = 402.252544e6 / 67176386
WARP_INST_PER_SEG_MEASURED = 1520147524 / 67176386
ISSUE_SLOTS_PER_CYCLE = 148 * 4  # SMs x warp schedulers, one warp instruction each per cycle


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.t0 = self.t1 = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.5)  # let the sampler start before the timed region
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        import datetime

        if not getattr(self, "out", ""):
            return None
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                if self.t0 is not None and not (self.t0 - 0.25 <= ts <= self.t1 + 0.25):
                    continue
                sm.append(float(f[2]))
                smax.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(names, f[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "note": "no nvidia-smi sample fell inside the timed region"}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_run(scale: float, steps: int, warmup: int, nthreads: int):
    """Crooked pipe on the FP64 CPU oracle at `scale` x the particle counts."""
    from oracle import oracle as O
    from radtranbook_b200 import problems

    p = problems.crooked_pipe(scale=scale)
    e1, e2 = p["edges1"], p["edges2"]
    vol = O.flat2d(np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :])
    rc = 0.5 * (e1[:-1] + e1[1:])
    face = [None, None, np.where(rc < 0.5, 0.5, 0.0), None]
    run = O.OracleGray("rz", e1, e2, vol, 0x5EED0001, p["Ntarget"], p["Tinit"], p["Tr_init"], p["eos_host"],
                       p["inv_eos_host"], nthreads=nthreads)
    kw = dict(Ntarget=p["Ntarget"], Nboundary=p["Nboundary"], Nsource=0, Nmax=p["Nmax"], face_T=face, dt=p["dt"],
              sigma_a_func=p["sigma_host"], inv_eos=p["inv_eos_host"], cv=p["cv_host"], reflect=p["reflect"],
              max_events=1_000_000)
    for _ in range(warmup):
        run.step(**kw)
    seg = 0
    hist = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        r = run.step(**kw)
        seg += int(r["stats"][0])
        hist += int(r["n_transported"])
    dt = time.perf_counter() - t0
    return seg / dt, hist / dt, dt, seg


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    scale = args.cpu_scale
    # the same workload and steps as the GPU arm (the crooked pipe at --cpu-scale x its particle
    # counts, 1 = the full configuration), on every host thread
    v, h, dt, seg = cpu_oracle_run(scale, args.steps, args.warmup, nthreads)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / max(args.steps, 1) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "crooked_pipe_rz_60x210", "source_particles_per_step": int(round(2e6 * scale)),
                   "nmax": int(round(6.67e6 * scale)), "sample_scale": scale},
        "histories_per_s": h,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": f"crooked pipe, {scale:g} x particles ({int(round(2e6 * scale))} src/step), "
                                   f"{args.warmup} warm-up + {args.steps} timed steps, FP64 C++ oracle, OpenMP"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _gpu_steps(p, state, steps, use_device, dist=None):
    """Run `steps` drop-in steps; return (segments, histories)."""
    from radtranbook_b200 import imc2d

    sig = p["sigma_dev"] if use_device else p["sigma_host"]
    cv = p["cv_dev"] if use_device else p["cv_host"]
    inv = p["inv_eos_dev"] if use_device else p["inv_eos_host"]
    seg = hist = 0
    info = None
    for _ in range(steps):
        state, info = imc2d.step(state, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"],
                                 p["edges1"], p["edges2"], sig, inv, cv, p["source"], reflect=p["reflect"],
                                 geometry="rz", boundary_source_func=p["boundary_source_func"],
                                 _allreduce=dist)
        te = info["profiling"]["transport_events"]
        seg += te["total"]
        hist += te["n_particles_transported"]
        CLOSURE[0] = max(CLOSURE[0], abs(info["ledger"]["relative_closure"]))
    return state, seg, hist, info


CLOSURE = [0.0]  # worst |energy closure| / total energy over the steps run


def _fom(x_runs: np.ndarray, t_runs: list) -> dict:
    """FOM = 1 / (R^2 T): R^2 = mean over the region of interest (cells whose mean tally
    exceeds 1e-3 of the largest) of Var_s(X_c) / mean_s(X_c)^2 across independent seeds,
    T = mean wall time of one run."""
    m = x_runs.mean(0)
    roi = m > 1e-3 * m.max()
    r2 = float(np.mean(x_runs[:, roi].var(0, ddof=1) / m[roi] ** 2))
    t = float(np.mean(t_runs))
    return {"fom": 1.0 / (r2 * t), "rel_var": r2, "rel_err": float(np.sqrt(r2)), "seconds_per_run": t,
            "seeds": int(x_runs.shape[0]), "roi_cells": int(roi.sum())}


def fom_gpu(p, steps: int, seeds: int, launch: dict | None) -> dict:
    """Crooked pipe, `steps` drop-in steps per seed (device material callables), last-step
    deposition per cell as the tally; run wall time by CUDA events around the steps."""
    import torch

    from radtranbook_b200 import imc2d

    xs, ts = [], []
    for s in range(seeds):
        st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                                   p["inv_eos_dev"], geometry="rz", seed=0xF0E00000 + s)
        if launch:
            st._engine.launch.update(launch)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        st, _, _, _ = _gpu_steps(p, st, steps, True)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e-3)
        xs.append(st._engine.dep[: st._engine.nc].double().cpu().numpy().copy())
    out = _fom(np.array(xs), ts)
    out["particles_per_step"] = p["Ntarget"] + p["Nboundary"]
    out["steps"] = steps
    return out


def fom_cpu(scale: float, steps: int, seeds: int, nthreads: int) -> dict:
    """The same FOM for the FP64 CPU oracle at `scale` x the particle counts (the FOM is
    nearly independent of the particle count: R^2 ~ 1/N, T ~ N)."""
    from oracle import oracle as O
    from radtranbook_b200 import problems

    p = problems.crooked_pipe(scale=scale)
    e1, e2 = p["edges1"], p["edges2"]
    vol = O.flat2d(np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :])
    rc = 0.5 * (e1[:-1] + e1[1:])
    face = [None, None, np.where(rc < 0.5, 0.5, 0.0), None]
    kw = dict(Ntarget=p["Ntarget"], Nboundary=p["Nboundary"], Nsource=0, Nmax=p["Nmax"], face_T=face, dt=p["dt"],
              sigma_a_func=p["sigma_host"], inv_eos=p["inv_eos_host"], cv=p["cv_host"], reflect=p["reflect"],
              max_events=1_000_000)
    xs, ts = [], []
    for s in range(seeds):
        run = O.OracleGray("rz", e1, e2, vol, 0xC0E00000 + s, p["Ntarget"], p["Tinit"], p["Tr_init"], p["eos_host"],
                           p["inv_eos_host"], nthreads=nthreads)
        t0 = time.perf_counter()
        r = None
        for _ in range(steps):
            r = run.step(**kw)
        ts.append(time.perf_counter() - t0)
        xs.append(np.asarray(r["dep"], dtype=np.float64).copy())
    out = _fom(np.array(xs), ts)
    out["particles_per_step"] = p["Ntarget"] + p["Nboundary"]
    out["steps"] = steps
    out["cores"] = nthreads
    return out


def form_batched(steps: int, tune: bool, n_inst: int = 256, particle_scale: float = 1.0, form: int = 0) -> dict:
    """Uneven slab batch (n_inst instances, per-instance particles 10^U[4,6] x particle_scale):
    the batched engine (one CUDA graph per step) and the plain form (the single-problem
    drop-in, one instance after the other) on the same histories (each instance draws
    identical Philox streams in both forms)."""
    import torch

    from radtranbook_b200 import _lib, batch

    spec = batch.uneven_slab_batch(n_inst=n_inst, particle_scale=particle_scale)
    eng = batch.BatchEngine(spec)
    if form:
        eng.launch["form"] = form  # fixed tracking form (1 work units, 2 entry queue)
    eng.init()
    tuned = None
    if tune:
        # tune on a developed state (the first step's histories, from the cold initial state,
        # are far shorter than the run's): five eager steps, then the tuner replays the sixth
        eng.step(5, graph=False)
        tuned = batch.tune(eng, grid={"block_size": (256,), "blocks_per_sm": (4, 8), "chunk": (1024, 4096),
                                      "refill_min": (1, 8), "form": (form,) if form else (1, 2)})
        eng.init()  # start over from the initial state
    eng.capture()
    torch.cuda.synchronize()
    # the batched steps in windows of `window` steps (CUDA events around each window)
    window = max(1, min(10, steps))
    win_b = []
    done = 0
    while done < steps:
        n = min(window, steps - done)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.step(n)
        e1.record()
        torch.cuda.synchronize()
        win_b.append(e0.elapsed_time(e1) * 1e-3)
        done += n
    eng.check()
    tb = float(sum(win_b))
    ev_b = eng.total_events()
    L = eng.ledger()
    t0 = time.perf_counter()
    pl = batch.run_plain(spec, steps, launch=None)
    torch.cuda.synchronize()
    tp = time.perf_counter() - t0
    # the plain loop's time in the same windows: every instance's steps of that window
    st_s = np.array(pl["step_s"])  # [instance, step]
    win_p = [float(st_s[:, w * window:(w + 1) * window].sum()) for w in range(len(win_b))]
    return {"workload": "uneven_slab_batch_%d%s" % (spec.K, "" if particle_scale == 1.0 else "_x%g" % particle_scale),
            "steps": steps, "instances": spec.K,
            "particles_per_step": int((spec.n_target + spec.n_boundary).sum()),
            "batched_segments_per_s": ev_b / tb, "plain_segments_per_s": pl["events"] / tp,
            "speedup": (ev_b / tb) / (pl["events"] / tp), "same_histories": bool(ev_b == pl["events"]),
            "batched_s": tb, "plain_s": tp,
            "windows": {"steps_per_window": window, "batched_s": win_b, "plain_s": win_p,
                        "speedup": [p_ / b_ for p_, b_ in zip(win_p, win_b)]},
            "energy_closure_max_rel": float(L[:, _lib.BL_MAX_REL].max()),
            "launch": dict(eng.launch), "autotune": None if tuned is None else
            {"best_ms": tuned["best_ms"], "worst_ms": tuned["worst_ms"], "candidates": len(tuned["trials"])}}


def form_adjoint(repeats: int = 3, fd_cells: int = 64) -> dict:
    """128 x 128 random-opacity XY step (4e6 histories): forward and VJP device time, and
    the VJP against central differences with common random numbers on random cells."""
    import torch

    from radtranbook_b200 import adjoint

    prob, sigma_np = adjoint.opacity_field_problem()
    sig = torch.as_tensor(sigma_np, device=prob.device)
    cot = torch.as_tensor(adjoint.unit_cotangent(prob.nc), device=prob.device)
    prob.forward(sig)
    prob.vjp(sig, cot)
    fw, bw = [], []
    for _ in range(repeats):
        prob.forward(sig)
        fw.append(prob.forward_ms)
    segs = int(prob.engine.host_stats()[0][0])
    for _ in range(repeats):
        g = prob.vjp(sig, cot)
        bw.append(prob.backward_ms)
    # central differences on `fd_cells` random cells drawn from the significant set: cells whose
    # VJP component is above 1e-3 of the largest (the others carry almost no deposition)
    gn = g.cpu().numpy()
    significant = np.flatnonzero(np.abs(gn) > 1e-3 * np.abs(gn).max())
    rng = np.random.default_rng(0xFDC)
    cells = rng.choice(significant, min(fd_cells, len(significant)), replace=False)
    fd = adjoint.fd_check(prob, sig, cot, cells, rel=1e-3)
    ga = gn[cells]
    rel = np.abs(ga - fd) / np.maximum(np.abs(fd), 1e-300)
    return {"workload": "random_opacity_xy_128x128", "histories": prob.setup.n_boundary,
            "forward_ms": float(np.median(fw)), "backward_ms": float(np.median(bw)),
            "backward_over_forward": float(np.median(bw) / np.median(fw)), "segments_per_forward": segs,
            "significant_cells": int(len(significant)), "fd_cells": int(len(cells)),
            "fd_rel_err_vector": float(np.linalg.norm(ga - fd) / np.linalg.norm(fd)),
            "fd_max_rel_err": float(rel.max()), "fd_median_rel_err": float(np.median(rel)),
            "fd_cells_within_2pct": int((rel <= 0.02).sum())}


def form_event_based(steps: int = 10, warmup: int = 5, launch: dict | None = None) -> dict:
    """The crooked-pipe step with the two forms of the tracking from the same state: the
    persistent history-based kernel (each warp keeps 32 histories in registers and refills
    idle lanes) and the event-by-event loop (one launch per event over the live histories,
    survivors compacted between launches).  Both follow identical histories; CUDA events
    around the tracking phase of each step."""
    import torch

    from radtranbook_b200 import imc2d, problems

    p = problems.crooked_pipe()
    out = {}
    for name, ev in (("history_based", False), ("event_based", True)):
        st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                                   p["inv_eos_dev"], geometry="rz", seed=0xE7E7)
        if launch:
            st._engine.launch.update(launch)
        st._engine.launch["event_based"] = 1 if ev else 0
        st, _, _, _ = _gpu_steps(p, st, warmup, True)
        seg = 0
        track = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            st, sg, _, info = _gpu_steps(p, st, 1, True)
            seg += sg
            track.append(info["profiling"]["phase_times_s"]["transport"] * 1e3)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[name] = {"ms_per_step": ms / steps, "track_ms_per_step": float(np.mean(track)),
                     "segments_per_step": seg / steps, "segments_per_s": seg / (ms * 1e-3),
                     "tracking_segments_per_s": seg / (float(np.sum(track)) * 1e-3)}
    out["event_over_history_tracking"] = (out["event_based"]["tracking_segments_per_s"]
                                          / out["history_based"]["tracking_segments_per_s"])
    out["workload"] = "crooked_pipe_rz_60x210"
    return out


def form_carter_forest(steps: int = 10, warmup: int = 2) -> dict:
    """The headline crooked-pipe step with Carter-Forest transport (IMC/IMC2D_CarterForest.py
    semantics): true absorption with delayed re-emission instead of the Fleck factor, same
    sources, mesh and particle counts; device material callables, CUDA-event timing."""
    import torch

    from radtranbook_b200 import imc2d_cf, problems

    p = problems.crooked_pipe(scale=1.0)
    st = imc2d_cf.init_simulation(p["Ntarget"], p["Tinit"], p["Tinit"], p["edges1"], p["edges2"], p["eos_dev"],
                                  p["inv_eos_dev"], geometry="rz", seed=0xCF0D)

    def run(n, st):
        seg = capt = reem = 0
        worst = 0.0
        for _ in range(n):
            st, info = imc2d_cf.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"],
                                     p["edges1"], p["edges2"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"],
                                     p["source"], reflect=p["reflect"], geometry="rz",
                                     boundary_source_func=p["boundary_source_func"])
            te = info["profiling"]["transport_events"]
            seg += te["total"]
            capt += te["absorption_capture_events"]
            reem += te["absorption_continue_events"]
            worst = max(worst, abs(info["ledger"]["relative_closure"]))
        return st, seg, capt, reem, worst

    st = run(warmup, st)[0]  # no info of the warm-up kept (its arrays view the step's buffer)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    st, seg, capt, reem, worst = run(steps, st)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"workload": "crooked_pipe_rz_60x210, Carter-Forest", "steps": steps, "segments_per_s": seg / (ms * 1e-3),
            "ms_per_step": ms / steps, "segments_per_step": seg / steps, "captures_per_step": capt / steps,
            "reemissions_per_step": reem / steps, "energy_closure_max_rel": worst}


def form_device_loop(steps: int = 20, launch: dict | None = None) -> dict:
    """The same crooked-pipe steps run eagerly (drop-in step: one host synchronisation per
    step) and as the device-resident loop (one captured two-step graph replayed, dt and Philox
    step read from device memory): full size and a 1/100 launch-bound size."""
    import torch

    from radtranbook_b200 import driver, imc2d, problems

    out = {}
    for tag, scale, nr, nz in (("full", 1.0, 60, 210), ("small", 0.01, 30, 105)):
        p = problems.crooked_pipe(scale=scale, nr=nr, nz=nz)

        def init():
            s = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"],
                                      p["eos_dev"], p["inv_eos_dev"], geometry="rz", seed=0xD1)
            if launch and tag == "full":  # the headline's tuned tracking shape, in both arms
                s._engine.launch.update(launch)
            return s

        st = init()
        st, _, _, _ = _gpu_steps(p, st, 3, True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st, seg_e, _, _ = _gpu_steps(p, st, steps, True)
        e1.record()
        torch.cuda.synchronize()
        ms_e = e0.elapsed_time(e1) / steps
        st2 = init()
        st2, _, _, _ = _gpu_steps(p, st2, 3, True)
        loop = driver.DeviceLoop(st2, Ntarget=p["Ntarget"], Nboundary=p["Nboundary"], Nsource=0, Nmax=p["Nmax"],
                                 T_boundary=p["T_boundary"], sigma_a_func=p["sigma_dev"], inv_eos=p["inv_eos_dev"],
                                 cv=p["cv_dev"], source=p["source"], reflect=p["reflect"], geometry="rz",
                                 max_events=1_000_000, boundary_source_func=p["boundary_source_func"])
        loop.run([p["dt"]] * steps)  # capture and a first run outside the timing
        res = loop.run([p["dt"]] * steps)
        ms_g = res["device_ms"] / steps
        seg_g = sum(s["transport_events"]["total"] for s in res["steps"])
        out[tag] = {"particles_per_step": p["Ntarget"] + p["Nboundary"], "eager_ms_per_step": ms_e,
                    "device_loop_ms_per_step": ms_g, "speedup": ms_e / ms_g,
                    "eager_segments_per_s": seg_e / (ms_e * steps * 1e-3),
                    "device_loop_segments_per_s": seg_g / (ms_g * steps * 1e-3),
                    "max_relative_closure": res["max_relative_closure"]}
    return out


def form_mg_crooked_pipe(steps: int = 12, warmup: int = 3) -> dict:
    """The multigroup crooked pipe (MG_IMC/problems/crooked_pipe_multigroup_imc.py, 10 groups,
    60 x 210 RZ, 'standard' preset: 200k emission + 200k surface-source particles per step,
    Nmax 1e6 growing by 5e4 per step) through the mg_imc2d drop-in step with device
    material laws, dt from 1e-4 ns growing by 1.1; CUDA-event timing of whole steps after
    `warmup` untimed steps, with each step's host wall time (a step takes under 1 ms, so a
    pause of the host, e.g. Python's cyclic garbage collector, shows as one long step; the
    collector runs once before the timed steps).  The same
    steps (same dt and Nmax sequence, from the same state) are also run as the device-resident
    loop (one replayed graph, radtranbook_b200.driver.DeviceLoop)."""
    import torch

    from radtranbook_b200 import driver, mg_imc2d, problems

    p = problems.mg_crooked_pipe(mode="standard")
    e1, e2, ge = p["edges1"], p["edges2"], p["energy_edges"]

    def init():
        return mg_imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], e1, e2, ge, p["eos_dev"],
                                        p["inv_eos_dev"], T_emit_floor=p["T_emit_floor"], geometry="rz", seed=0x36C9)

    st = init()
    state = {"dt": p["dt_initial"], "k": 0}

    def run(n, st):
        seg = hist = 0
        worst = 0.0
        for _ in range(n):
            Nmax = min(p["Nmax"] + state["k"] * p["Nmax_growth"], p["Nmax_final"])
            st, info = mg_imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, Nmax, p["T_boundary"], state["dt"], e1,
                                     e2, ge, p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"],
                                     reflect=p["reflect"], geometry="rz",
                                     boundary_source_func=p["boundary_source_func"], T_emit_floor=p["T_emit_floor"],
                                     Nmax_growth=p["Nmax_growth"], Nmax_final=p["Nmax_final"])
            te = info["profiling"]["transport_events"]
            seg += te["total"]
            hist += te["n_particles_transported"]
            track.append(info["profiling"]["phase_times_s"]["transport"] * 1e3)
            worst = max(worst, abs(info["ledger"]["relative_closure"]))
            used.append(state["dt"])
            state["dt"] = min(state["dt"] * p["dt_growth"], p["dt_max"])
            state["k"] += 1
            walls.append(time.perf_counter())
        return st, seg, hist, worst, info

    track, used, walls = [], [], []
    st = run(warmup, st)[0]  # no info of the warm-up kept (its arrays view the step's buffer)
    track.clear()
    del used[:]
    del walls[:]
    e0 = torch.cuda.Event(enable_timing=True)
    e1_ = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    gc.collect()
    e0.record()
    t_start = time.perf_counter()
    st, seg, hist, worst, info = run(steps, st)
    e1_.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1_)
    step_wall_ms = list(np.diff([t_start] + walls) * 1e3)
    track_ms = float(np.mean(track))  # before the device loop's warm-up steps append to it
    peak, _ = measured_peaks()
    dts = list(used)
    # the same steps as the device-resident loop
    st2 = init()
    state.update(dt=p["dt_initial"], k=0)
    st2 = run(warmup, st2)[0]
    loop = driver.DeviceLoop(st2, Ntarget=p["Ntarget"], Nboundary=p["Nboundary"], Nsource=0,
                             Nmax=p["Nmax"] + warmup * p["Nmax_growth"], T_boundary=p["T_boundary"],
                             sigma_a_func=p["sigma_dev"], inv_eos=p["inv_eos_dev"], cv=p["cv_dev"],
                             reflect=p["reflect"], geometry="rz", max_events=1_000_000,
                             boundary_source_func=p["boundary_source_func"], T_emit_floor=p["T_emit_floor"],
                             Nmax_growth=p["Nmax_growth"], Nmax_final=p["Nmax_final"])
    res = loop.run(dts)
    seg_g = sum(s["transport_events"]["total"] for s in res["steps"])
    loop_ms = res["device_ms"] / steps
    return {"workload": "mg_crooked_pipe_rz_60x210_10g_standard", "steps": steps, "warmup": warmup,
            "segments_per_s": seg / (ms * 1e-3), "histories_per_s": hist / (ms * 1e-3), "ms_per_step": ms / steps,
            "segments_per_step": seg / steps, "census_after": int(info["N_particles"]), "time_ns": float(st.time),
            "transport_ms_per_step": track_ms, "step_wall_ms": [round(x, 4) for x in step_wall_ms],
            "step_wall_ms_median": float(np.median(step_wall_ms)),
            "step_transport_ms": [round(x, 4) for x in track[:steps]],
            "step_roofline_frac": B_SEG_2D_MG * seg / (ms * 1e-3) / 1e9 / peak,
            "bytes_per_segment_algorithmic": B_SEG_2D_MG, "energy_closure_max_rel": worst,
            "device_loop": {"ms_per_step": loop_ms, "speedup_over_eager": (ms / steps) / loop_ms,
                            "segments_per_s": seg_g / (loop_ms * steps * 1e-3),
                            "same_census_as_eager": int(res["steps"][-1]["N_particles"]) == int(info["N_particles"]),
                            "max_relative_closure": res["max_relative_closure"]}}


def form_other_configs(steps: int = 20, warmup: int = 5, tune: bool = True) -> dict:
    """The other two single-problem workloads at full size through the drop-in steps with device
    callables (CUDA-event timing of whole steps): the slab Marshak wave (20k + 20k particles
    per step, 100 cells) and the multigroup Marshak wave (1e6 particles per step, 200 cells x
    10 groups, problems.marshak_mg)."""
    import torch

    from radtranbook_b200 import imc1d, mg_imc2d, problems

    out = {}
    p = problems.marshak_slab()
    st = imc1d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["mesh"], p["eos_dev"], p["inv_eos_dev"],
                               seed=0xC0F1)

    track = []  # tracking kernel time per step (ms, CUDA events in the library)

    def slab(st, n):
        seg = 0
        for _ in range(n):
            st, info = imc1d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"],
                                  p["mesh"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"])
            seg += info["profiling"]["transport_events"]["total"]
            track.append(info["profiling"]["phase_times_s"]["transport"] * 1e3)
        return st, seg

    q = problems.marshak_mg()
    sm = mg_imc2d.init_simulation(q["Ntarget"], q["Tinit"], q["Tr_init"], q["edges1"], q["edges2"],
                                  q["energy_edges"], q["eos_dev"], q["inv_eos_dev"], geometry="xy", seed=0xC0F3)

    def mg(sm, n):
        seg = 0
        for _ in range(n):
            sm, info = mg_imc2d.step(sm, q["Ntarget"], q["Nboundary"], 0, q["Nmax"], q["T_boundary"], q["dt"],
                                     q["edges1"], q["edges2"], q["energy_edges"], q["sigma_dev"], q["inv_eos_dev"],
                                     q["cv_dev"], q["source"], reflect=q["reflect"], geometry="xy")
            seg += info["profiling"]["transport_events"]["total"]
            track.append(info["profiling"]["phase_times_s"]["transport"] * 1e3)
        return sm, seg

    peak, peak_kind = measured_peaks()
    for tag, fn, s0, bseg, kern, mod in (("slab_marshak_100_cells", slab, st, B_SEG_1D, "k_track<slab>", imc1d),
                                         ("mg_marshak_200x10", mg, sm, B_SEG_2D_MG, "k_track<XY, multigroup>",
                                          mg_imc2d)):
        s0, _ = fn(s0, warmup)
        tuned = mod.tune(s0) if tune else None  # the launch shape for this problem (autotuner)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        track.clear()
        e0.record()
        s0, seg = fn(s0, steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        t_launch = float(np.mean(track)) * 1e-3
        achieved = bseg * (seg / steps) / t_launch / 1e9
        out[tag] = {"steps": steps, "after_warmup_steps": warmup, "ms_per_step": ms / steps,
                    "segments_per_step": seg / steps, "segments_per_s": seg / (ms * 1e-3),
                    "track_ms_per_launch": t_launch * 1e3,
                    "launch": dict(s0._engine.launch),
                    "autotune": None if tuned is None else {"best_ms": tuned["best_ms"], "worst_ms": tuned["worst_ms"],
                                                            "candidates": len(tuned["trials"])},
                    "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                 "frac": achieved / peak, "kernel": kern, "peak_source": peak_kind,
                                 "bytes_per_segment_algorithmic": bseg}}
    return out


def form_slab_event_cap(steps: int = 15) -> dict:
    """How the slab tracking kernel's time depends on its longest histories: after `steps`
    drop-in steps of the slab Marshak wave, the transport of the next step (the state's census,
    the law's opacity at the current temperature, the last step's sources) is replayed from the
    same census with an events-per-history cap K (the reference's max_events_per_particle);
    each replay reports the tracking time, the events and the histories the cap stopped (those
    longer than K events)."""
    import torch

    from radtranbook_b200 import imc1d, problems
    from radtranbook_b200._lib import STAT_CAP, STAT_EVENTS, ImcStepSummary
    from radtranbook_b200.autotune import _restore, _snapshot

    p = problems.marshak_slab()
    st = imc1d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["mesh"], p["eos_dev"], p["inv_eos_dev"],
                               seed=0xC0F1)
    for _ in range(steps):
        st, _ = imc1d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], p["mesh"],
                           p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"])
    eng = st._engine
    args, kw = eng._last_transport
    _, sig, cvv = st.__dict__["_law_next"]
    args = (st._T, sig, cvv) + tuple(args[3:])
    snap = _snapshot(eng.bank)
    rows = []
    for K in (0, 500, 400, 300, 200, 100):
        best = float("inf")
        for _ in range(3):
            _restore(eng.bank, snap)
            eng._census_dev_valid = False
            eng.transport_async(*args, **dict(kw, max_events=K))
            torch.cuda.synchronize()
            best = min(best, eng.phase_times()[1])
        sm = ImcStepSummary.from_buffer_copy(eng.summary_dev.cpu().numpy().tobytes())
        rows.append({"cap": K, "track_ms": best, "events": int(sm.stats[STAT_EVENTS]),
                     "histories_capped": int(sm.stats[STAT_CAP])})
    _restore(eng.bank, snap)
    eng._census_dev_valid = False
    return {"workload": "slab_marshak_100_cells, transport of step %d replayed" % (steps + 1),
            "census_entries": int(snap["_n"]), "launch": dict(eng.launch), "caps": rows}


def form_mg_crooked_pipe_run(output_times=(1.0, 5.0, 10.0)) -> dict:
    """The multigroup crooked pipe driven by driver.mg_crooked_pipe_run to the last output time
    ('standard' preset, adaptive dt from 1e-4 ns by 1.1 to 0.01 ns, Nmax growing to 5e6):
    device time, steps, census, worst closure and the fiducial temperatures at each output."""
    from radtranbook_b200 import driver, mg_imc2d, problems

    p = problems.mg_crooked_pipe(mode="standard")
    st = mg_imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"],
                                  p["energy_edges"], p["eos_dev"], p["inv_eos_dev"], T_emit_floor=p["T_emit_floor"],
                                  geometry="rz", seed=0x36CA)
    times, fid, fid_rad, snaps, res = driver.mg_crooked_pipe_run(st, p, list(output_times))
    idx = {t: int(np.argmin(np.abs(np.array(times) - t))) for t in output_times}
    seg = sum(s["transport_events"]["total"] for s in res["steps"])
    return {"workload": "mg_crooked_pipe_rz_60x210_10g_standard, device loop to %g ns" % max(output_times),
            "steps": len(res["steps"]), "device_s": res["device_ms"] * 1e-3,
            "segments_per_s": seg / (res["device_ms"] * 1e-3), "census_final": res["steps"][-1]["N_particles"],
            "max_relative_closure": res["max_relative_closure"],
            "fiducial_T": {lbl: {str(t): fid[lbl][i] for t, i in idx.items()} for lbl in fid},
            "fiducial_Tr": {lbl: {str(t): fid_rad[lbl][i] for t, i in idx.items()} for lbl in fid_rad}}


def max_time_and_totals(dist, ms: float, counts: list, device) -> tuple:
    """Whole-job figures of a timed region: the slowest rank's device time (ms) and the
    sum over ranks of each count (segments, histories)."""
    if dist is None:
        return float(ms), [float(c) for c in counts]
    import torch

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if not counts:
        return float(t.item()), []
    tot = torch.tensor([float(c) for c in counts], dtype=torch.float64, device=device)
    dist.all_reduce(tot)
    return float(t.item()), [float(x) for x in tot.cpu()]


def run_ours(args, rank: int, world: int):
    import torch

    from radtranbook_b200 import _lib, imc2d, problems

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    lib = _lib.load()
    dist = None
    if world > 1:
        import torch.distributed as td

        dist = td
    # weak scaling: N ranks partition N times the one-GPU particle counts
    p = problems.crooked_pipe(scale=args.scale * world)
    seed = 0x5EED0001

    def fresh():
        return imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                                     p["inv_eos_dev"], geometry="rz", seed=seed, _allreduce=dist)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---------------- device-resident value ----------------
    state = fresh()
    state, _, _, _ = _gpu_steps(p, state, args.warmup, True, dist)
    eng = state._engine
    tuned = None
    if args.launch:
        # a fixed launch shape (block, blocks per SM, chunk, smem cells[, prefetched refills]),
        # e.g. the tuner's choice
        vals = [int(x) for x in args.launch.split(",")]
        b, bps, ch, sm = vals[:4]
        eng.launch.update(block_size=b, blocks_per_sm=bps, chunk=ch, smem_cells=sm,
                          prefetch=vals[4] if len(vals) > 4 else 0)
        launch_shape = dict(eng.launch)
        tuned = {"best_ms": None, "worst_ms": None, "trials": [], "fixed": args.launch}
    elif not args.no_tune:
        tuned = imc2d.tune(state)
        launch_shape = dict(eng.launch)
        if args.tune_log:
            with open(args.tune_log, "w") as f:
                json.dump(tuned, f, indent=1)
    barrier()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    launches0 = lib.imc_kernel_launches()
    CLOSURE[0] = 0.0
    track_ms = []
    segs_per_step = []
    clocks = ClockSampler(dev.index)
    with clocks:
        clocks.mark_start()
        s0.record()
        seg = hist = 0
        for _ in range(args.steps):
            state, sg, hs, info = _gpu_steps(p, state, 1, True, dist)
            seg += sg
            hist += hs
            track_ms.append(info["profiling"]["phase_times_s"]["transport"] * 1e3)
            segs_per_step.append(sg)
        s1.record()
        barrier()
        clocks.mark_end()
    launches = lib.imc_kernel_launches() - launches0
    # the slowest rank's time; the partitioned step's info counts are already summed over the ranks
    tmax, _ = max_time_and_totals(dist, s0.elapsed_time(s1), [], dev)
    seg_all, hist_all = float(seg), float(hist)
    value = seg_all / (tmax * 1e-3)

    # ---------------- end to end through the drop-in API with host callables ----------------
    state2 = fresh()
    if tuned is not None:
        state2._engine.launch.update(launch_shape)
    state2, _, _, _ = _gpu_steps(p, state2, args.warmup, False, dist)
    barrier()
    tr0 = dict(_lib.TRANSFER)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    state2, seg2, hist2, _ = _gpu_steps(p, state2, args.steps, False, dist)
    e1.record()
    barrier()
    ms2, _ = max_time_and_totals(dist, e0.elapsed_time(e1), [], dev)
    h2d = (_lib.TRANSFER["h2d"] - tr0["h2d"]) / args.steps
    d2h = (_lib.TRANSFER["d2h"] - tr0["d2h"]) / args.steps
    e2e = seg2 / (ms2 * 1e-3)

    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    # dominant kernel: tracking.  per-launch average over the timed steps
    seg_per_launch = float(np.mean(segs_per_step))
    t_launch = float(np.mean(track_ms)) * 1e-3
    achieved = B_SEG_2D * seg_per_launch / t_launch / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": DRAM_B_PER_SEG_MEASURED * seg_per_launch, "kernel": "k_track<RZ>", "peak_source": peak_kind,
            "traffic_source": "ncu dram bytes of one full-size k_track launch (%.2f B/segment), scaled to the "
                              "segments per launch of this run" % DRAM_B_PER_SEG_MEASURED,
            "segments_per_launch": seg_per_launch, "bytes_per_segment_algorithmic": B_SEG_2D,
            "track_ms_per_launch": t_launch * 1e3}
    # the bound the kernel actually meets: warp-instruction issue (4 schedulers per SM, one
    # instruction per cycle each, at the SM clock sampled during the timed region)
    csum = clocks.summary() or {}
    mhz, clock_src = csum.get("sm_mhz"), "SM clock sampled in the timed region"
    if not mhz:  # a timed region shorter than the sampling interval: the pool's maximum SM clock
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                mhz, clock_src = float(json.load(f)["sm_max_mhz"]), "sm_max_mhz of MEASURED_PEAKS.json (no sample in the timed region)"
        except (OSError, KeyError, ValueError):
            mhz = None
    if mhz:
        ach = WARP_INST_PER_SEG_MEASURED * seg_per_launch / t_launch / 1e9
        pk = ISSUE_SLOTS_PER_CYCLE * mhz * 1e6 / 1e9
        roof["issue"] = {"bound": "issue", "achieved": ach, "peak": pk, "unit": "G warp-instructions/s", "frac": ach / pk,
                         "warp_instructions_per_segment": WARP_INST_PER_SEG_MEASURED,
                         "source": "ncu smsp__inst_executed.sum of one full-size k_track launch over its segments; "
                                   "peak = 148 SMs x 4 schedulers x the SM clock", "clock_mhz": mhz,
                         "clock_source": clock_src}
    cpu = None
    if not args.no_cpu_baseline:
        v, h, dtc, _ = cpu_oracle_run(args.cpu_scale, args.cpu_steps, 1, os.cpu_count() or 1)
        cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"crooked pipe, {args.cpu_scale:g} x particles, 1 warm-up + {args.cpu_steps} timed steps, "
                         f"FP64 C++ oracle, OpenMP ({dtc:.1f} s)", "histories_per_s": h}
    forms = fom = None
    if world == 1 and not args.no_forms:
        forms = {"batched": form_batched(args.batch_steps, not args.no_tune, form=args.batch_form),
                 "batched_small": form_batched(10, not args.no_tune, n_inst=512, particle_scale=0.01,
                                               form=args.batch_form),
                 "adjoint": form_adjoint(),
                 "carter_forest": form_carter_forest(), "device_loop": form_device_loop(launch=dict(eng.launch)),
                 "mg_crooked_pipe": form_mg_crooked_pipe(), "other_configs": form_other_configs(),
                 "event_based": form_event_based(launch=dict(eng.launch))}
        forms["carter_forest"]["over_fleck_cummings"] = forms["carter_forest"]["segments_per_s"] / value
    if world == 1 and not args.no_fom:
        fom = {"gpu": fom_gpu(p, args.fom_steps, args.fom_seeds, dict(eng.launch))}
        if not args.no_cpu_baseline:
            fom["cpu"] = fom_cpu(args.fom_cpu_scale, args.fom_steps, args.fom_cpu_seeds, os.cpu_count() or 1)
            fom["gpu_over_cpu"] = fom["gpu"]["fom"] / fom["cpu"]["fom"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tmax / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "crooked_pipe_rz_60x210", "source_particles_per_step": p["Ntarget"] + p["Nboundary"],
                   "nmax": p["Nmax"], "scale": args.scale, "precision": "f32 tracking, f64 tallies/ledger",
                   "l2": "bank of ~8.7e6 particles x 32 B > 126 MB L2 (inputs larger than L2)",
                   "parallelism": f"particles partitioned over {world} ranks" if world > 1 else "single",
                   "launch": dict(eng.launch),
                   "autotune": None if tuned is None else {"best_ms": tuned["best_ms"], "worst_ms": tuned["worst_ms"],
                                                           "candidates": len(tuned["trials"])}},
        "histories_per_s": hist_all / (tmax * 1e-3),
        # histories against HBM / (2 x 36-byte record + 28-byte source fill) per history
        "histories_roofline_frac": hist_all / (tmax * 1e-3) * (2 * 36 + 28) / (peak * 1e9),
        "segments_per_step": seg_all / args.steps,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "energy_closure_max_rel": CLOSURE[0],
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "fom": fom,
        "forms": forms,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="particle-count scale of the workload")
    ap.add_argument("--cpu-scale", type=float, default=1.0,
                    help="particle-count scale of the CPU runs (cpu_baseline and the reference arm)")
    ap.add_argument("--cpu-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--launch", default=None,
                    help="fixed tracking launch shape 'block,blocks_per_sm,chunk,smem_cells[,prefetch]' instead of tuning")
    ap.add_argument("--tune-log", default=None, help="write the autotuner's trials to this JSON file")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and adjoint forms")
    ap.add_argument("--only-form", default=None,
                    choices=["batched", "adjoint", "carter_forest", "device_loop", "mg_crooked_pipe",
                             "mg_crooked_pipe_run", "other_configs", "event_based", "slab_event_cap",
                             "batched_small"],
                    help="run one further form alone on GPU 0 and print its JSON (no headline line)")
    ap.add_argument("--batch-steps", type=int, default=50, help="steps of the batched form (the workload's 50)")
    ap.add_argument("--batch-instances", type=int, default=256,
                    help="instances of the batched form (the workload's 256; fewer for a small profiling case)")
    ap.add_argument("--batch-form", type=int, default=0, choices=(0, 1, 2, 3),
                    help="batched tracking form: 0 the tuner's choice, 1 work units, 2 the entry queue, 3 work units with prefetched refills")
    ap.add_argument("--no-fom", action="store_true")
    ap.add_argument("--fom-seeds", type=int, default=32)
    ap.add_argument("--fom-steps", type=int, default=100)
    ap.add_argument("--fom-cpu-seeds", type=int, default=8)
    ap.add_argument("--fom-cpu-scale", type=float, default=0.01)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.only_form:
        import torch

        torch.cuda.set_device(0)
        fn = {"batched": lambda: form_batched(args.batch_steps, not args.no_tune, n_inst=args.batch_instances,
                                             form=args.batch_form),
              "adjoint": form_adjoint,
              "batched_small": lambda: form_batched(10, not args.no_tune, n_inst=512, particle_scale=0.01,
                                                    form=args.batch_form),
              "carter_forest": form_carter_forest, "device_loop": form_device_loop,
              "mg_crooked_pipe": form_mg_crooked_pipe, "mg_crooked_pipe_run": form_mg_crooked_pipe_run,
              "other_configs": lambda: form_other_configs(tune=not args.no_tune),
              "event_based": form_event_based, "slab_event_cap": form_slab_event_cap}[args.only_form]
        print(json.dumps({"form": args.only_form, **fn()}), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        try:
            run_ours(args, rank, world)
        finally:
            td.destroy_process_group()
    else:
        run_ours(args, rank, world)


if __name__ == "__main__":
    main()
