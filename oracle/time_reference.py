"""Time the reference's own Numba step (IMC/IMC2D.py:1591-1897) on this host's cores, beside
the FP64 C++ port of the oracle on the same cores and the same problem.

Test infrastructure (a CPU baseline record), not product code.  The reference is Python and
Numba and is not present where the GPU runs, so it is timed where its checkout is (the path
in RADTRANBOOK_REF), with matplotlib stubbed and a private NUMBA_CACHE_DIR; the port's own
numbers on the GPU host are in bench.py's cpu_baseline and reference arm.

Workload: the 60 x 210 RZ crooked pipe of radtranbook_b200.problems.crooked_pipe at `scale`
x its particle counts (2e6 source particles and Nmax 6.67e6 at scale 1), `steps` steps from
t = 0 per seed, after one untimed step of a separate run (Numba compilation).  Reported per
implementation: wall time per run, track segments/s (the reference's
info['profiling']['transport_events']['total']; the port's event count), histories/s, and the
FOM 1/(R^2 T) with R^2 the mean relative variance over seeds of the last step's per-cell
deposition in the cells above 1e-3 of the largest mean (the reference's deposition is
recovered from its material update: e_new - e_old + emitted / V).

  RADTRANBOOK_REF=<checkout> python oracle/time_reference.py --scale 0.01 --steps 100 --seeds 8
"""
from __future__ import annotations

import argparse
import contextlib
import io
import json
import os
import sys
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def load_reference_imc2d():
    ref = os.environ.get("RADTRANBOOK_REF", "")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("set RADTRANBOOK_REF to the reference checkout")
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/radtranbook_ref_nbcache")
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    sys.path.insert(0, os.path.join(ref, "IMC"))
    import IMC2D  # noqa: E402

    return IMC2D


def fom(xs, ts):
    xs = np.array(xs)
    m = xs.mean(0)
    roi = m > 1e-3 * m.max()
    r2 = float(np.mean(xs[:, roi].var(0, ddof=1) / m[roi] ** 2))
    t = float(np.mean(ts))
    return {"fom": 1.0 / (r2 * t), "rel_err": float(np.sqrt(r2)), "seconds_per_run": t, "roi_cells": int(roi.sum())}


def run_reference(IMC2D, p, steps, seeds):
    import random

    import numba

    @numba.njit
    def seed_nb(s):
        np.random.seed(s)
        random.seed(s)

    e1, e2 = p["edges1"], p["edges2"]
    vol = np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :]
    sig, cvg = p["sigma_host"](p["Tinit"]), p["cv_host"](p["Tinit"])
    a, c = 0.01372, 29.98

    def one_run(n_steps, s):
        np.random.seed(s); random.seed(s); seed_nb(s)
        st = IMC2D.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], e1, e2, p["eos_host"], p["inv_eos_host"],
                                   geometry="rz")
        seg = hist = 0
        dep = None
        t0 = time.perf_counter()
        for k in range(n_steps):
            T_old, e_old = st.temperature.copy(), st.internal_energy.copy()
            st, info = IMC2D.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], e1, e2,
                                  p["sigma_host"], p["inv_eos_host"], p["cv_host"], p["source"], reflect=p["reflect"],
                                  geometry="rz", boundary_source_func=p["boundary_source_func"])
            te = info["profiling"]["transport_events"]
            seg += int(te["total"])
            hist += int(te["n_particles_transported"])
            if k == n_steps - 1:
                beta = 4.0 * a * T_old ** 3 / cvg
                f = 1.0 / (1.0 + beta * sig * c * p["dt"])
                emitted = a * c * T_old ** 4 * f * sig * p["dt"] * vol
                dep = st.internal_energy - e_old + emitted / vol
        return time.perf_counter() - t0, seg, hist, dep

    with contextlib.redirect_stdout(io.StringIO()):
        one_run(1, 12345)  # Numba compilation
        runs = [one_run(steps, 1000 + s) for s in range(seeds)]
    ts = [r[0] for r in runs]
    out = fom([r[3].T.reshape(-1) for r in runs], ts)
    out.update(segments_per_s=sum(r[1] for r in runs) / sum(ts), histories_per_s=sum(r[2] for r in runs) / sum(ts),
               numba_threads=int(numba.get_num_threads()))
    return out


def run_port(p, steps, seeds, nthreads):
    from oracle import oracle as O

    e1, e2 = p["edges1"], p["edges2"]
    vol = O.flat2d(np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :])
    rc = 0.5 * (e1[:-1] + e1[1:])
    face = [None, None, np.where(rc < 0.5, 0.5, 0.0), None]
    kw = dict(Ntarget=p["Ntarget"], Nboundary=p["Nboundary"], Nsource=0, Nmax=p["Nmax"], face_T=face, dt=p["dt"],
              sigma_a_func=p["sigma_host"], inv_eos=p["inv_eos_host"], cv=p["cv_host"], reflect=p["reflect"],
              max_events=1_000_000)
    xs, ts, seg, hist = [], [], 0, 0
    for s in range(seeds):
        run = O.OracleGray("rz", e1, e2, vol, 0xC0E00000 + s, p["Ntarget"], p["Tinit"], p["Tr_init"], p["eos_host"],
                           p["inv_eos_host"], nthreads=nthreads)
        t0 = time.perf_counter()
        r = None
        for _ in range(steps):
            r = run.step(**kw)
            seg += int(r["stats"][0])
            hist += int(r["n_transported"])
        ts.append(time.perf_counter() - t0)
        xs.append(np.asarray(r["dep"], dtype=np.float64).copy())
    out = fom(xs, ts)
    out.update(segments_per_s=seg / sum(ts), histories_per_s=hist / sum(ts), threads=nthreads)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.01)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--seeds", type=int, default=8)
    args = ap.parse_args()
    from radtranbook_b200 import problems

    p = problems.crooked_pipe(scale=args.scale)
    IMC2D = load_reference_imc2d()
    cpu = os.cpu_count() or 1
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            model = next((ln.split(":", 1)[1].strip() for ln in f if ln.startswith("model name")), "")
    except OSError:
        pass
    res = {"workload": "crooked_pipe_rz_60x210", "scale": args.scale,
           "source_particles_per_step": p["Ntarget"] + p["Nboundary"], "nmax": p["Nmax"], "steps": args.steps,
           "seeds": args.seeds, "host": {"cpu": model, "logical_cores": cpu},
           "reference_numba": run_reference(IMC2D, p, args.steps, args.seeds),
           "port_cpp_openmp": run_port(p, args.steps, args.seeds, cpu)}
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
