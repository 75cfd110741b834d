"""The bounds-checked build (libimcb200_checked.so, selected by IMCB200_CHECKED=1): the same
steps run through it and through the normal library give the same results, and no check
fires on valid inputs (a firing check raises IMC_ERR_BOUNDS).

Each library is loaded in its own Python process (the loader binds one library per process).
Tolerance: particle counts and event counts exact, temperatures to 1e-12 relative (only the
order of a few FP64 atomic sums can differ between runs).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, ROOT)
from radtranbook_b200 import _lib, imc1d, imc2d, mg_imc2d, problems
out = {"lib": _lib.LIB_PATH.name}
p = problems.crooked_pipe(scale=0.01, nr=30, nz=105)
st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                           p["inv_eos_dev"], geometry="rz", seed=41)
ev = []
for _ in range(3):
    st, info = imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], p["edges1"],
                          p["edges2"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"], reflect=p["reflect"],
                          geometry="rz", boundary_source_func=p["boundary_source_func"])
    ev.append(info["profiling"]["transport_events"]["total"])
out["rz"] = {"T": st.temperature.tolist(), "n": int(info["N_particles"]), "events": ev}
q = problems.mg_crooked_pipe(nr=30, nz=105, mode="quick")
sm = mg_imc2d.init_simulation(q["Ntarget"], q["Tinit"], q["Tr_init"], q["edges1"], q["edges2"], q["energy_edges"],
                              q["eos_dev"], q["inv_eos_dev"], T_emit_floor=q["T_emit_floor"], geometry="rz", seed=42)
for _ in range(2):
    sm, info = mg_imc2d.step(sm, q["Ntarget"], q["Nboundary"], 0, q["Nmax"], q["T_boundary"], q["dt_initial"],
                             q["edges1"], q["edges2"], q["energy_edges"], q["sigma_dev"], q["inv_eos_dev"], q["cv_dev"],
                             q["source"], reflect=q["reflect"], geometry="rz",
                             boundary_source_func=q["boundary_source_func"], T_emit_floor=q["T_emit_floor"])
out["mg"] = {"T": sm.temperature.tolist(), "n": int(info["N_particles"]),
             "events": info["profiling"]["transport_events"]["total"]}
mp = problems.marshak_slab()
s1 = imc1d.init_simulation(2000, mp["Tinit"], mp["Tr_init"], mp["mesh"], mp["eos_dev"], mp["inv_eos_dev"], seed=43)
for _ in range(3):
    s1, info = imc1d.step(s1, 2000, 2000, 0, 8000, mp["T_boundary"], mp["dt"], mp["mesh"], mp["sigma_dev"],
                          mp["inv_eos_dev"], mp["cv_dev"], mp["source"])
out["slab"] = {"T": s1.temperature.tolist(), "n": int(info["N_particles"]),
               "events": info["profiling"]["transport_events"]["total"]}
print(json.dumps(out))
""".replace("ROOT", repr(ROOT))


def _run(checked: bool) -> dict:
    env = dict(os.environ, IMCB200_CHECKED="1" if checked else "0")
    r = subprocess.run([sys.executable, "-c", SCRIPT], env=env, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_checked_build_matches_normal_build(cuda):
    if not os.path.exists(os.path.join(ROOT, "radtranbook_b200", "libimcb200_checked.so")):
        pytest.fail("libimcb200_checked.so is missing: run __graft_entry__.build()")
    plain, checked = _run(False), _run(True)
    assert plain["lib"] == "libimcb200.so" and checked["lib"] == "libimcb200_checked.so"
    for k in ("rz", "mg", "slab"):
        assert checked[k]["n"] == plain[k]["n"], k
        assert checked[k]["events"] == plain[k]["events"], k
        np.testing.assert_allclose(np.array(checked[k]["T"]), np.array(plain[k]["T"]), rtol=1e-12, atol=0)
