"""The multigroup crooked pipe (MG_IMC/problems/crooked_pipe_multigroup_imc.py) on the GPU.

Tolerances:
  - one transport step on the problem's own geometry, opacities and surface source (a
    coarser 30 x 105 mesh, 10 groups, the reference's first dt) from an identical bank,
    against the FP64 oracle: boundary energy to FP32 weight rounding, emitted energy per
    cell to FP32 weight rounding, per-(group, cell) deposition and scalar intensity
    relative L1 <= 5e-4, event count relative 2e-3;
  - the drop-in MG step on the full 60 x 210 mesh with the 'quick' particle preset: FP64
    energy closure <= 1e-12 per step, the census within the comb cap, and heat arriving
    only through the source end of the pipe.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200 import mg_imc2d, problems
from radtranbook_b200.engine import Engine

pytestmark = pytest.mark.gpu

SEED = 0x5EED0C9


def test_mg_crooked_pipe_transport_matches_oracle(cuda):
    p = problems.mg_crooked_pipe(nr=30, nz=105)
    e1, e2, ge = p["edges1"], p["edges2"], p["energy_edges"]
    nx, ny, G = len(e1) - 1, len(e2) - 1, len(ge) - 1
    v = np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :]
    eng = Engine("rz", e1, e2, O.flat2d(v), seed=SEED, n_groups=G, group_edges=ge)
    orc = O.Oracle("rz", e1, e2, O.flat2d(v), SEED, n_groups=G)
    rc = 0.5 * (e1[:-1] + e1[1:])
    zc = 0.5 * (e2[:-1] + e2[1:])
    # a heated plug in the pipe near the source, so material emission above the floor is exercised
    T2 = np.full((nx, ny), 0.05)
    T2[np.ix_(rc < 0.5, zc < 1.0)] = 0.3
    T = O.flat2d(T2)
    tr = O.flat2d(np.full((nx, ny), 0.05))
    assert eng.init_census(torch.as_tensor(tr, device=cuda), 3000) == orc.init_ic_mg(tr, 3000, ge)
    b = eng.bank
    orc.set_bank(*(b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")),
                 b.view("cell").cpu().numpy(), b.view("group").cpu().numpy())
    sig = np.stack([O.flat2d(f(T2)) for f in p["sigma_host"]]).reshape(-1)
    cv = O.flat2d(p["cv_host"](T2))
    face_z = np.where(rc < 0.5, 0.5, 0.0)
    face = [None, None, face_z, None]
    dt = p["dt_initial"]
    dev = lambda a: None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=cuda)  # noqa: E731
    res = eng.transport(dev(T), dev(sig), dev(cv), None, 1, dt, 1.0, 3000, 3000, 0, [dev(f) for f in face],
                        p["reflect"], max_events=1_000_000, t_emit_floor=p["T_emit_floor"])
    ro = orc.transport_mg(T, sig, cv, None, 1, dt, 1.0, 3000, 3000, 0, face, p["reflect"], ge,
                          max_events=1_000_000, t_emit_floor=p["T_emit_floor"])
    rep = res.report
    assert rep.n_transported == ro["n_transported"]
    np.testing.assert_allclose(rep.boundary_emission, ro["boundary_emission"], rtol=1e-7)
    emitted = eng.emitted.cpu().numpy()
    np.testing.assert_allclose(emitted, ro["emitted"], rtol=1e-7, atol=1e-300)
    assert emitted.sum() > 0 and emitted[T <= p["T_emit_floor"]].sum() == 0.0
    l1 = lambda a, b: np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)  # noqa: E731
    dep, si = eng.dep.cpu().numpy(), eng.si.cpu().numpy()
    assert l1(dep, ro["dep"]) < 5e-4, l1(dep, ro["dep"])
    assert l1(si, ro["si"]) < 5e-4, l1(si, ro["si"])
    stats, esc = eng.host_stats()
    np.testing.assert_allclose(stats[0], ro["stats"][0], rtol=2e-3)


def test_mg_crooked_pipe_dropin_steps_close(cuda):
    p = problems.mg_crooked_pipe(mode="quick")
    e1, e2, ge = p["edges1"], p["edges2"], p["energy_edges"]
    st = mg_imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], e1, e2, ge, p["eos_dev"],
                                  p["inv_eos_dev"], T_emit_floor=p["T_emit_floor"], geometry="rz", seed=SEED)
    dt = p["dt_initial"]
    for k in range(4):
        Nmax = min(p["Nmax"] + k * p["Nmax_growth"], p["Nmax_final"])
        st, info = mg_imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, Nmax, p["T_boundary"], dt, e1, e2, ge,
                                 p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"], reflect=p["reflect"],
                                 geometry="rz", boundary_source_func=p["boundary_source_func"],
                                 T_emit_floor=p["T_emit_floor"])
        assert abs(info["ledger"]["relative_closure"]) < 1e-12, info["ledger"]
        assert info["N_particles"] <= Nmax + 2 * 60 * 210 * 10
        assert info["boundary_emission"] > 0
        dt = min(dt * p["dt_growth"], p["dt_max"])
    T = st.temperature
    assert np.isfinite(T).all() and T.min() >= 0.05 * (1 - 1e-9)
    # heat enters only at the source end: the far end of the pipe has not moved after 4 short steps
    assert T[:8, :10].max() > 0.05 and np.allclose(T[:, 150:], 0.05, rtol=1e-9)
    erg = st.radiation_energy_by_group
    assert erg.shape == (10, 60, 210) and np.isfinite(erg).all()
