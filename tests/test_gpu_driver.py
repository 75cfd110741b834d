"""The device-resident time loop (radtranbook_b200.driver) against the eager drop-in step: the
same dt sequence replayed from one captured graph gives the same states.

Tolerance as the restart tests: temperatures and energy totals to 1e-12 relative, particle
counts exact (only the order of a few FP64 atomic sums differs between runs); the ledger
rebuilt from the recorded summaries closes to 1e-12 per step.
"""
import numpy as np
import pytest

from radtranbook_b200 import driver, imc1d, imc2d, imc2d_cf, problems

pytestmark = pytest.mark.gpu


def _eager(mod, p, st, dts, method_kw=None):
    out = []
    for dt in dts:
        st, info = mod.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], dt, p["edges1"],
                            p["edges2"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"],
                            reflect=p["reflect"], geometry="rz", boundary_source_func=p["boundary_source_func"],
                            **(method_kw or {}))
        out.append((info, st.temperature.copy(), st.radiation_temperature.copy()))
    return st, out


@pytest.mark.parametrize("mod,method", [(imc2d, "fc"), (imc2d_cf, "cf")])
@pytest.mark.parametrize("n_steps", [6, 7])
def test_device_loop_matches_eager_steps(cuda, mod, method, n_steps):
    p = problems.crooked_pipe(scale=0.01, nr=30, nz=105)
    sched, _ = driver.adaptive_schedule(0.0, [0.004, 0.01 * n_steps], 0.001, 0.01, 1.5)
    dts = [dt for dt, _ in sched][:n_steps]
    init = lambda: mod.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"],  # noqa: E731
                                       p["eos_dev"], p["inv_eos_dev"], geometry="rz", seed=99)
    a, eager = _eager(mod, p, init(), dts)
    b = init()
    cells = [(0, 2), (5, 40), (12, 60)]
    loop = driver.DeviceLoop(b, Ntarget=p["Ntarget"], Nboundary=p["Nboundary"], Nsource=0, Nmax=p["Nmax"],
                             T_boundary=p["T_boundary"], sigma_a_func=p["sigma_dev"], inv_eos=p["inv_eos_dev"],
                             cv=p["cv_dev"], source=p["source"], reflect=p["reflect"], geometry="rz",
                             max_events=1_000_000, boundary_source_func=p["boundary_source_func"], method=method,
                             fiducial_cells=cells)
    res = loop.run(dts, {2: "after-3"})
    assert res["max_relative_closure"] < 1e-12
    for k, (info, T, Tr) in enumerate(eager):
        s = res["steps"][k]
        assert s["N_particles"] == info["N_particles"]
        np.testing.assert_allclose(s["total_energy"], info["total_energy"], rtol=1e-12)
        np.testing.assert_allclose(res["fiducial_T"][k], [T[i, j] for i, j in cells], rtol=1e-12)
    np.testing.assert_allclose(b.temperature, a.temperature, rtol=1e-12, atol=0)
    np.testing.assert_allclose(b.internal_energy, a.internal_energy, rtol=1e-12, atol=0)
    np.testing.assert_allclose(res["snapshots"]["after-3"][0], eager[2][1], rtol=1e-12)
    assert b.count == a.count and abs(b.time - a.time) < 1e-15
    # the state carries on with eager steps after the loop
    _, more_a = _eager(mod, p, a, [0.01])
    _, more_b = _eager(mod, p, b, [0.01])
    np.testing.assert_allclose(more_b[0][1], more_a[0][1], rtol=1e-12)


def test_crooked_pipe_driver_hits_output_times(cuda):
    p = problems.crooked_pipe(scale=0.01, nr=30, nz=105)
    st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                               p["inv_eos_dev"], geometry="rz", seed=5)
    times, fid, fid_rad, snaps, res = driver.crooked_pipe_run(st, p, [0.01, 0.05], dt_initial=0.002, dt_max=0.01,
                                                              growth=1.2)
    assert set(snaps) == {0.01, 0.05}
    assert any(abs(t - 0.01) < 1e-12 for t in times) and abs(times[-1] - 0.05) < 1e-12
    assert all(len(v) == len(times) for v in fid.values())
    assert res["max_relative_closure"] < 1e-12
    np.testing.assert_allclose(snaps[0.05][0], st.temperature, rtol=0)


def test_slab_device_loop(cuda):
    mp = problems.marshak_slab()
    st_a = imc1d.init_simulation(2000, mp["Tinit"], mp["Tr_init"], mp["mesh"], mp["eos_dev"], mp["inv_eos_dev"], seed=1)
    st_b = imc1d.init_simulation(2000, mp["Tinit"], mp["Tr_init"], mp["mesh"], mp["eos_dev"], mp["inv_eos_dev"], seed=1)
    for _ in range(5):
        st_a, info = imc1d.step(st_a, 2000, 2000, 0, 8000, mp["T_boundary"], mp["dt"], mp["mesh"], mp["sigma_dev"],
                                mp["inv_eos_dev"], mp["cv_dev"], mp["source"])
    loop = driver.DeviceLoop(st_b, Ntarget=2000, Nboundary=2000, Nsource=0, Nmax=8000, T_boundary=mp["T_boundary"],
                             sigma_a_func=mp["sigma_dev"], inv_eos=mp["inv_eos_dev"], cv=mp["cv_dev"],
                             source=mp["source"], reflect=(False, False), geometry="slab", fiducial_cells=[0, 3])
    loop.run([mp["dt"]] * 5)
    np.testing.assert_allclose(st_b.temperature, st_a.temperature, rtol=1e-12, atol=0)
    # a second run reuses the captured graphs (odd counts start from the other bank)
    for _ in range(3):
        st_a, info = imc1d.step(st_a, 2000, 2000, 0, 8000, mp["T_boundary"], mp["dt"], mp["mesh"], mp["sigma_dev"],
                                mp["inv_eos_dev"], mp["cv_dev"], mp["source"])
    res = loop.run([mp["dt"]] * 3)
    np.testing.assert_allclose(st_b.temperature, st_a.temperature, rtol=1e-12, atol=0)
    assert res["steps"][-1]["N_particles"] == info["N_particles"] and res["device_ms"] > 0


def test_mg_device_loop_matches_eager_steps(cuda):
    """Multigroup crooked pipe (coarse mesh, 'quick' counts): the replayed graph with the
    growing Nmax and per-group comb against eager mg_imc2d steps."""
    from radtranbook_b200 import mg_imc2d

    p = problems.mg_crooked_pipe(nr=30, nz=105, mode="quick")
    e1, e2, ge = p["edges1"], p["edges2"], p["energy_edges"]
    sched, _ = driver.adaptive_schedule(0.0, [4e-4, 1e-3], p["dt_initial"], p["dt_max"], 1.5)
    dts = [dt for dt, _ in sched][:7]
    assert len(dts) >= 6

    def init():
        return mg_imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], e1, e2, ge, p["eos_dev"],
                                        p["inv_eos_dev"], T_emit_floor=p["T_emit_floor"], geometry="rz", seed=31)

    a = init()
    eager = []
    for k, dt in enumerate(dts):
        Nmax = min(p["Nmax"] + k * p["Nmax_growth"], p["Nmax_final"])
        a, info = mg_imc2d.step(a, p["Ntarget"], p["Nboundary"], 0, Nmax, p["T_boundary"], dt, e1, e2, ge,
                                p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"], reflect=p["reflect"],
                                geometry="rz", boundary_source_func=p["boundary_source_func"],
                                T_emit_floor=p["T_emit_floor"])
        eager.append((info, a.temperature.copy()))
    b = init()
    cells = [(0, 2), (3, 10), (12, 40)]
    loop = driver.DeviceLoop(b, Ntarget=p["Ntarget"], Nboundary=p["Nboundary"], Nsource=0, Nmax=p["Nmax"],
                             T_boundary=p["T_boundary"], sigma_a_func=p["sigma_dev"], inv_eos=p["inv_eos_dev"],
                             cv=p["cv_dev"], reflect=p["reflect"], geometry="rz", max_events=1_000_000,
                             boundary_source_func=p["boundary_source_func"], T_emit_floor=p["T_emit_floor"],
                             fiducial_cells=cells, Nmax_growth=p["Nmax_growth"], Nmax_final=p["Nmax_final"])
    res = loop.run(dts[:4], {1: "after-2"})
    res2 = loop.run(dts[4:])  # the Nmax schedule continues across calls
    assert res["max_relative_closure"] < 1e-12 and res2["max_relative_closure"] < 1e-12
    steps = res["steps"] + res2["steps"]
    fid_Eg = np.concatenate([res["fiducial_Erad_by_group"], res2["fiducial_Erad_by_group"]])
    for k, (info, T) in enumerate(eager):
        assert steps[k]["N_particles"] == info["N_particles"], k
        np.testing.assert_allclose(steps[k]["total_energy"], info["total_energy"], rtol=1e-12)
        Eg = info["radiation_energy_by_group"]
        np.testing.assert_allclose(fid_Eg[k], np.stack([Eg[:, i, j] for i, j in cells], axis=1), rtol=1e-12,
                                   atol=1e-300)
    np.testing.assert_allclose(b.temperature, a.temperature, rtol=1e-12, atol=0)
    np.testing.assert_allclose(b.radiation_energy_by_group, a.radiation_energy_by_group, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(res["snapshots_Erad_by_group"]["after-2"], eager[1][0]["radiation_energy_by_group"],
                               rtol=1e-12, atol=1e-300)
    assert res2["Nmax_next"] == min(p["Nmax"] + len(dts) * p["Nmax_growth"], p["Nmax_final"])
    assert b.count == a.count


def test_mg_crooked_pipe_driver_hits_output_times(cuda):
    from radtranbook_b200 import mg_imc2d

    p = problems.mg_crooked_pipe(nr=30, nz=105, mode="quick")
    st = mg_imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"],
                                  p["energy_edges"], p["eos_dev"], p["inv_eos_dev"], T_emit_floor=p["T_emit_floor"],
                                  geometry="rz", seed=8)
    times, fid, fid_rad, snaps, res = driver.mg_crooked_pipe_run(st, p, [5e-4, 2e-3])
    assert set(snaps) == {5e-4, 2e-3}
    assert any(abs(t - 5e-4) < 1e-12 for t in times) and abs(times[-1] - 2e-3) < 1e-12
    assert all(len(v) == len(times) for v in fid.values()) and len(fid) == 5
    assert res["max_relative_closure"] < 1e-12
    T, Tr, Eg = snaps[2e-3]
    np.testing.assert_allclose(T, st.temperature, rtol=0)
    assert Eg.shape == (10, 30, 105) and (Eg >= 0).all() and Eg[:, :3, :3].sum() > 0
