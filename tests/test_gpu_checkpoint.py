"""Checkpoint / restart (radtranbook_b200.checkpoint): a run interrupted after k steps,
written to disk, restored into a fresh state (built with a different seed, which the
restore replaces) and continued, reproduces the uninterrupted run.

Tolerance: material temperature and energy totals to 1e-12 relative, particle counts and
time exact.  The step is deterministic (integer source counts, fixed-point deposition,
Philox streams keyed by (seed, step)); only the order of FP64 atomic sums in a few per-cell
reductions can differ between runs, at the last bit.
"""
import numpy as np
import pytest

from radtranbook_b200 import checkpoint, imc1d, imc2d, mg_imc1d, problems

pytestmark = pytest.mark.gpu


def _crooked(seed):
    p = problems.crooked_pipe(scale=0.01, nr=30, nz=105)
    st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                               p["inv_eos_dev"], geometry="rz", seed=seed)
    return p, st


def _crooked_steps(p, st, n):
    info = None
    for _ in range(n):
        st, info = imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], p["edges1"],
                              p["edges2"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"],
                              reflect=p["reflect"], geometry="rz", boundary_source_func=p["boundary_source_func"])
    return st, info


def _same(a, b, ia, ib):
    np.testing.assert_allclose(b.temperature, a.temperature, rtol=1e-12, atol=0)
    np.testing.assert_allclose(b.internal_energy, a.internal_energy, rtol=1e-12, atol=0)
    assert ib["N_particles"] == ia["N_particles"]
    assert b.time == a.time and b.count == a.count
    np.testing.assert_allclose(ib["total_energy"], ia["total_energy"], rtol=1e-12)
    assert abs(ib["ledger"]["relative_closure"]) < 1e-12


@pytest.mark.parametrize("fmt", ["npz", "pickle"])
def test_crooked_pipe_restart_reproduces_the_uninterrupted_run(cuda, tmp_path, fmt):
    p, a = _crooked(77)
    a, ia = _crooked_steps(p, a, 4)
    p, b = _crooked(77)
    b, _ = _crooked_steps(p, b, 2)
    path = str(tmp_path / ("ck.npz" if fmt == "npz" else "ck.pkl"))
    fid = {"r=0,z=0.25": [0.05, 0.06]}
    if fmt == "npz":
        checkpoint.save_checkpoint_npz(b, 2, [0.0, 0.01, 0.02], fid, fid, {0.02}, p["dt"], path)
    else:
        checkpoint.save_checkpoint(path, b, 2, 0.0, [], {"nr": 30})
    census = len(b.weights)
    p, c = _crooked(12345)  # another seed: the restore brings back the checkpoint's
    if fmt == "npz":
        step_count, times, fd, fdr, saved, cur_dt, meta = checkpoint.load_checkpoint_npz(path, c, None)
        assert step_count == 2 and times == [0.0, 0.01, 0.02] and fd == fid and saved == {0.02}
        assert cur_dt == p["dt"] and meta["method"] == "fc"
    else:
        payload = checkpoint.load_checkpoint(path)
        assert payload["philox"] == {"seed": 77, "step": 2}
        checkpoint.restore_state(c, payload["state"])
    assert len(c.weights) == census
    c, ic = _crooked_steps(p, c, 2)
    _same(a, c, ia, ic)


def test_npz_keys_follow_the_reference_driver(cuda, tmp_path):
    """Every key of IMC/CrookedPipe2D.py:480-505, with the census present."""
    p, b = _crooked(5)
    b, _ = _crooked_steps(p, b, 1)
    path = str(tmp_path / "ck.npz")
    checkpoint.save_checkpoint_npz(b, 1, [0.0, 0.01], {}, {}, set(), p["dt"], path)
    ck = np.load(path, allow_pickle=True)
    ref_keys = {"chkpt_temperature", "chkpt_radiation_temperature", "chkpt_internal_energy", "chkpt_weights",
                "chkpt_mu", "chkpt_eta", "chkpt_particle_times", "chkpt_r", "chkpt_z", "chkpt_time",
                "chkpt_current_dt", "chkpt_step_count", "chkpt_times", "chkpt_output_saved", "chkpt_fiducial_labels",
                "chkpt_fiducial_temps", "chkpt_fiducial_temps_rad", "chkpt_method", "chkpt_fastpath_threshold",
                "chkpt_no_progress_rel_tol", "chkpt_no_progress_max_streak", "chkpt_profile_phase_totals_s",
                "chkpt_profile_event_totals", "chkpt_profile_transported_particles_total", "chkpt_profile_step_count"}
    assert ref_keys <= set(ck.files)
    assert len(ck["chkpt_weights"]) == len(b.weights) > 0
    assert ck["chkpt_temperature"].shape == (30, 105)
    np.testing.assert_array_equal(ck["chkpt_r"], b.pos1)


def test_slab_and_mg_sphere_restart(cuda, tmp_path):
    mp = problems.marshak_slab()
    mesh = mp["mesh"]

    def slab(seed):
        return imc1d.init_simulation(2000, mp["Tinit"], mp["Tr_init"], mesh, mp["eos_dev"], mp["inv_eos_dev"],
                                     seed=seed)

    def slab_steps(st, n):
        info = None
        for _ in range(n):
            st, info = imc1d.step(st, 2000, 2000, 0, 8000, mp["T_boundary"], mp["dt"], mesh, mp["sigma_dev"],
                                  mp["inv_eos_dev"], mp["cv_dev"], mp["source"])
        return st, info

    a, ia = slab_steps(slab(3), 4)
    b, _ = slab_steps(slab(3), 2)
    checkpoint.save_checkpoint(str(tmp_path / "s.pkl"), b, 2, 0.0, [], {})
    c = slab(9)
    checkpoint.restore_state(c, checkpoint.load_checkpoint(str(tmp_path / "s.pkl"))["state"])
    c, ic = slab_steps(c, 2)
    _same(a, c, ia, ic)

    e = np.linspace(0.0, 1.0, 21)
    sm = np.stack([e[:-1], e[1:]], axis=1)
    ge = np.logspace(-2, np.log10(20.0), 5)
    fns = [(lambda T, nu=nu: np.clip(2.0 * nu ** -3 * T ** -0.5, 0.1, 1e4)) for nu in 0.5 * (ge[:-1] + ge[1:])]

    def sph(seed):
        return mg_imc1d.init_simulation(2000, np.full(20, 0.05), np.full(20, 0.05), sm, ge, lambda T: 0.2 * T,
                                        lambda u: u / 0.2, seed=seed)

    def sph_steps(st, n):
        info = None
        for _ in range(n):
            st, info = mg_imc1d.step(st, 2000, 2000, 0, 6000, (0.0, 1.0), 0.01, sm, ge, fns, lambda u: u / 0.2,
                                     lambda T: 0.2 + 0 * T, np.zeros(20))
        return st, info

    a, ia = sph_steps(sph(4), 3)
    b, _ = sph_steps(sph(4), 1)
    checkpoint.save_checkpoint(str(tmp_path / "m.pkl"), b, 1, 0.0, [], {})
    c = sph(8)
    checkpoint.restore_state(c, checkpoint.load_checkpoint(str(tmp_path / "m.pkl"))["state"])
    np.testing.assert_array_equal(c.groups, b.groups)
    c, ic = sph_steps(c, 2)
    _same(a, c, ia, ic)
    np.testing.assert_allclose(ic["radiation_energy_by_group"], ia["radiation_energy_by_group"], rtol=1e-12,
                               atol=1e-300)
