"""The fused material update (imc_material_update_law): with a LinearEOS, Constant heat
capacity and Constant / PowerLawOpacity opacity, the drop-in step does e += dep - emitted/V,
the radiation temperature, T = e / cv and the next step's opacity in one kernel.

  - same results: the reduced crooked pipe (per-cell constant opacity and heat capacity,
    linear EOS) run with the parametric materials and with plain device callables of the
    same arithmetic, from the same seed, gives the same temperatures (relative 1e-12) and
    event counts (exactly) over four steps, and both ledgers close to 1e-12;
  - the power law: after a slab step the opacity the kernel evaluated for the next step
    equals the law evaluated by torch on the new temperature (relative 1e-14), and setting
    the temperature by hand discards it;
  - the multigroup law (GroupPowerLawOpacity, the multigroup crooked pipe): after three
    mg_imc2d steps the kernel's opacity of every group equals the law evaluated by torch on
    the new temperature (relative 1e-14; torch takes T^-1/2 as rsqrt, the kernel as pow), its
    heat capacity is the problem's, and T = e / cv exactly;
  - the post-comb radiation energy by group that the comb writes per bin (copies x FP32
    weight) equals the energy of the new census summed entry by entry (relative 1e-12).
"""
import numpy as np
import pytest
import torch

from radtranbook_b200 import imc1d, imc2d, mg_imc2d, problems
from radtranbook_b200.materials import device_callable

pytestmark = pytest.mark.gpu


def _pipe_run(p, sig, cv, eos, inv_eos, steps=4):
    st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], eos, inv_eos,
                               geometry="rz", seed=0x1A7)
    rec = []
    for _ in range(steps):
        st, info = imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], p["edges1"],
                              p["edges2"], sig, inv_eos, cv, p["source"], reflect=p["reflect"], geometry="rz",
                              boundary_source_func=p["boundary_source_func"])
        rec.append((info["profiling"]["transport_events"]["total"], info["N_particles"],
                    info["ledger"]["relative_closure"]))
    return st, rec


def test_fused_material_update_matches_device_callables(cuda):
    p = problems.crooked_pipe(scale=0.02, nr=30, nz=105)
    st_law, rec_law = _pipe_run(p, p["sigma_dev"], p["cv_dev"], p["eos_dev"], p["inv_eos_dev"])
    assert st_law.__dict__.get("_law_next") is not None  # the fused path ran
    sig_t = torch.as_tensor(p["sigma_host"](p["Tinit"]), device=cuda)
    cvg = torch.as_tensor(p["cv_host"](p["Tinit"]), device=cuda)
    st_fn, rec_fn = _pipe_run(p, device_callable(lambda T: sig_t), device_callable(lambda T: cvg),
                              device_callable(lambda T: cvg * T), device_callable(lambda e: e / cvg))
    assert st_fn.__dict__.get("_law_next") is None  # plain callables: the unfused path
    for (ev1, n1, c1), (ev2, n2, c2) in zip(rec_law, rec_fn):
        assert ev1 == ev2 and n1 == n2
        assert abs(c1) < 1e-12 and abs(c2) < 1e-12
    np.testing.assert_allclose(st_law.temperature, st_fn.temperature, rtol=1e-12, atol=0)
    np.testing.assert_allclose(st_law.radiation_temperature, st_fn.radiation_temperature, rtol=1e-12, atol=0)


def test_power_law_next_opacity_is_the_law(cuda):
    q = problems.marshak_slab(scale=0.2)
    st = imc1d.init_simulation(q["Ntarget"], q["Tinit"], q["Tr_init"], q["mesh"], q["eos_dev"], q["inv_eos_dev"])
    for _ in range(3):
        st, info = imc1d.step(st, q["Ntarget"], q["Nboundary"], 0, q["Nmax"], q["T_boundary"], q["dt"], q["mesh"],
                              q["sigma_dev"], q["inv_eos_dev"], q["cv_dev"], q["source"])
        assert abs(info["ledger"]["relative_closure"]) < 1e-12
    key, sig_next, cv_next = st.__dict__["_law_next"]
    T = st._T
    torch.testing.assert_close(sig_next, q["sigma_dev"](T), rtol=1e-14, atol=0)
    torch.testing.assert_close(cv_next, torch.full_like(T, 0.3), rtol=0, atol=0)
    st.temperature = st.temperature * 1.01  # a temperature set by hand: the next opacity is re-evaluated
    assert st.__dict__.get("_law_next") is None
    st, info = imc1d.step(st, q["Ntarget"], q["Nboundary"], 0, q["Nmax"], q["T_boundary"], q["dt"], q["mesh"],
                          q["sigma_dev"], q["inv_eos_dev"], q["cv_dev"], q["source"])
    assert info["profiling"]["transport_events"]["total"] > 0


def _mg_pipe_steps(p, steps):
    e1, e2, ge = p["edges1"], p["edges2"], p["energy_edges"]
    st = mg_imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], e1, e2, ge, p["eos_dev"],
                                  p["inv_eos_dev"], T_emit_floor=p["T_emit_floor"], geometry="rz", seed=0x6A7)
    dt, infos = p["dt_initial"], []
    for k in range(steps):
        st, info = mg_imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"] + k * p["Nmax_growth"],
                                 p["T_boundary"], dt, e1, e2, ge, p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"],
                                 p["source"], reflect=p["reflect"], geometry="rz",
                                 boundary_source_func=p["boundary_source_func"], T_emit_floor=p["T_emit_floor"],
                                 Nmax_growth=p["Nmax_growth"], Nmax_final=p["Nmax_final"])
        assert abs(info["ledger"]["relative_closure"]) < 1e-12
        infos.append(info)
        dt = min(dt * p["dt_growth"], p["dt_max"])
    return st, infos


def test_group_power_law_next_opacity_is_the_law(cuda):
    p = problems.mg_crooked_pipe(nr=30, nz=105, mode="quick")
    st, _ = _mg_pipe_steps(p, 3)
    key, sig_next, cv_next = st.__dict__["_law_next"]
    like = st.grid(st._T)
    want = p["sigma_dev"].all_groups(like).transpose(1, 2).reshape(-1)  # (G, nx, ny) -> [g][c] cell order
    torch.testing.assert_close(sig_next, want, rtol=1e-14, atol=0)
    cvg = st.flat(torch.as_tensor(p["cv_host"](p["Tinit"]), device=cuda))
    torch.testing.assert_close(cv_next, cvg, rtol=0, atol=0)
    torch.testing.assert_close(st._T, st._e / cvg, rtol=0, atol=0)
    assert float(st._T.max()) > 0.05  # heated near the source: the opacities changed


def test_comb_after_energy_is_the_new_census(cuda):
    p = problems.mg_crooked_pipe(nr=30, nz=105, mode="quick")
    st, infos = _mg_pipe_steps(p, 2)
    G, nx, ny = 10, 30, 105
    census = mg_imc2d._rad_by_group(st._engine).view(G, ny, nx).transpose(1, 2).cpu().numpy()
    post = infos[-1]["radiation_energy_by_group_postcomb"]
    assert post.shape == (G, nx, ny) and post.sum() > 0
    np.testing.assert_allclose(post, census, rtol=1e-12, atol=1e-300)


def test_mg_report_fields_are_the_engine_fields(cuda):
    """The step's reported arrays come from one gather kernel (imc_mg_report_fields) and one
    copy: they equal, bit for bit, the fields computed from the engine's tensors on the host
    (si / c and comb_after / V by group, NumPy's correctly rounded divisions, transposed to
    (G, nx, ny); T, Tr, e in (nx, ny); the boundary and escaped energy by group)."""
    from radtranbook_b200.engine import C_LIGHT

    p = problems.mg_crooked_pipe(nr=30, nz=105, mode="quick")
    st, infos = _mg_pipe_steps(p, 2)
    eng, info = st._engine, infos[-1]
    G, nx, ny, nc = 10, 30, 105, 30 * 105

    def grid3(x):
        return x.reshape(G, ny, nx).transpose(0, 2, 1)

    si, after, vol = (t.cpu().numpy() for t in (eng.si, eng.comb_after, eng.vol))
    np.testing.assert_array_equal(info["radiation_energy_by_group"], grid3(si.reshape(G, nc) / C_LIGHT))
    np.testing.assert_array_equal(info["radiation_energy_by_group_postcomb"],
                                  grid3(after.reshape(G, nc) / vol.reshape(1, nc)))
    np.testing.assert_array_equal(info["temperature"], st.grid(st._T).cpu().numpy())
    np.testing.assert_array_equal(info["radiation_temperature"], st.grid(st._Tr).cpu().numpy())
    np.testing.assert_array_equal(st.internal_energy, st.grid(st._e).cpu().numpy())
    np.testing.assert_array_equal(info["boundary_emission_by_group"], eng.boundary_group.cpu().numpy())
    np.testing.assert_array_equal(info["boundary_outgoing_by_group"], eng.escaped_group.cpu().numpy())


def test_mg_report_sections_make_the_full_report(cuda):
    """imc_mg_report_fields with NULL inputs skips their sections: the early call (all but the
    post-comb energies) and the post-comb call fill, between them, the buffer one full call
    fills, entry for entry."""
    p = problems.mg_crooked_pipe(nr=30, nz=105, mode="quick")
    st, _ = _mg_pipe_steps(p, 2)
    eng = st._engine
    eng.mg_report_fields(st._e, st._T, st._Tr)
    full = eng.report_dev.clone()
    eng.report_dev.fill_(float("nan"))
    eng.mg_report_fields(st._e, st._T, st._Tr, sections="early")
    G, nc = eng.ng, eng.nc
    assert torch.isnan(eng.report_dev[G * nc:2 * G * nc]).all()  # the post-comb section is left alone
    eng.mg_report_fields(None, None, None, sections="post")
    torch.cuda.synchronize()
    assert torch.equal(eng.report_dev, full)
