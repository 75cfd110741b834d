"""The fused material update (imc_material_update_law): with a LinearEOS, Constant heat
capacity and Constant / PowerLawOpacity opacity, the drop-in step does e += dep - emitted/V,
the radiation temperature, T = e / cv and the next step's opacity in one kernel.

  - same results: the reduced crooked pipe (per-cell constant opacity and heat capacity,
    linear EOS) run with the parametric materials and with plain device callables of the
    same arithmetic, from the same seed, gives the same temperatures (relative 1e-12) and
    event counts (exactly) over four steps, and both ledgers close to 1e-12;
  - the power law: after a slab step the opacity the kernel evaluated for the next step
    equals the law evaluated by torch on the new temperature (relative 1e-14), and setting
    the temperature by hand discards it.
"""
import numpy as np
import pytest
import torch

from radtranbook_b200 import imc1d, imc2d, problems
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
