"""The arrays a step returns (info and the state's host mirrors) view the pinned buffer that
the step's device-to-host copy filled.  A loop that keeps only the last info keeps the views
(a fresh buffer each step from torch's caching pinned allocator); a loop that keeps every
info makes the state switch to one buffer of its own and copies, and every kept array still
holds the values it was returned with."""
import numpy as np
import pytest

from radtranbook_b200 import imc1d, mg_imc2d, problems

pytestmark = pytest.mark.gpu


def _slab_steps(n, keep):
    q = problems.marshak_slab(scale=0.2)
    st = imc1d.init_simulation(q["Ntarget"], q["Tinit"], q["Tr_init"], q["mesh"], q["eos_dev"], q["inv_eos_dev"])
    kept = []
    for _ in range(n):
        st, info = imc1d.step(st, q["Ntarget"], q["Nboundary"], 0, q["Nmax"], q["T_boundary"], q["dt"], q["mesh"],
                              q["sigma_dev"], q["inv_eos_dev"], q["cv_dev"], q["source"])
        if keep:
            kept.append((info, info["temperature"].copy(), info["radiation_temperature"].copy()))
    return st, kept


def test_gray_kept_infos_are_intact(cuda):
    st, kept = _slab_steps(6, keep=True)
    assert st.__dict__.get("_host_copy_mode")
    for info, T, Tr in kept:
        np.testing.assert_array_equal(info["temperature"], T)
        np.testing.assert_array_equal(info["radiation_temperature"], Tr)
    assert not np.array_equal(kept[0][1], kept[-1][1])  # the wave moved: the arrays differ
    st2, _ = _slab_steps(6, keep=False)
    assert not st2.__dict__.get("_host_copy_mode")


def test_mg_kept_infos_are_intact(cuda):
    p = problems.mg_crooked_pipe(nr=30, nz=105, mode="quick")
    e1, e2, ge = p["edges1"], p["edges2"], p["energy_edges"]
    st = mg_imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], e1, e2, ge, p["eos_dev"],
                                  p["inv_eos_dev"], T_emit_floor=p["T_emit_floor"], geometry="rz", seed=0x4B1)
    kept, dt = [], p["dt_initial"]
    for _ in range(5):
        st, info = mg_imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], dt, e1, e2, ge,
                                 p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"], reflect=p["reflect"],
                                 geometry="rz", boundary_source_func=p["boundary_source_func"],
                                 T_emit_floor=p["T_emit_floor"])
        kept.append((info, {k: np.array(info[k]) for k in ("radiation_energy_by_group",
                                                            "radiation_energy_by_group_postcomb", "temperature",
                                                            "boundary_emission_by_group")}))
        dt *= p["dt_growth"]
    assert st.__dict__.get("_host_copy_mode")
    for info, snap in kept:
        for k, v in snap.items():
            np.testing.assert_array_equal(info[k], v)
    np.testing.assert_array_equal(st.temperature, kept[-1][0]["temperature"])
