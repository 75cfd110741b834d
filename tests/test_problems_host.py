"""Host-side checks of the problem definitions (no GPU): the multigroup crooked pipe's
geometry and materials follow MG_IMC/problems/crooked_pipe_multigroup_imc.py, and its grouped
opacity evaluation gives exactly the per-group callables' numbers."""
import numpy as np
import torch

from radtranbook_b200 import problems
from radtranbook_b200.materials import GroupedOpacity, evaluate_groups


def test_mg_crooked_pipe_layout():
    p = problems.mg_crooked_pipe()
    assert p["edges1"][-1] == 2.0 and p["edges2"][-1] == 7.0 and p["rho"].shape == (60, 210)
    rc = 0.5 * (p["edges1"][:-1] + p["edges1"][1:])
    zc = 0.5 * (p["edges2"][:-1] + p["edges2"][1:])
    R, Z = np.meshgrid(rc, zc, indexing="ij")
    # the pipe: axis channel below z = 3 and above z = 4, the two radial legs, the outer leg
    assert np.all(p["rho"][(R < 0.5) & (Z < 2.9)] == 0.1)
    assert np.all(p["rho"][(R > 1.0) & (R < 1.5) & (Z > 2.6) & (Z < 4.4)] == 0.1)
    assert np.all(p["rho"][(R > 1.6)] == 2.0) and np.all(p["rho"][(R > 0.55) & (R < 0.95) & (Z < 2.4)] == 2.0)
    np.testing.assert_allclose(p["energy_edges"], np.logspace(-2, 1, 11))
    assert p["boundary_source_func"](0.2, 0.0, "zmin") == 0.5 and p["boundary_source_func"](0.7, 0.0, "zmin") == 0.0
    assert p["reflect"] == (True, False, False, False) and p["T_emit_floor"] == 0.075


def test_grouped_opacity_equals_per_group_callables():
    p = problems.mg_crooked_pipe(nr=30, nz=105)
    assert isinstance(p["sigma_dev"], GroupedOpacity) and len(p["sigma_dev"]) == 10
    rng = np.random.default_rng(3)
    T = torch.as_tensor(rng.uniform(0.001, 2.0, (30, 105)))
    grouped = evaluate_groups(p["sigma_dev"], T, None, T)
    each = torch.stack([f(T) for f in p["sigma_dev"]])
    assert torch.equal(grouped, each)
    host = np.stack([f(T.numpy()) for f in p["sigma_host"]])
    np.testing.assert_allclose(grouped.numpy(), host, rtol=1e-14)
    # a plain list falls back to one evaluation per group
    plain = evaluate_groups(list(p["sigma_dev"]), T, None, T)
    assert torch.equal(plain, each)


def test_group_power_law_builds_the_device_law():
    """The multigroup problems' device materials are laws the step evaluates in its material
    update kernel: the fields of imc_material_law they produce (no GPU: CPU tensors)."""
    from radtranbook_b200.materials import GroupPowerLawOpacity, material_law

    p = problems.mg_crooked_pipe(nr=30, nz=105)
    flat = lambda t: t.T.reshape(-1)  # noqa: E731  (nx, ny) -> cell order c = i + nx j
    law, keep = material_law(p["sigma_dev"], p["cv_dev"], p["inv_eos_dev"], flat, torch.device("cpu"))
    assert isinstance(p["sigma_dev"], GroupPowerLawOpacity)
    assert (law.sigma_A, law.sigma_n, law.sigma_T_floor, law.sigma_lo, law.sigma_hi) == (10.0, 0.5, 1e-2, 0.0, 0.0)
    assert law.sigma_scale and law.sigma_group and law.cv_array and law.cv_eos_array and not law.sigma_array
    ptrs = {t.data_ptr(): t for t in keep}
    np.testing.assert_array_equal(ptrs[law.sigma_scale].numpy(), flat(torch.as_tensor(p["rho"])).numpy())
    e = p["energy_edges"]
    np.testing.assert_array_equal(ptrs[law.sigma_group].numpy(), (e[:-1] * e[1:]) ** -1.5)
    q = problems.marshak_mg()
    law, keep = material_law(q["sigma_dev"], q["cv_dev"], q["inv_eos_dev"], flat, torch.device("cpu"))
    assert (law.sigma_lo, law.sigma_hi, law.sigma_T_floor) == (1e-2, 1e6, 0.0) and not law.sigma_scale
    assert law.cv == 0.3 and law.cv_eos == 0.3 and not law.cv_array
    # host and device evaluation of the Marshak law agree with the problem's host callables
    T = np.random.default_rng(5).uniform(1e-3, 2.0, (200, 1))
    host = np.stack([f(T) for f in q["sigma_host"]])
    np.testing.assert_allclose(q["sigma_dev"].all_groups(T), host, rtol=1e-14)
    np.testing.assert_allclose(q["sigma_dev"].all_groups(torch.as_tensor(T)).numpy(), host, rtol=1e-14)
    # a plain callable is no law
    assert material_law(list(p["sigma_dev"]), p["cv_dev"], p["inv_eos_dev"], flat, torch.device("cpu")) is None
