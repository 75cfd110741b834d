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
