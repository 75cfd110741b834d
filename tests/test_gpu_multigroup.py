"""GPU parity of the multigroup path (MG_IMC/MG_IMC2D.py semantics) against the FP64 oracle.

Tolerances:
  - initial census: cells exact; groups from the double-precision Planck sampler on both
    sides: at least 99.9 % identical (a uniform that lands within one ulp of a group edge
    may round the other way), positions/directions FP32 rounding;
  - one step from an identical bank: boundary energy by group and emitted energy by cell
    to FP32 weight rounding; per-(group, cell) deposition and scalar intensity relative L1
    <= 5e-4; event count relative 1e-3;
  - per-(cell, group) comb of an identical bank: copies exact;
  - the drop-in MG step: FP64 energy closure <= 1e-12 per step.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200.engine import Engine

pytestmark = pytest.mark.gpu

SEED = 0x5EED0002
G = 8
EDGES = np.logspace(-3, np.log10(30.0), G + 1)
NU = 0.5 * (EDGES[:-1] + EDGES[1:])


def _mesh(geometry):
    e1 = np.linspace(0.0, 1.0, 13)
    e2 = np.linspace(0.0, 2.0, 21)
    if geometry == "xy":
        v = np.diff(e1)[:, None] * np.diff(e2)[None, :]
    else:
        v = np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :]
    return e1, e2, O.flat2d(v)


def _pair(geometry):
    e1, e2, vol = _mesh(geometry)
    eng = Engine(geometry, e1, e2, vol, seed=SEED, n_groups=G, group_edges=EDGES)
    orc = O.Oracle(geometry, e1, e2, vol, SEED, n_groups=G)
    return eng, orc, e1, e2


def _temperature(nx, ny):
    return O.flat2d(np.outer(np.linspace(0.1, 1.0, nx), np.linspace(1.0, 0.3, ny)))


def _sigma(T):
    return np.stack([np.clip(5.0 * n ** -3 * T ** -0.5, 1e-2, 1e5) for n in NU]).reshape(-1)


def _bank_to_oracle(eng, orc):
    b = eng.bank
    orc.set_bank(*(b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")),
                 b.view("cell").cpu().numpy(), b.view("group").cpu().numpy())


@pytest.mark.parametrize("geometry", ["xy", "rz"])
def test_multigroup_initial_census_matches_oracle(cuda, geometry):
    eng, orc, e1, e2 = _pair(geometry)
    tr = _temperature(len(e1) - 1, len(e2) - 1)
    n_gpu = eng.init_census(torch.as_tensor(tr, device=cuda), 6000)
    n_orc = orc.init_ic_mg(tr, 6000, EDGES)
    assert n_gpu == n_orc
    ob = orc.get_bank()
    np.testing.assert_array_equal(eng.bank.view("cell").cpu().numpy(), ob["cell"])
    same = np.mean(eng.bank.view("group").cpu().numpy() == ob["group"])
    assert same >= 0.999, same
    np.testing.assert_allclose(eng.bank.view("weight").cpu().numpy(), ob["weight"], rtol=1e-7)
    np.testing.assert_allclose(eng.bank.view("pos1").cpu().numpy(), ob["pos1"], rtol=2e-6, atol=1e-7)
    np.testing.assert_allclose(eng.bank.view("dir2").cpu().numpy(), ob["dir2"], rtol=2e-6, atol=1e-6)


@pytest.mark.parametrize("geometry", ["xy", "rz"])
def test_multigroup_transport_matches_oracle(cuda, geometry):
    eng, orc, e1, e2 = _pair(geometry)
    nx, ny = len(e1) - 1, len(e2) - 1
    nc = nx * ny
    T = _temperature(nx, ny)
    eng.init_census(torch.as_tensor(T, device=cuda), 4000)
    _bank_to_oracle(eng, orc)
    sig = _sigma(T)
    cv = np.full(nc, 0.2)
    src = np.zeros((G, nc))
    src[2, : nx * 3] = 0.5  # fixed source in group 2 on the first rows
    face = [np.full(ny, 1.0), None, None, None] if geometry == "xy" else [None, None, np.full(nx, 0.8), None]
    reflect = (False, False, True, True) if geometry == "xy" else (True, False, False, False)
    dev = lambda a: None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=cuda)  # noqa: E731
    res = eng.transport(dev(T), dev(sig), dev(cv), dev(src), 2, 0.01, 1.0, 4000, 3000, 2000,
                        [dev(f) for f in face], reflect, max_events=1_000_000, rz_linear_source=False)
    ro = orc.transport_mg(T, sig, cv, src.reshape(-1), 2, 0.01, 1.0, 4000, 3000, 2000, face, reflect, EDGES,
                          max_events=1_000_000)
    rep = res.report
    assert rep.n_transported == ro["n_transported"]
    np.testing.assert_allclose(rep.boundary_emission, ro["boundary_emission"], rtol=1e-7)
    bg = eng.boundary_group.cpu().numpy()
    assert np.abs(bg - ro["bnd_by_group"]).sum() <= 2e-3 * ro["boundary_emission"]
    np.testing.assert_allclose(eng.emitted.cpu().numpy(), ro["emitted"], rtol=1e-7, atol=1e-300)
    l1 = lambda a, b: np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)  # noqa: E731
    dep = eng.dep.cpu().numpy()
    si = eng.si.cpu().numpy()
    assert l1(dep, ro["dep"]) < 5e-4, l1(dep, ro["dep"])
    assert l1(si, ro["si"]) < 5e-4, l1(si, ro["si"])
    stats, esc = eng.host_stats()
    np.testing.assert_allclose(stats[0], ro["stats"][0], rtol=1e-3)
    tot_in = ro["boundary_emission"] + ro["source_emission"] + ro["emission_total"]
    assert abs(esc[:4].sum() - ro["escaped"].sum()) <= 5e-4 * tot_in
    assert np.abs(eng.escaped_group.cpu().numpy() - ro["esc_by_group"]).sum() <= 1e-3 * tot_in


def test_multigroup_comb_per_group_matches_oracle(cuda):
    eng, orc, e1, e2 = _pair("xy")
    nc = (len(e1) - 1) * (len(e2) - 1)
    rng = np.random.default_rng(9)
    n = 30000
    w = rng.uniform(0.1, 2.0, n).astype(np.float32).astype(np.float64)
    cell = rng.integers(0, nc, n).astype(np.int32)
    grp = rng.integers(0, G, n).astype(np.int32)
    f = lambda: rng.uniform(0, 1, n).astype(np.float32).astype(np.float64)  # noqa: E731
    d1, d2, p1, p2 = f(), f(), f(), f()
    eng.bank.load(w, d1, d2, np.zeros(n), p1, p2, cell, grp)
    orc.set_bank(w, d1, d2, np.zeros(n), p1, p2, cell, grp)
    rep = eng.comb(12000, 4, per_group=True)
    disc_o = orc.comb(12000, 4, per_group=True)
    ob = orc.get_bank()
    assert rep.n_out == len(ob["weight"])
    np.testing.assert_array_equal(eng.bank.view("cell").cpu().numpy(), ob["cell"])
    np.testing.assert_array_equal(eng.bank.view("group").cpu().numpy(), ob["group"])
    np.testing.assert_allclose(eng.bank.view("weight").cpu().numpy(), ob["weight"], rtol=1e-7)
    np.testing.assert_allclose(eng.disc.cpu().numpy()[: nc * G], disc_o, atol=1e-4 * w.sum() / (nc * G))


def test_multigroup_dropin_ledger_closes(cuda):
    """Four steps of mg_imc2d on a hot-wall slab: FP64 energy closure <= 1e-12."""
    from radtranbook_b200 import mg_imc2d

    nx, L = 40, 0.5
    x_e = np.linspace(0.0, L, nx + 1)
    y_e = np.array([0.0, 1.0])
    edges = np.logspace(-4, np.log10(20.0), 11)
    nu = 0.5 * (edges[:-1] + edges[1:])
    cv = 0.3
    T0 = np.full((nx, 1), 0.01)
    eos = lambda T: cv * T  # noqa: E731
    inv_eos = lambda e: e / cv  # noqa: E731
    st = mg_imc2d.init_simulation(20000, T0, T0, x_e, y_e, edges, eos, inv_eos, geometry="xy")
    sig = [(lambda T, n=n: np.clip(10.0 * n ** -3 * np.maximum(T, 1e-4) ** -0.5, 1e-2, 1e6)) for n in nu]
    for _ in range(4):
        st, info = mg_imc2d.step(st, 20000, 10000, 0, 60000, (1.0, 0.0, 0.0, 0.0), 0.005, x_e, y_e, edges, sig,
                                 inv_eos, lambda T: np.full_like(T, cv), 0.0, reflect=(False, False, True, True))
        assert abs(info["ledger"]["relative_closure"]) < 1e-12, info["ledger"]
        assert info["profiling"]["transport_events"]["total"] > 0
    assert np.all(np.isfinite(info["temperature"]))
    assert info["temperature"][0, 0] > 0.05
    assert info["radiation_energy_by_group"].shape == (10, nx, 1)
