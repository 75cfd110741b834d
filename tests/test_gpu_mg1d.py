"""GPU parity of the multigroup 1-D sphere path (MG_IMC/MG_IMC1D.py semantics) against the
FP64 oracle, and of the drop-in step against the reference's own statistics.

Tolerances:
  - initial census and sources: per-(group, cell) counts and cells exact (the counts come
    from the same FP64 operation order on both sides); groups from the double-precision
    Planck sampler at least 99.9 % identical (a uniform within one ulp of a group edge may
    round the other way); weights FP32 rounding (rtol 1e-7);
  - one step from an identical bank: per-(group, cell) deposition and scalar intensity
    relative L1 <= 5e-4, event count relative 1e-3, escaped energy by group within 1e-3 of
    the energy put in;
  - comb modes on an identical bank: copies exact, weights FP32 rounding;
  - the drop-in step: FP64 energy closure <= 1e-12 per step in every comb-energy mode, and
    32-seed means of T and Tr within the combined standard errors of MG_IMC1D.step's
    (tests/golden/stats_mg1d.npz).
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200.engine import Engine

pytestmark = pytest.mark.gpu

SEED = 0x5EED0003
G = 6
EDGES = np.logspace(-2, np.log10(20.0), G + 1)
NU = 0.5 * (EDGES[:-1] + EDGES[1:])
I = 40


def _pair():
    e = np.linspace(0.0, 1.0, I + 1) ** 1.2
    vol = 4.0 / 3.0 * np.pi * (e[1:] ** 3 - e[:-1] ** 3)
    eng = Engine("spherical", e, np.array([0.0, 1.0]), vol, seed=SEED, n_groups=G, group_edges=EDGES)
    orc = O.Oracle("spherical", e, np.array([0.0, 1.0]), vol, SEED, n_groups=G)
    return eng, orc, e


def _temperature():
    return np.linspace(1.0, 0.05, I)


def _sigma(T):
    return np.stack([np.clip(3.0 * n ** -3 * T ** -0.5, 0.05, 1e4) for n in NU])


def _bank_to_oracle(eng, orc):
    b = eng.bank
    orc.set_bank(*(b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")),
                 b.view("cell").cpu().numpy(), b.view("group").cpu().numpy())


def _dev(a, cuda):
    return None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=cuda)


def test_mg1d_initial_census_matches_oracle(cuda):
    eng, orc, e = _pair()
    tr = _temperature()
    tr[5] = 0.0  # an empty shell
    n_gpu = eng.init_census(torch.as_tensor(tr, device=cuda), 7000)
    n_orc = orc.init_ic_mg1d(tr, 7000, EDGES)
    assert n_gpu == n_orc
    ob = orc.get_bank()
    np.testing.assert_array_equal(eng.bank.view("cell").cpu().numpy(), ob["cell"])
    assert np.mean(eng.bank.view("group").cpu().numpy() == ob["group"]) >= 0.999
    np.testing.assert_allclose(eng.bank.view("weight").cpu().numpy(), ob["weight"], rtol=1e-7)
    np.testing.assert_allclose(eng.bank.view("pos1").cpu().numpy(), ob["pos1"], rtol=2e-6, atol=1e-7)
    np.testing.assert_allclose(eng.bank.view("dir1").cpu().numpy(), ob["dir1"], rtol=2e-6, atol=1e-6)


def test_mg1d_sources_match_oracle(cuda):
    """Stratified emission and fixed-source bins and the boundary: the sources alone."""
    eng, orc, e = _pair()
    T = _temperature()
    sig = _sigma(T)
    cv = np.full(I, 0.1)
    src = np.zeros((G, I))
    src[1, :10] = 2.0
    src[4, 20:] = 0.5
    face = [None, np.array([0.7]), None, None]
    dt = 0.005
    rep = eng.transport(_dev(T, cuda), _dev(sig, cuda), _dev(cv, cuda), _dev(src, cuda), 1, dt, 1.0, 5000, 3000, 2000,
                        [_dev(f, cuda) for f in face], (True, False), max_events=0, rz_linear_source=False).report
    ro = orc.transport_mg1d(T, sig, cv, src, 1, dt, 1.0, 5000, 3000, 2000, face, (True, False, False, False), EDGES,
                            sources_only=True)
    n_all = orc.size
    orc2 = _pair()[1]
    orc2.transport_mg1d(T, sig, cv, src, 1, dt, 1.0, 0, 3000, 2000, face, (True, False, False, False), EDGES,
                        sources_only=True)
    assert rep.n_transported == n_all
    assert rep.n_boundary == 3000
    assert rep.n_source == orc2.size - 3000
    assert rep.n_emission == n_all - orc2.size
    np.testing.assert_allclose(rep.boundary_emission, ro["boundary_emission"], rtol=1e-7)
    np.testing.assert_allclose(rep.source_emission, ro["source_emission"], rtol=1e-6)
    np.testing.assert_allclose(rep.emission_total, ro["emission_total"], rtol=1e-6)
    np.testing.assert_allclose(eng.emitted.cpu().numpy(), ro["emitted"], rtol=1e-6, atol=1e-300)
    np.testing.assert_allclose(eng.sigma_a.cpu().numpy(), ro["sigma_a"].reshape(-1), rtol=1e-14)


def test_mg1d_transport_matches_oracle(cuda):
    eng, orc, e = _pair()
    T = _temperature()
    eng.init_census(torch.as_tensor(T, device=cuda), 5000)
    _bank_to_oracle(eng, orc)
    sig = _sigma(T)
    cv = np.full(I, 0.1)
    face = [None, np.array([0.7]), None, None]
    dt = 0.005
    res = eng.transport(_dev(T, cuda), _dev(sig, cuda), _dev(cv, cuda), None, 2, dt, 1.0, 5000, 3000, 0,
                        [_dev(f, cuda) for f in face], (True, False), max_events=0, rz_linear_source=False)
    ro = orc.transport_mg1d(T, sig, cv, None, 2, dt, 1.0, 5000, 3000, 0, face, (True, False, False, False), EDGES)
    rep = res.report
    assert rep.n_transported == ro["n_transported"]
    np.testing.assert_allclose(rep.weight_floor, ro["weight_floor"], rtol=1e-6)
    l1 = lambda a, b: np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)  # noqa: E731
    assert l1(eng.dep.cpu().numpy(), ro["dep"]) < 5e-4
    assert l1(eng.si.cpu().numpy(), ro["si"]) < 5e-4
    stats, esc = eng.host_stats()
    np.testing.assert_allclose(stats[0], ro["stats"][0], rtol=1e-3)
    tot_in = ro["boundary_emission"] + ro["emission_total"] + float(np.sum(orc.get_bank()["weight"]))
    assert np.abs(eng.escaped_group.cpu().numpy() - ro["esc_by_group"]).sum() <= 1e-3 * tot_in


def _random_bank(eng, orc, n, seed):
    rng = np.random.default_rng(seed)
    w = (rng.uniform(0.1, 2.0, n) * (rng.uniform(size=n) > 0.1)).astype(np.float32).astype(np.float64)
    cell = rng.integers(0, I, n).astype(np.int32)
    grp = rng.integers(0, G, n).astype(np.int32)
    f = lambda: rng.uniform(0, 1, n).astype(np.float32).astype(np.float64)  # noqa: E731
    d1, p1, t = f(), f(), f()
    eng.bank.load(w, d1, np.zeros(n), t, p1, np.zeros(n), cell, grp)
    orc.set_bank(w, d1, np.zeros(n), t, p1, np.zeros(n), cell, grp)
    return w


@pytest.mark.parametrize("nmax,conserve", [(15000, False), (15000, True), (0, False), (-10**7, False),
                                           (-15000, False)])
def test_mg1d_comb_modes_match_oracle(cuda, nmax, conserve):
    eng, orc, e = _pair()
    w = _random_bank(eng, orc, 40000, 11)
    rep = eng.comb(nmax, 3, per_group=True, conserve_radiation=conserve)
    disc_o = orc.comb(nmax, 3, per_group=True, conserve_radiation=conserve)
    ob = orc.get_bank()
    assert rep.n_out == len(ob["weight"])
    np.testing.assert_array_equal(eng.bank.view("cell").cpu().numpy(), ob["cell"])
    np.testing.assert_array_equal(eng.bank.view("group").cpu().numpy(), ob["group"])
    np.testing.assert_array_equal(eng.bank.view("pos1").cpu().numpy(), ob["pos1"].astype(np.float32))
    np.testing.assert_allclose(eng.bank.view("weight").cpu().numpy(), ob["weight"], rtol=1e-7)
    assert np.all(eng.bank.view("time").cpu().numpy() == 0.0)
    np.testing.assert_allclose(eng.disc.cpu().numpy()[: I * G], disc_o, atol=1e-6 * w.sum() / (I * G))
    if nmax == 0 or nmax == -10**7:
        assert rep.n_out == int(np.sum(w > 0))  # compact only
        assert np.all(eng.disc.cpu().numpy()[: I * G] == 0.0)


@pytest.mark.parametrize("conserve", [True, "radiation", False])
def test_mg1d_dropin_ledger_closes(cuda, conserve):
    from radtranbook_b200 import mg_imc1d

    e = np.linspace(0.0, 1.0, 31)
    mesh = np.stack([e[:-1], e[1:]], axis=1)
    edges = np.logspace(-2, np.log10(20.0), 5)
    nu = 0.5 * (edges[:-1] + edges[1:])
    cv = 0.2
    funcs = [(lambda T, n=n: np.clip(2.0 * n ** -3 * np.power(T, -0.5), 0.1, 1e4)) for n in nu]
    st = mg_imc1d.init_simulation(3000, np.full(30, 0.05), np.full(30, 0.05), mesh, edges, lambda T: cv * T,
                                  lambda u: u / cv)
    src = np.zeros(30)
    src[:5] = 1.0
    for k in range(4):
        st, info = mg_imc1d.step(st, 3000, 3000, 1000, 8000, (0.0, 1.0), 0.01, mesh, edges, funcs, lambda u: u / cv,
                                 lambda T: cv + 0 * T, src, conserve_comb_energy=conserve)
        assert abs(info["ledger"]["relative_closure"]) < 1e-12, info["ledger"]
        if conserve is True:
            assert abs(info["energy_residual"]) < 1e-12 * info["total_energy"]
    assert info["radiation_energy_by_group"].shape == (4, 30)
    assert info["radiation_flux_by_group"].shape == (4, 30)
    assert st.groups.shape == st.weights.shape
    np.testing.assert_allclose(info["radiation_energy_by_group"].sum(), info["total_radiation_energy"], rtol=1e-9)


def test_mg1d_dropin_budget_and_threshold(cuda):
    """particle_budget_fmin splits Ntarget over the sources by energy (per-side boundary
    counts); Nmax < 0 combs only above the threshold."""
    from radtranbook_b200 import mg_imc1d

    e = np.linspace(0.2, 1.0, 21)
    mesh = np.stack([e[:-1], e[1:]], axis=1)
    edges = np.logspace(-2, np.log10(20.0), 4)
    cv = 0.2
    funcs = [lambda T: np.full_like(T, 3.0)] * 3
    st = mg_imc1d.init_simulation(2000, np.full(20, 0.1), np.full(20, 0.1), mesh, edges, lambda T: cv * T,
                                  lambda u: u / cv)
    st, info = mg_imc1d.step(st, 6000, 0, 0, -10**8, (0.5, 1.0), 0.01, mesh, edges, funcs, lambda u: u / cv,
                             lambda T: cv + 0 * T, np.zeros(20), particle_budget_fmin=0.05)
    r0, r1 = e[0], e[-1]
    E_in, E_out = (0.01372 * 29.98 * Tb ** 4 / 4.0 * 0.01 * 4 * np.pi * R * R for Tb, R in ((0.5, r0), (1.0, r1)))
    # counts in proportion to energy, at least 5 % of the budget each
    assert info["N_boundary"] >= 2 * 300
    assert abs(info["ledger"]["relative_closure"]) < 1e-12
    np.testing.assert_allclose(info["boundary_emission"], E_in + E_out, rtol=1e-6)
    # threshold far above the census: no comb, every live entry kept, nothing lost
    assert info["ledger"]["comb_discrepancy"] == 0.0
    assert 0 < info["N_particles"] <= info["profiling"]["transport_events"]["n_particles_transported"]


def test_threshold_comb_reads_the_tracking_live_count(cuda):
    """A threshold comb (Nmax < 0) decides from the live count the tracking leaves in the
    workspace; tracking and comb lay the workspace out for different bank sizes, so that count
    (like the census sums) must sit at an offset independent of them.  With every workspace
    byte set to 0xFF before each step, a threshold far above the census still only drops dead
    entries, step after step."""
    from radtranbook_b200 import mg_imc1d

    e = np.linspace(0.2, 1.0, 21)
    mesh = np.stack([e[:-1], e[1:]], axis=1)
    edges = np.logspace(-2, np.log10(20.0), 4)
    cv = 0.2
    funcs = [lambda T: np.full_like(T, 3.0)] * 3
    st = mg_imc1d.init_simulation(2000, np.full(20, 0.1), np.full(20, 0.1), mesh, edges, lambda T: cv * T,
                                  lambda u: u / cv)
    args = (6000, 0, 0, -10**8, (0.5, 1.0), 0.01, mesh, edges, funcs, lambda u: u / cv, lambda T: cv + 0 * T,
            np.zeros(20))
    st, info = mg_imc1d.step(st, *args)  # sizes the workspace
    for _ in range(3):
        st._engine.ws.fill_(0xFF)
        st, info = mg_imc1d.step(st, *args)
        assert info["ledger"]["comb_discrepancy"] == 0.0
        assert 0 < info["N_particles"] <= info["profiling"]["transport_events"]["n_particles_transported"]
        assert abs(info["ledger"]["relative_closure"]) < 1e-12


def test_mg1d_dropin_matches_reference_statistically(cuda):
    from radtranbook_b200 import mg_imc1d
    from tests.stat_problems import compare_means

    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "stats_mg1d.npz"))
    d = {k: (ref[k].item() if ref[k].ndim == 0 else ref[k]) for k in ref.files}
    I_, cv = int(d["I"]), float(d["cv"])
    e = np.linspace(0.0, float(d["R"]), I_ + 1)
    mesh = np.stack([e[:-1], e[1:]], axis=1)
    edges = np.logspace(-2, np.log10(20.0), int(d["G"]) + 1)
    nu = 0.5 * (edges[:-1] + edges[1:])
    funcs = [(lambda T, n=n: np.clip(2.0 * n ** -3 * np.power(T, -0.5), 0.1, 1e4)) for n in nu]
    Ts, Trs = [], []
    seeds = int(d["seeds"])
    for s in range(seeds):
        st = mg_imc1d.init_simulation(int(d["Ntarget"]), np.full(I_, float(d["T0"])), np.full(I_, float(d["T0"])),
                                      mesh, edges, lambda T: cv * T, lambda u: u / cv, seed=0xA000 + s)
        for _ in range(int(d["steps"])):
            st, info = mg_imc1d.step(st, int(d["Ntarget"]), int(d["Nboundary"]), 0, int(d["Nmax"]),
                                     (0.0, float(d["Tb"])), float(d["dt"]), mesh, edges, funcs, lambda u: u / cv,
                                     lambda T: cv + 0 * T, np.zeros(I_))
        Ts.append(st.temperature.copy())
        Trs.append(st.radiation_temperature.copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    roi = np.ones(I_, dtype=bool)
    compare_means(Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds), ref["T_mean"], ref["T_se"], roi)
    compare_means(Trs.mean(0), Trs.std(0, ddof=1) / np.sqrt(seeds), ref["Tr_mean"], ref["Tr_se"], roi)
