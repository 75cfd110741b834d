"""Multigroup 1-D sphere (MG_IMC/MG_IMC1D.py) oracle checks, no GPU: the oracle's
stratified emission / fixed-source / initial-census counts and weights, per-(cell, group)
comb (both energy modes), spherical event and Planck sampler against golden vectors
recorded from the reference (tests/golden/mg1d.npz, with the reference's own draws
replayed), energy closure, and statistical parity of whole steps with MG_IMC1D.step
(tests/golden/stats_mg1d.npz, planck_shim standing in for planck_integrals).

Tolerances: counts, cells, groups and comb copies are exact; FP64 weights agree to 1e-12
relative (the Planck fractions here are a series, the reference's are quadrature through
the shim: 1e-13 apart).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_pins import _uniforms

G_DIR = os.path.join(os.path.dirname(__file__), "golden")


def _pins():
    return np.load(os.path.join(G_DIR, "mg1d.npz"))


def _sphere(e, G, seed=1):
    vol = 4.0 / 3.0 * np.pi * (e[1:] ** 3 - e[:-1] ** 3)
    return O.Oracle("spherical", e, np.array([0.0, 1.0]), vol, seed, n_groups=G)


def _per_bin(b, I, G):
    """counts and the (common) weight per (group, cell) bin, bins g*I + i"""
    bins = b["cell"] + I * b["group"]
    cnt = np.bincount(bins, minlength=G * I)
    w = np.zeros(G * I)
    w[bins] = b["weight"]
    return cnt, w


def test_mg1d_emission_counts_and_weights_match_reference():
    d = _pins()
    edges = d["edges"]
    G = len(edges) - 1
    for q in range(len(d["N"])):
        e = d["mesh"][q]
        I = len(e) - 1
        o = _sphere(e, G)
        # cv -> infinity makes the Fleck factor exactly 1, so sigma_a = the reference's input
        r = o.transport_mg1d(d["T"][q], d["saf"][q], np.full(I, 1e300), None, 0, float(d["dt"][q]), 1.0,
                             int(d["N"][q]), 0, 0, [None] * 4, (False,) * 4, edges, sources_only=True)
        cnt, w = _per_bin(o.get_bank(), I, G)
        np.testing.assert_array_equal(cnt, d["emit_counts"][q])
        np.testing.assert_allclose(w, d["emit_w"][q], rtol=1e-12, atol=0)
        np.testing.assert_allclose(r["emitted"], d["emit_by_group"][q].sum(0), rtol=1e-12)


def test_mg1d_fixed_source_counts_match_reference():
    d = _pins()
    edges = d["edges"]
    G = len(edges) - 1
    for q in range(len(d["N"])):
        e = d["mesh"][q]
        I = len(e) - 1
        o = _sphere(e, G)
        o.transport_mg1d(d["T"][q], np.ones((G, I)), np.full(I, 1e300), d["src"][q], 0, float(d["dt"][q]), 1.0, 0, 0,
                         int(d["src_N"][q]), [None] * 4, (False,) * 4, edges, sources_only=True)
        cnt, w = _per_bin(o.get_bank(), I, G)
        np.testing.assert_array_equal(cnt, d["src_counts"][q])
        np.testing.assert_allclose(w, d["src_w"][q], rtol=1e-12, atol=0)


def test_mg1d_initial_census_counts_match_reference():
    d = _pins()
    edges = d["edges"]
    G = len(edges) - 1
    for q in range(len(d["ic_N"])):
        e = d["mesh"][q]
        I = len(e) - 1
        o = _sphere(e, G)
        o.init_ic_mg1d(d["ic_Tr"][q], int(d["ic_N"][q]), edges)
        b = o.get_bank()
        np.testing.assert_array_equal(np.bincount(b["cell"], minlength=I), d["ic_counts"][q])
        w = np.zeros(I)
        w[b["cell"]] = b["weight"]
        np.testing.assert_allclose(w, d["ic_w"][q], rtol=1e-12, atol=0)
        assert np.all((b["group"] >= 0) & (b["group"] < G))
        assert np.all((b["pos1"] >= e[b["cell"]]) & (b["pos1"] <= e[b["cell"] + 1]))


@pytest.mark.parametrize("mode", ["none", "radiation"])
def test_mg1d_comb_matches_reference(mode):
    d = _pins()
    edges = d["edges"]
    G = len(edges) - 1
    I = 20
    o = _sphere(np.linspace(0, 1, I + 1), G)
    x = d[f"comb_{mode}_in"]
    n = len(x)
    o.set_bank(x[:, 0], x[:, 3], np.zeros(n), x[:, 4], x[:, 5], np.zeros(n), x[:, 1].astype(np.int32),
               x[:, 2].astype(np.int32))
    disc = o.comb_mg_with_xi(int(d["comb_nmax"]), d[f"comb_{mode}_xi"], conserve_radiation=(mode == "radiation"))
    b = o.get_bank()
    ref = d[f"comb_{mode}_out"]
    assert len(b["weight"]) == len(ref)
    np.testing.assert_array_equal(b["cell"], ref[:, 1].astype(np.int32))
    np.testing.assert_array_equal(b["group"], ref[:, 2].astype(np.int32))
    np.testing.assert_array_equal(b["dir1"], ref[:, 3])
    np.testing.assert_array_equal(b["pos1"], ref[:, 4])
    np.testing.assert_allclose(b["weight"], ref[:, 0], rtol=1e-13)
    np.testing.assert_allclose(disc, d[f"comb_{mode}_disc"].reshape(-1), atol=1e-12 * x[:, 0].sum())


def test_mg1d_event_matches_reference():
    d = _pins()
    for row, r, ref in zip(d["ev_in"], d["ev_r"], d["ev_out"]):
        got = O.event("spherical", list(row) + _uniforms("spherical", row, r))
        assert int(got[9]) == int(ref[9]) and int(got[8]) == int(ref[8]), (row, got, ref)
        tau = row[9] * max(row[11] - ref[7], 0.0)
        np.testing.assert_allclose(got[0], ref[0], rtol=1e-12 * (1.0 + 10.0 * tau), atol=1e-300)
        np.testing.assert_allclose(got[7], ref[7], rtol=1e-9, atol=1e-14)
        vol = 4.0 / 3.0 * np.pi * (row[6] ** 3 - row[5] ** 3)
        ulp_w = 64 * np.finfo(float).eps * row[0] / vol
        np.testing.assert_allclose(got[5], ref[5], rtol=1e-9, atol=ulp_w)
        np.testing.assert_allclose(got[6], ref[6], rtol=1e-9, atol=ulp_w / row[9] if row[9] > 1e-10 else ulp_w)
        np.testing.assert_allclose(got[1], ref[1], rtol=1e-9, atol=1e-10)
        np.testing.assert_allclose(got[3], ref[3], rtol=1e-10, atol=1e-12)
    assert set(np.unique(d["ev_out"][:, 9]).astype(int)) == {0, 1, 2}


def test_mg1d_planck_sampler_matches_reference():
    d = _pins()
    lib = O.load()
    edges = np.ascontiguousarray(d["edges"])
    G = len(edges) - 1
    for row, g_ref in zip(d["planck_in"], d["planck_group"]):
        u = np.ascontiguousarray(row[1:6])
        assert lib.orc_planck_group_mg1d(float(row[0]), edges.ctypes.data, G, u.ctypes.data) == g_ref


# ---------------------------------------------------------------- whole steps
def _mg1d_problem():
    ref = np.load(os.path.join(G_DIR, "stats_mg1d.npz"))
    d = {k: (ref[k].item() if ref[k].ndim == 0 else ref[k]) for k in ref.files}
    edges = np.logspace(-2, np.log10(20.0), int(d["G"]) + 1)
    nu = 0.5 * (edges[:-1] + edges[1:])
    return d, edges, nu


def run_oracle_mg1d(seed, d, edges, nu, nthreads=2, conserve="material", Nmax=None):
    """MG_IMC1D.step semantics on the oracle (default conserve_comb_energy=True: the comb
    discrepancy goes into the material).  Returns T, Tr and the per-step relative closure."""
    I, G, cv = int(d["I"]), int(d["G"]), float(d["cv"])
    e = np.linspace(0, float(d["R"]), I + 1)
    o = _sphere(e, G, seed)
    T = np.full(I, float(d["T0"]))
    u = cv * T
    o.init_ic_mg1d(T, int(d["Ntarget"]), edges)
    prev = np.sum(u * o.vol) + np.sum(o.get_bank()["weight"])
    closures = []
    Tr = None
    nmax = int(d["Nmax"]) if Nmax is None else Nmax
    for s in range(int(d["steps"])):
        sig = np.stack([np.clip(2.0 * n ** -3 * T ** -0.5, 0.1, 1e4) for n in nu])
        r = o.transport_mg1d(T, sig, np.full(I, cv), None, s, float(d["dt"]), 1.0, int(d["Ntarget"]),
                             int(d["Nboundary"]), 0, [None, np.array([float(d["Tb"])]), None, None],
                             (False, False, False, False), edges, nthreads=nthreads)
        u = u + r["dep"].reshape(G, I).sum(0) - r["emitted"] / o.vol
        Tr = np.sqrt(np.sqrt(r["si"].reshape(G, I).sum(0) / O.A_RAD / O.C_LIGHT))
        disc = o.comb(nmax, s, per_group=True, conserve_radiation=(conserve == "radiation"))
        if conserve == "material":
            u = u + disc.reshape(G, I).sum(0) / o.vol
        T = u / cv
        total = np.sum(u * o.vol) + np.sum(o.get_bank()["weight"])
        closure = total - prev - r["boundary_emission"] + r["escaped"].sum()
        if conserve != "material":
            closure += disc.sum()
        closures.append(closure / total)
        prev = total
    return T, Tr, closures


@pytest.mark.parametrize("conserve", ["material", "radiation", "none"])
def test_mg1d_oracle_closes_energy(conserve):
    d, edges, nu = _mg1d_problem()
    _, _, closures = run_oracle_mg1d(5, d, edges, nu, conserve=conserve)
    assert max(abs(c) for c in closures) < 1e-12, closures


@pytest.mark.parametrize("nmax", [0, -100000, -100])
def test_mg1d_oracle_comb_threshold_modes(nmax):
    """Nmax = 0 and a threshold above the live count keep every live entry unchanged (no
    discrepancy); a threshold below it combs."""
    d, edges, nu = _mg1d_problem()
    T, _, closures = run_oracle_mg1d(6, d, edges, nu, Nmax=nmax)
    assert max(abs(c) for c in closures) < 1e-12
    assert np.all(np.isfinite(T))


def test_mg1d_matches_reference_statistically():
    from tests.stat_problems import compare_means

    ref = np.load(os.path.join(G_DIR, "stats_mg1d.npz"))
    d, edges, nu = _mg1d_problem()
    seeds = int(ref["seeds"])
    runs = [run_oracle_mg1d(4000 + s, d, edges, nu) for s in range(seeds)]
    Ts = np.array([r[0] for r in runs])
    Trs = np.array([r[1] for r in runs])
    roi = np.ones(int(d["I"]), dtype=bool)
    compare_means(Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds), ref["T_mean"], ref["T_se"], roi)
    compare_means(Trs.mean(0), Trs.std(0, ddof=1) / np.sqrt(seeds), ref["Tr_mean"], ref["Tr_se"], roi)
