"""Multigroup oracle checks (no GPU): the incomplete Planck integral against quadrature,
the Planck group sampler against the reference's own draws (tests/golden/planck.npz),
energy closure, and statistical parity of whole MG steps with MG_IMC2D.step
(tests/golden/stats_mg.npz, recorded with planck_shim standing in for planck_integrals)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

G_DIR = os.path.join(os.path.dirname(__file__), "golden")


def test_planck_fraction_series_matches_quadrature():
    from scipy.integrate import quad

    lib = O.load()
    for x in np.concatenate([np.logspace(-4, 2, 60), [0.999, 1.0, 1.001]]):
        ex = 15 / np.pi ** 4 * quad(lambda t: t ** 3 / np.expm1(t), 0, x, epsabs=0, epsrel=1e-13, limit=200)[0]
        assert abs(lib.orc_planck_F(x) - ex) <= 1e-13 * ex + 1e-300, x


def test_planck_group_sampler_matches_reference():
    d = np.load(os.path.join(G_DIR, "planck.npz"))
    lib = O.load()
    edges = np.ascontiguousarray(d["planck_edges"])
    G = len(edges) - 1
    same = 0
    for row, g_ref in zip(d["planck_in"], d["planck_group"]):
        u = np.ascontiguousarray(row[1:6])
        g = lib.orc_planck_group(float(row[0]), edges.ctypes.data, G, u.ctypes.data)
        same += int(g == g_ref)
    assert same == len(d["planck_group"])


def _mg_problem():
    d = dict(nx=40, L=0.5, G=10, cv=0.3, T0=0.001, dt=0.005, steps=3, Ntarget=4000, Nboundary=2000, Nmax=12000)
    edges = np.logspace(-4, np.log10(20.0), d["G"] + 1)
    nu = 0.5 * (edges[:-1] + edges[1:])
    return d, edges, nu


def _run_oracle_mg(seed, d, edges, nu, nthreads=2):
    nx, G, cv = d["nx"], d["G"], d["cv"]
    x_e = np.linspace(0, d["L"], nx + 1)
    y_e = np.array([0.0, 1.0])
    o = O.Oracle("xy", x_e, y_e, np.diff(x_e), seed, n_groups=G)
    T = np.full(nx, d["T0"])
    e = cv * T
    o.init_ic_mg(T, d["Ntarget"], edges)
    prev = np.sum(e * o.vol) + np.sum(o.get_bank()["weight"])
    out = []
    for s in range(d["steps"]):
        sig = np.stack([np.clip(10.0 * n ** -3 * T ** -0.5, 1e-2, 1e6) for n in nu])
        r = o.transport_mg(T, sig, np.full(nx, cv), None, s, d["dt"], 1.0, d["Ntarget"], d["Nboundary"], 0,
                           [np.array([1.0]), None, None, None], (False, False, True, True), edges, nthreads=nthreads)
        e = e + r["dep"].reshape(G, nx).sum(0) - r["emitted"] / o.vol
        T = e / cv
        disc = o.comb(d["Nmax"], s, per_group=True)
        total = np.sum(e * o.vol) + np.sum(o.get_bank()["weight"])
        closure = total - prev - r["boundary_emission"] + r["escaped"].sum() - r["source_emission"] + disc.sum()
        out.append(closure / total)
        prev = total
    return T, out


def test_multigroup_oracle_closes_energy():
    d, edges, nu = _mg_problem()
    _, closures = _run_oracle_mg(5, d, edges, nu)
    assert max(abs(c) for c in closures) < 1e-12, closures


def test_multigroup_matches_reference_statistically():
    path = os.path.join(G_DIR, "stats_mg.npz")
    if not os.path.exists(path):
        pytest.skip("stats_mg.npz not generated")
    ref = np.load(path)
    d, edges, nu = _mg_problem()
    d["steps"] = int(ref["steps"])
    seeds = int(ref["seeds"])
    Ts = np.array([_run_oracle_mg(3000 + s, d, edges, nu)[0] for s in range(seeds)])
    m, se = Ts.mean(0), Ts.std(0, ddof=1) / np.sqrt(seeds)
    from tests.stat_problems import compare_means

    roi = ref["T_mean"] > 10 * d["T0"]
    compare_means(m, se, ref["T_mean"], ref["T_se"], roi)
