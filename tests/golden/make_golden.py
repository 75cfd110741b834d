"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run where a reference checkout exists, with its path in the RADTRANBOOK_REF environment
variable (required); the fixtures it writes are small .npz files committed with this script.

  events.npz     the reference's own jitted event functions (IMC/IMC1D.py:75 move_particle,
                 :336 move_particle_spherical, IMC/IMC2D.py:739 _move_particle_xy_jit,
                 :826 _move_particle_rz_jit) on random inputs, with the uniforms they drew
                 (Numba's `random` stream is seeded per case and replayed)
  comb.npz       IMC/IMC1D.py:770 comb and IMC/IMC2D.py:1448 _comb on random banks, with the
                 Python `random` draws they consumed
  samplers.npz   IMC/IMC1D.py:203 sample_linear_density, :578 _solve_spherical_cdf,
                 IMC/IMC2D.py:1293 _solve_r_linear_cdf
  sources.npz    per-cell counts and weights of IMC/IMC1D.py:251 emitted_particles and
                 IMC/IMC2D.py:1326 _sample_source_rz_linear (the deterministic part of sampling)
  planck.npz     MG_IMC/MG_IMC2D.py:202 Planck (mixture-of-Gammas) group sampler, with its draws
  cf.npz         Carter-Forest pins: the four event functions of IMC/IMC1D_CarterForest.py and
                 IMC/IMC2D_CarterForest.py with their draws, and the emission samplers' counts,
                 weights and energies
  mg1d.npz       MG_IMC/MG_IMC1D.py pins: stratified emission / IC / fixed-source counts and
                 weights, the per-(cell, group) comb in both energy modes, the spherical event
                 and the Planck sampler, with their draws
  stats_*.npz    multi-seed statistics of whole reference steps (IMC1D.step, IMC2D.step,
                 MG_IMC2D.step and MG_IMC1D.step with planck_shim/ standing in for the
                 external planck_integrals; IMC1D_CarterForest.step, IMC2D_CarterForest.step):
                 per-cell mean and standard error of material and radiation temperature
                 (--stats-only: the slab, RZ and multigroup ones, 32 seeds x 10 steps)
  loops.json     the run_simulation loops of the six step modules on small problems (output
                 times, history shapes, info-history times and key trees) and the info key
                 tree of one step() of each module (--loops-only)

The reference's random numbers cannot be reproduced by a different generator, so whole-step
parity is statistical; the event, comb and sampler fixtures pin the arithmetic exactly.
"""
from __future__ import annotations

import os
import random
import sys
import time
import types

import numpy as np

REF = os.environ.get("RADTRANBOOK_REF", "")
HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference():
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/radtranbook_golden_nbcache")
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    sys.path.insert(0, os.path.join(REF, "IMC"))
    import IMC1D  # noqa: E402
    import IMC2D  # noqa: E402
    return IMC1D, IMC2D


def nb_helpers():
    from numba import njit

    @njit
    def seed_py(s):
        random.seed(s)

    @njit
    def seed_np(s):
        np.random.seed(s)

    @njit
    def draw_py(k):
        out = np.empty(k)
        for i in range(k):
            out[i] = random.random()
        return out

    @njit
    def draw_np(k):
        return np.random.uniform(0.0, 1.0, k)

    return seed_py, seed_np, draw_py, draw_np


def gen_events(IMC1D, IMC2D, n=400, seed=20261203):
    """Inputs use the oracle's event layout: w d1 d2 p1 p2 lo1 hi1 lo2 hi2 sa ss dcen."""
    seed_py, _, draw_py, _ = nb_helpers()
    rng = np.random.default_rng(seed)
    out = {}

    def sig():
        k = rng.integers(0, 5)
        if k == 0:
            return 0.0
        return float(10 ** rng.uniform(-3, 7))

    # ---- slab ----
    rows, draws, res = [], [], []
    for q in range(n):
        xl = rng.uniform(0, 1); dx = 10 ** rng.uniform(-3, -1); xr = xl + dx
        x = xl + dx * rng.choice([0.0, 1.0, rng.uniform()], p=[0.1, 0.1, 0.8])
        mu = rng.uniform(-1, 1)
        if x == xl and mu < 0: mu = -mu
        if x == xr and mu > 0: mu = -mu
        w = 10 ** rng.uniform(-3, 1); sa = sig(); ss = sig(); dcen = 10 ** rng.uniform(-4, 0)
        seed_py(1000 + q); r = draw_py(4)
        seed_py(1000 + q)
        o = IMC1D.move_particle(w, mu, x, xl, xr, sa, ss, dcen)
        rows.append([w, mu, 0, x, 0, xl, xr, 0, 1, sa, ss, dcen]); draws.append(r)
        # (w, mu, x, new_loc, dep_w, dep_i, dcen, evt)
        res.append([o[0], o[1], 0, o[2], 0, o[4], o[5], o[6], {1: 1, -1: 2, 0: 0}[o[3]], {1: 1, 2: 2, 3: 0}[o[7]]])
    out["slab_in"], out["slab_r"], out["slab_out"] = np.array(rows), np.array(draws), np.array(res)

    # ---- sphere ----
    rows, draws, res = [], [], []
    for q in range(n):
        r0 = rng.choice([0.0, 10 ** rng.uniform(-2, 0)], p=[0.2, 0.8]); dr = 10 ** rng.uniform(-3, -1); r1 = r0 + dr
        x = r0 + dr * rng.uniform(0.01, 0.99)
        mu = rng.uniform(-1, 1)
        w = 10 ** rng.uniform(-3, 1); sa = sig(); ss = sig(); dcen = 10 ** rng.uniform(-4, 0)
        seed_py(5000 + q); r = draw_py(4)
        seed_py(5000 + q)
        o = IMC1D.move_particle_spherical(w, mu, x, r0, r1, sa, ss, dcen)
        rows.append([w, mu, 0, x, 0, r0, r1, 0, 1, sa, ss, dcen]); draws.append(r)
        res.append([o[0], o[1], 0, o[2], 0, o[4], o[5], o[6], {1: 1, -1: 2, 0: 0}[o[3]], {1: 1, 2: 2, 3: 0}[o[7]]])
    out["sphere_in"], out["sphere_r"], out["sphere_out"] = np.array(rows), np.array(draws), np.array(res)

    # ---- xy and rz ----
    for geo in ("xy", "rz"):
        rows, draws, res = [], [], []
        e1 = np.concatenate([[0.0], np.cumsum(10 ** rng.uniform(-2, -0.5, 12))])
        e2 = np.concatenate([[0.0], np.cumsum(10 ** rng.uniform(-2, -0.5, 12))])
        for q in range(n):
            i = int(rng.integers(0, 12)); j = int(rng.integers(0, 12))
            a1, b1, a2, b2 = e1[i], e1[i + 1], e2[j], e2[j + 1]
            p1 = a1 + (b1 - a1) * rng.uniform(0.02, 0.98)
            p2 = a2 + (b2 - a2) * rng.uniform(0.02, 0.98)
            if geo == "xy":
                uz = rng.uniform(-1, 1); ph = rng.uniform(0, 2 * np.pi); rxy = np.sqrt(1 - uz * uz)
                d1, d2 = rxy * np.cos(ph), rxy * np.sin(ph)
            else:
                d1, d2 = rng.uniform(-1, 1), rng.uniform(-1, 1)
            w = 10 ** rng.uniform(-3, 1); sa = sig(); ss = sig(); dcen = 10 ** rng.uniform(-4, 0)
            seed_py(9000 + q); r = draw_py(4)
            seed_py(9000 + q)
            fn = IMC2D._move_particle_xy_jit if geo == "xy" else IMC2D._move_particle_rz_jit
            o = fn(w, d1, d2, p1, p2, i, j, e1, e2, sa, ss, dcen)
            rows.append([w, d1, d2, p1, p2, a1, b1, a2, b2, sa, ss, dcen]); draws.append(r)
            # (w, d1, d2, p1, p2, crossed, dep_w, dep_i, dcen, evt)
            res.append([o[0], o[1], o[2], o[3], o[4], o[6], o[7], o[8], o[5], o[9]])
        out[f"{geo}_in"], out[f"{geo}_r"], out[f"{geo}_out"] = np.array(rows), np.array(draws), np.array(res)
    return out


def gen_comb(IMC1D, IMC2D, seed=7):
    rng = np.random.default_rng(seed)
    out = {}
    n, I = 3000, 40
    w = rng.gamma(2.0, 1.0, n) * (rng.uniform(size=n) > 0.05)
    cell = rng.integers(0, I, n)
    mu = rng.uniform(-1, 1, n); t = rng.uniform(0, 0.01, n); x = rng.uniform(0, 1, n)
    random.seed(99)
    xi = np.array([random.random() for _ in range(int(np.sum(w > 0)))])
    random.seed(99)
    nw, nc, nmu, nt, nx, disc = IMC1D.comb(w.copy(), cell.copy(), mu.copy(), t.copy(), x.copy(), 2500, I)
    out.update(c1_w=w, c1_cell=cell, c1_mu=mu, c1_t=t, c1_x=x, c1_xi=xi, c1_nmax=2500,
               c1_out_w=nw, c1_out_cell=nc, c1_out_mu=nmu, c1_out_x=nx, c1_disc=disc)
    nx2, ny2 = 6, 5
    w = rng.gamma(2.0, 1.0, n) * (rng.uniform(size=n) > 0.05)
    ci = rng.integers(0, nx2, n); cj = rng.integers(0, ny2, n)
    d1 = rng.uniform(-1, 1, n); d2 = rng.uniform(-1, 1, n); t = np.zeros(n)
    p1 = rng.uniform(size=n); p2 = rng.uniform(size=n)
    random.seed(123)
    xi = np.array([random.random() for _ in range(int(np.sum(w > 0)))])
    random.seed(123)
    r = IMC2D._comb(w.copy(), ci.copy(), cj.copy(), d1.copy(), d2.copy(), t.copy(), p1.copy(), p2.copy(), 2000, nx2, ny2)
    out.update(c2_w=w, c2_ci=ci, c2_cj=cj, c2_d1=d1, c2_d2=d2, c2_p1=p1, c2_p2=p2, c2_xi=xi, c2_nmax=2000,
               c2_nx=nx2, c2_ny=ny2, c2_out_w=r[0], c2_out_ci=r[1], c2_out_cj=r[2], c2_out_p1=r[6], c2_disc=r[8])
    return out


def gen_samplers(IMC1D, IMC2D, seed=11):
    _, seed_np, _, draw_np = nb_helpers()
    rng = np.random.default_rng(seed)
    out = {}
    rows, res = [], []
    for q in range(200):
        dx = 10 ** rng.uniform(-3, -1); T = 10 ** rng.uniform(-2, 0)
        s = rng.uniform(-3, 3) * 2 * T / dx ** 2
        seed_np(700 + q); xi = draw_np(5)
        seed_np(700 + q); xs = IMC1D.sample_linear_density(dx, s, T, 5)
        for k in range(5):
            rows.append([dx, s, T, xi[k]]); res.append(xs[k])
    out["slab_linear_in"], out["slab_linear_out"] = np.array(rows), np.array(res)
    rows, res = [], []
    for q in range(300):
        r0 = rng.choice([0.0, 10 ** rng.uniform(-2, 0)]); r1 = r0 + 10 ** rng.uniform(-3, 0)
        a = 10 ** rng.uniform(-4, 0); M = rng.uniform(-1, 1) * a / (r1 - r0); xi = rng.uniform()
        rows.append([r0, r1, a, M, xi])
        res.append([IMC1D._solve_spherical_cdf(r0, r1, a, M, xi), IMC2D._solve_r_linear_cdf(r0, r1, a, M, xi)])
    out["cdf_in"], out["cdf_out"] = np.array(rows), np.array(res)
    return out


def gen_sources(IMC1D, IMC2D, seed=13):
    rng = np.random.default_rng(seed)
    out = {}
    I = 50
    mesh = np.array([[i * 0.01, (i + 1) * 0.01] for i in range(I)])
    T = 10 ** rng.uniform(-1.5, 0, I)
    sa = 10 ** rng.uniform(0, 3, I)
    p = IMC1D.emitted_particles(20000, T, 0.01, mesh, sa)
    out.update(e1d_T=T, e1d_sa=sa, e1d_N=20000, e1d_dt=0.01,
               e1d_counts=np.bincount(p[4], minlength=I), e1d_w=np.array([p[0][p[4] == i][0] for i in range(I)]),
               e1d_E=p[5])
    nx, ny = 8, 10
    r_e = np.linspace(0, 2, nx + 1); z_e = np.linspace(0, 3, ny + 1)
    T2 = 10 ** rng.uniform(-1.5, 0, (nx, ny))
    src = 10 ** rng.uniform(-2, 2, (nx, ny))
    np.random.seed(5); random.seed(5)
    r = IMC2D._sample_source_rz_linear(30000, src, T2, 0.01, r_e, z_e)
    flat = r[6] + nx * r[7]
    counts = np.bincount(flat, minlength=nx * ny)
    wc = np.zeros(nx * ny)
    for c in range(nx * ny):
        if counts[c]:
            wc[c] = r[0][flat == c][0]
    out.update(rz_T=T2, rz_src=src, rz_N=30000, rz_dt=0.01, rz_r_edges=r_e, rz_z_edges=z_e,
               rz_counts=counts, rz_w=wc)
    return out


def run_stats_slab(IMC1D, seeds=32, steps=10):
    I = 100
    mesh = np.array([[i * 0.002, (i + 1) * 0.002] for i in range(I)])
    cv = 0.3
    kw = dict(Ntarget=2000, Nboundary=2000, Nsource=0, NMax=8000, T_boundary=(1.0, 0.0), dt=0.01, mesh=mesh,
              sigma_a_func=lambda T: 300.0 * T ** -3, inv_eos=lambda e: e / cv, cv=lambda T: cv + 0 * T,
              source=np.zeros(I))
    seed_py, seed_np, _, _ = nb_helpers()
    Ts, Trs = [], []
    for s in range(seeds):
        np.random.seed(s); random.seed(s); seed_py(s); seed_np(s)
        st = IMC1D.init_simulation(2000, np.full(I, 0.001), np.full(I, 0.001), mesh, lambda T: cv * T,
                                   lambda e: e / cv)
        for _ in range(steps):
            st, info = IMC1D.step(st, kw["Ntarget"], kw["Nboundary"], 0, kw["NMax"], kw["T_boundary"], kw["dt"], mesh,
                                  kw["sigma_a_func"], kw["inv_eos"], kw["cv"], kw["source"])
        Ts.append(st.temperature.copy()); Trs.append(st.radiation_temperature.copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    return dict(T_mean=Ts.mean(0), T_se=Ts.std(0, ddof=1) / np.sqrt(seeds), Tr_mean=Trs.mean(0),
                Tr_se=Trs.std(0, ddof=1) / np.sqrt(seeds), seeds=seeds, steps=steps, Ntarget=2000, Nboundary=2000,
                NMax=8000, dt=0.01)


def run_stats_rz(IMC2D, seeds=32, steps=10):
    nr, nz = 30, 105
    r_e = np.linspace(0, 2, nr + 1); z_e = np.linspace(0, 7, nz + 1)
    rc = 0.5 * (r_e[:-1] + r_e[1:]); zc = 0.5 * (z_e[:-1] + z_e[1:])
    R, Z = np.meshgrid(rc, zc, indexing="ij")
    thin = (((R < 0.5) & (Z <= 3.0)) | ((R >= 0.5) & (R < 1.5) & (Z >= 2.5) & (Z <= 3.0))
            | ((R >= 1.0) & (R <= 1.5) & (Z >= 3.0) & (Z <= 4.0)) | ((R >= 0.5) & (R < 1.5) & (Z >= 4.0) & (Z <= 4.5))
            | ((R < 0.5) & (Z >= 4.0)))
    sig = np.where(thin, 0.2, 2000.0); cvg = np.where(thin, 0.001, 0.5)
    bsf = lambda r, z, side: 0.5 if (side == "zmin" and r < 0.5) else 0.0  # noqa: E731
    seed_py, seed_np, _, _ = nb_helpers()
    Ts, Trs = [], []
    for s in range(seeds):
        np.random.seed(s); random.seed(s); seed_py(s); seed_np(s)
        st = IMC2D.init_simulation(6000, np.full((nr, nz), 0.05), np.full((nr, nz), 0.05), r_e, z_e,
                                   lambda T: cvg * T, lambda e: e / cvg, geometry="rz")
        for _ in range(steps):
            st, info = IMC2D.step(st, 6000, 3000, 0, 30000, (0.0, 0.0, 0.0, 0.0), 0.01, r_e, z_e,
                                  lambda T: sig.copy(), lambda e: e / cvg, lambda T: cvg.copy(), np.zeros((nr, nz)),
                                  reflect=(True, False, False, False), geometry="rz", boundary_source_func=bsf)
        Ts.append(st.temperature.copy()); Trs.append(st.radiation_temperature.copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    return dict(T_mean=Ts.mean(0), T_se=Ts.std(0, ddof=1) / np.sqrt(seeds), Tr_mean=Trs.mean(0),
                Tr_se=Trs.std(0, ddof=1) / np.sqrt(seeds), seeds=seeds, steps=steps, nr=nr, nz=nz)


MG = dict(nx=40, L=0.5, G=10, cv=0.3, T0=0.001, dt=0.005, steps=10, Ntarget=4000, Nboundary=2000, Nmax=12000)


def mg_setup():
    edges = np.logspace(-4, np.log10(20.0), MG["G"] + 1)
    nu = 0.5 * (edges[:-1] + edges[1:])
    funcs = [(lambda T, n=n: np.clip(10.0 * n ** -3 * np.power(T, -0.5), 1e-2, 1e6)) for n in nu]
    return edges, nu, funcs


def load_reference_mg():
    sys.path.insert(0, os.path.join(HERE, "planck_shim"))
    sys.path.insert(0, os.path.join(REF, "MG_IMC"))
    import MG_IMC2D  # noqa: E402
    assert MG_IMC2D._PLANCK_AVAILABLE, "planck_integrals stand-in not found"
    return MG_IMC2D


def gen_planck_sampler(MG_IMC2D, n=3000, seed=17):
    _, seed_np, _, draw_np = nb_helpers()
    rng = np.random.default_rng(seed)
    edges = np.logspace(-4, np.log10(20.0), 11)
    rows, res = [], []
    for q in range(40):
        T = 10 ** rng.uniform(-3, 0.5)
        seed_np(300 + q)
        u = draw_np(5 * 50).reshape(50, 5)
        seed_np(300 + q)
        _, g = MG_IMC2D._sample_planck_spectrum_mixture_of_gammas_jit(50, T, edges[:-1], edges[1:],
                                                                       MG_IMC2D._PLANCK_MIXTURE_CDF)
        for k in range(50):
            rows.append([T] + list(u[k])); res.append(g[k])
    return dict(planck_in=np.array(rows), planck_group=np.array(res), planck_edges=edges)


def run_stats_mg(MG_IMC2D, seeds=32):
    edges, nu, funcs = mg_setup()
    nx = MG["nx"]
    x_e = np.linspace(0, MG["L"], nx + 1); y_e = np.array([0.0, 1.0])
    cv = MG["cv"]
    seed_py, seed_np, _, _ = nb_helpers()
    Ts, Trs = [], []
    for s in range(seeds):
        np.random.seed(s); random.seed(s); seed_py(s); seed_np(s)
        st = MG_IMC2D.init_simulation(MG["Ntarget"], np.full((nx, 1), MG["T0"]), np.full((nx, 1), MG["T0"]), x_e, y_e,
                                      edges, lambda T: cv * T, lambda e: e / cv, geometry="xy")
        for _ in range(MG["steps"]):
            st, info = MG_IMC2D.step(st, MG["Ntarget"], MG["Nboundary"], 0, MG["Nmax"], (1.0, 0.0, 0.0, 0.0), MG["dt"],
                                     x_e, y_e, edges, funcs, lambda e: e / cv, lambda T: cv + 0 * T,
                                     np.zeros((nx, 1)), reflect=(False, False, True, True), geometry="xy")
        Ts.append(st.temperature[:, 0].copy()); Trs.append(st.radiation_temperature[:, 0].copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    return dict(T_mean=Ts.mean(0), T_se=Ts.std(0, ddof=1) / np.sqrt(seeds), Tr_mean=Trs.mean(0),
                Tr_se=Trs.std(0, ddof=1) / np.sqrt(seeds), seeds=seeds, **MG)


MG1 = dict(I=30, R=1.0, G=4, cv=0.2, T0=0.05, Tb=1.0, dt=0.01, steps=4, Ntarget=3000, Nboundary=3000, Nmax=8000)


def mg1d_setup():
    edges = np.logspace(-2, np.log10(20.0), MG1["G"] + 1)
    nu = 0.5 * (edges[:-1] + edges[1:])
    funcs = [(lambda T, n=n: np.clip(2.0 * n ** -3 * np.power(T, -0.5), 0.1, 1e4)) for n in nu]
    return edges, nu, funcs


def load_reference_mg1d():
    sys.path.insert(0, os.path.join(HERE, "planck_shim"))
    sys.path.insert(0, os.path.join(REF, "MG_IMC"))
    import MG_IMC1D  # noqa: E402
    assert MG_IMC1D._PLANCK_AVAILABLE, "planck_integrals stand-in not found"
    return MG_IMC1D


def gen_mg1d_pins(M, seed=23):
    """MG_IMC/MG_IMC1D.py pins: stratified emission / IC / fixed-source counts and weights
    (:514-743), the per-(cell, group) comb (:746-847) with its uniforms, the spherical event
    (:276-364) and the Planck sampler (:144-195) with their draws."""
    seed_py, seed_np, draw_py, draw_np = nb_helpers()
    rng = np.random.default_rng(seed)
    I, G = 20, 4
    edges = np.logspace(-2, np.log10(20.0), G + 1)
    out = {"edges": edges}
    meshes, Ts, sas, Ns, dts, cnt_e, w_e, emit = [], [], [], [], [], [], [], []
    srcs, cnt_s, w_s, Ns_s, cnt_ic, w_ic, Ns_ic = [], [], [], [], [], [], []
    for q in range(8):
        e = np.concatenate([[0.0], np.cumsum(10 ** rng.uniform(-2, -0.5, I))])
        mesh = np.stack([e[:-1], e[1:]], axis=1)
        T = 10 ** rng.uniform(-1.5, 0.3, I)
        saf = 10 ** rng.uniform(-1, 3, (G, I))
        N = int(rng.integers(500, 5000)); dt = float(10 ** rng.uniform(-3, -1))
        np.random.seed(q)
        w, mu, t, r, c, g, ebg = M._emitted_particles_spherical_mg(N, T, dt, mesh, saf, edges)
        b = c + g.astype(np.int64) * I
        cnt = np.bincount(b, minlength=G * I)
        wb = np.zeros(G * I); wb[b] = w
        meshes.append(e); Ts.append(T); sas.append(saf); Ns.append(N); dts.append(dt)
        cnt_e.append(cnt); w_e.append(wb); emit.append(ebg)
        src = 10 ** rng.uniform(-2, 1, (G, I)) * (rng.uniform(size=(G, I)) > 0.3)
        Nsrc = int(rng.integers(200, 3000))
        w, mu, t, r, c, g = M._sample_source_spherical_mg(Nsrc, src, dt, mesh, edges, T)
        b = c + g.astype(np.int64) * I
        cnt = np.bincount(b, minlength=G * I)
        wb = np.zeros(G * I); wb[b] = w
        srcs.append(src); Ns_s.append(Nsrc); cnt_s.append(cnt); w_s.append(wb)
        Nic = int(rng.integers(500, 5000))
        Tr = T * (rng.uniform(size=I) > 0.2)
        w, mu, t, r, c, g = M._equilibrium_sample_spherical_mg(Nic, Tr, mesh, edges)
        cnt = np.bincount(c, minlength=I)
        wb = np.zeros(I); wb[c] = w
        Ns_ic.append(Nic); cnt_ic.append(cnt); w_ic.append(wb)
        Ts[-1] = T
        out.setdefault("ic_Tr", []).append(Tr)
    out.update(mesh=np.array(meshes), T=np.array(Ts), saf=np.array(sas), N=np.array(Ns), dt=np.array(dts),
               emit_counts=np.array(cnt_e), emit_w=np.array(w_e), emit_by_group=np.array(emit),
               src=np.array(srcs), src_N=np.array(Ns_s), src_counts=np.array(cnt_s), src_w=np.array(w_s),
               ic_N=np.array(Ns_ic), ic_counts=np.array(cnt_ic), ic_w=np.array(w_ic))
    out["ic_Tr"] = np.array(out["ic_Tr"])
    # ---- comb, both energy modes ----
    for mode in ("none", "radiation"):
        n = 3000
        w = 10 ** rng.uniform(-3, 0, n) * (rng.uniform(size=n) > 0.1)
        c = rng.integers(0, I, n); g = rng.integers(0, G, n).astype(np.int32)
        mu = rng.uniform(-1, 1, n); t = rng.uniform(0, 0.01, n); r = rng.uniform(0, 1, n)
        nmax = 2500
        np.random.seed(77)
        xi = np.random.random(int(np.sum(w > 0)))
        np.random.seed(77)
        nw, nc, ng, nm, nt, npos, disc = M._comb_mg_1d(w, c, g, mu, t, r, nmax, I, G,
                                                        conserve_rad_energy=(mode == "radiation"))
        out.update({f"comb_{mode}_in": np.stack([w, c, g, mu, t, r], axis=1), f"comb_{mode}_xi": xi,
                    f"comb_{mode}_out": np.stack([nw, nc, ng, nm, npos], axis=1), f"comb_{mode}_disc": disc})
    out["comb_nmax"] = 2500
    # ---- spherical event of MG_IMC1D ----
    rows, draws, res = [], [], []
    for q in range(300):
        r0 = rng.choice([0.0, 10 ** rng.uniform(-2, 0)], p=[0.2, 0.8]); dr = 10 ** rng.uniform(-3, -1); r1 = r0 + dr
        x = r0 + dr * rng.uniform(0.01, 0.99)
        mu = rng.uniform(-1, 1)
        w = 10 ** rng.uniform(-3, 1)
        sa = 0.0 if rng.uniform() < 0.2 else float(10 ** rng.uniform(-3, 7))
        ss = 0.0 if rng.uniform() < 0.2 else float(10 ** rng.uniform(-3, 7))
        dcen = 10 ** rng.uniform(-4, 0)
        seed_py(7000 + q); rr = draw_py(4)
        seed_py(7000 + q)
        o = M._move_particle_spherical(w, mu, x, r0, r1, sa, ss, dcen)
        rows.append([w, mu, 0, x, 0, r0, r1, 0, 1, sa, ss, dcen]); draws.append(rr)
        res.append([o[0], o[1], 0, o[2], 0, o[4], o[5], o[6], {1: 1, -1: 2, 0: 0}[o[3]], {1: 1, 2: 2, 3: 0}[o[7]]])
    out["ev_in"], out["ev_r"], out["ev_out"] = np.array(rows), np.array(draws), np.array(res)
    # ---- Planck sampler of MG_IMC1D ----
    prow, pres = [], []
    for q in range(30):
        T = 10 ** rng.uniform(-2, 0.5)
        seed_np(400 + q)
        u = draw_np(5 * 40).reshape(40, 5)
        seed_np(400 + q)
        _, gg = M._sample_planck_spectrum_mg_jit(40, T, edges[:-1], edges[1:], M._PLANCK_MIXTURE_CDF)
        for k in range(40):
            prow.append([T] + list(u[k])); pres.append(gg[k])
    out["planck_in"], out["planck_group"] = np.array(prow), np.array(pres)
    return out


def run_stats_mg1d(M, seeds=32):
    edges, nu, funcs = mg1d_setup()
    I, R, cv = MG1["I"], MG1["R"], MG1["cv"]
    e = np.linspace(0, R, I + 1)
    mesh = np.stack([e[:-1], e[1:]], axis=1)
    seed_py, seed_np, _, _ = nb_helpers()
    Ts, Trs = [], []
    for s in range(seeds):
        np.random.seed(s); random.seed(s); seed_py(s); seed_np(s)
        st = M.init_simulation(MG1["Ntarget"], np.full(I, MG1["T0"]), np.full(I, MG1["T0"]), mesh, edges,
                               lambda T: cv * T, lambda u: u / cv)
        for _ in range(MG1["steps"]):
            st, info = M.step(st, MG1["Ntarget"], MG1["Nboundary"], 0, MG1["Nmax"], (0.0, MG1["Tb"]), MG1["dt"], mesh,
                              edges, funcs, lambda u: u / cv, lambda T: cv + 0 * T, np.zeros(I))
        Ts.append(st.temperature.copy()); Trs.append(st.radiation_temperature.copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    return dict(T_mean=Ts.mean(0), T_se=Ts.std(0, ddof=1) / np.sqrt(seeds), Tr_mean=Trs.mean(0),
                Tr_se=Trs.std(0, ddof=1) / np.sqrt(seeds), seeds=seeds, **MG1)


def main_mg1d():
    import contextlib
    import io

    t0 = time.time()
    M = load_reference_mg1d()
    with contextlib.redirect_stdout(io.StringIO()):
        pins = gen_mg1d_pins(M)
    np.savez_compressed(os.path.join(HERE, "mg1d.npz"), **pins)
    print(f"MG 1-D pins written ({time.time() - t0:.1f} s)")
    if "--no-stats" not in sys.argv:
        with contextlib.redirect_stdout(io.StringIO()):
            st = run_stats_mg1d(M)
        np.savez_compressed(os.path.join(HERE, "stats_mg1d.npz"), **st)
        print(f"MG 1-D statistics written ({time.time() - t0:.1f} s)")


def load_reference_cf():
    sys.path.insert(0, os.path.join(REF, "IMC"))
    import IMC1D_CarterForest as CF1  # noqa: E402
    import IMC2D_CarterForest as CF2  # noqa: E402
    return CF1, CF2


def gen_cf_pins(CF1, CF2, n=300, seed=29):
    """Carter-Forest pins: the four event functions (IMC/IMC1D_CarterForest.py:63 move_particle_cf,
    :614 move_particle_spherical_cf, IMC/IMC2D_CarterForest.py:102 _move_particle_xy_cf_jit,
    :216 _move_particle_rz_cf_jit) with the draws they consumed, and the emission samplers'
    per-cell counts, weights and energies (:442 emitted_particles, :889
    emitted_particles_spherical, IMC/IMC2D_CarterForest.py:876 _sample_internal_emission_cf)."""
    seed_py, seed_np, draw_py, _ = nb_helpers()
    rng = np.random.default_rng(seed)
    out = {}

    def sig():
        k = rng.integers(0, 5)
        return 0.0 if k == 0 else float(10 ** rng.uniform(-3, 7))

    def bet():
        return 1e-17 if rng.uniform() < 0.15 else float(10 ** rng.uniform(-4, 1))

    def fpath():
        return float(10 ** rng.uniform(-1, 1)) if rng.uniform() < 0.2 else 0.0

    rows, draws, res = [], [], []
    for q in range(n):  # slab
        xl = rng.uniform(0, 1); dx = 10 ** rng.uniform(-3, -1); xr = xl + dx
        x = xl + dx * rng.uniform(0.02, 0.98); mu = rng.uniform(-1, 1)
        w = 10 ** rng.uniform(-3, 1); sa = sig(); b = bet(); dcen = 10 ** rng.uniform(-4, 0); fp = fpath()
        seed_py(11000 + q); r = draw_py(6); seed_py(11000 + q)
        o = CF1.move_particle_cf(w, mu, x, 0.0, xl, xr, sa, b, dcen, fp)
        rows.append([w, mu, 0, x, 0, xl, xr, 0, 1, sa, b, dcen, fp]); draws.append(r)
        res.append([o[0], o[1], 0, o[2], 0, o[5], o[6], o[7], {1: 1, -1: 2, 0: 0}[o[4]], {1: 1, 2: 2, 3: 0, 4: 4}[o[8]]])
    out["slab_in"], out["slab_r"], out["slab_out"] = np.array(rows), np.array(draws), np.array(res)
    rows, draws, res = [], [], []
    for q in range(n):  # sphere
        r0 = rng.choice([0.0, 10 ** rng.uniform(-2, 0)], p=[0.2, 0.8]); dr = 10 ** rng.uniform(-3, -1); r1 = r0 + dr
        x = r0 + dr * rng.uniform(0.02, 0.98); mu = rng.uniform(-1, 1)
        w = 10 ** rng.uniform(-3, 1); sa = sig(); b = bet(); dcen = 10 ** rng.uniform(-4, 0); fp = fpath()
        seed_py(12000 + q); r = draw_py(6); seed_py(12000 + q)
        o = CF1.move_particle_spherical_cf(w, mu, x, 0.0, r0, r1, sa, b, dcen, fp)
        rows.append([w, mu, 0, x, 0, r0, r1, 0, 1, sa, b, dcen, fp]); draws.append(r)
        res.append([o[0], o[1], 0, o[2], 0, o[5], o[6], o[7], {1: 1, -1: 2, 0: 0}[o[4]], {1: 1, 2: 2, 3: 0, 4: 4}[o[8]]])
    out["sphere_in"], out["sphere_r"], out["sphere_out"] = np.array(rows), np.array(draws), np.array(res)
    for geo in ("xy", "rz"):
        rows, draws, res = [], [], []
        e1 = np.concatenate([[0.0], np.cumsum(10 ** rng.uniform(-2, -0.5, 12))])
        e2 = np.concatenate([[0.0], np.cumsum(10 ** rng.uniform(-2, -0.5, 12))])
        for q in range(n):
            i = int(rng.integers(0, 12)); j = int(rng.integers(0, 12))
            a1, b1, a2, b2 = e1[i], e1[i + 1], e2[j], e2[j + 1]
            p1 = a1 + (b1 - a1) * rng.uniform(0.02, 0.98); p2 = a2 + (b2 - a2) * rng.uniform(0.02, 0.98)
            if geo == "xy":
                uz = rng.uniform(-1, 1); ph = rng.uniform(0, 2 * np.pi); rxy = np.sqrt(1 - uz * uz)
                d1, d2 = rxy * np.cos(ph), rxy * np.sin(ph)
            else:
                d1, d2 = rng.uniform(-1, 1), rng.uniform(-1, 1)
            w = 10 ** rng.uniform(-3, 1); sa = sig(); b = bet(); dcen = 10 ** rng.uniform(-4, 0); fp = fpath()
            seed_py(13000 + q); r = draw_py(6); seed_py(13000 + q)
            fn = CF2._move_particle_xy_cf_jit if geo == "xy" else CF2._move_particle_rz_cf_jit
            o = fn(w, d1, d2, p1, p2, i, j, e1, e2, sa, b, dcen, 0.0, fp)
            rows.append([w, d1, d2, p1, p2, a1, b1, a2, b2, sa, b, dcen, fp]); draws.append(r)
            # (w, d1, d2, p1, p2, time, crossed, dep_w, dep_i, dcen, evt)
            res.append([o[0], o[1], o[2], o[3], o[4], o[7], o[8], o[9], o[6], o[10]])
        out[f"{geo}_in"], out[f"{geo}_r"], out[f"{geo}_out"] = np.array(rows), np.array(draws), np.array(res)
    # ---- emission samplers ----
    I = 25
    for geo in ("slab", "spherical"):
        Ts, sas, cvs, Ns, cnts, ws, Es = [], [], [], [], [], [], []
        for q in range(6):
            T = 10 ** rng.uniform(-1.5, 0.3, I); sa = 10 ** rng.uniform(-1, 3, I); cv = 10 ** rng.uniform(-2, 0, I)
            beta = 4.0 * 0.01372 * T ** 3 / cv
            N = int(rng.integers(500, 5000)); dt = 0.01
            e = np.linspace(0.0, 1.0, I + 1)
            mesh = np.stack([e[:-1], e[1:]], axis=1)
            seed_np(500 + q); seed_py(500 + q)
            fn = CF1.emitted_particles if geo == "slab" else CF1.emitted_particles_spherical
            w, mu, t, x, c, E = fn(N, T, dt, mesh, sa, beta)
            cnt = np.bincount(c, minlength=I); wc = np.zeros(I); wc[c] = w
            Ts.append(T); sas.append(sa); cvs.append(cv); Ns.append(N); cnts.append(cnt); ws.append(wc); Es.append(E)
        out.update({f"em_{geo}_T": np.array(Ts), f"em_{geo}_sa": np.array(sas), f"em_{geo}_cv": np.array(cvs),
                    f"em_{geo}_N": np.array(Ns), f"em_{geo}_counts": np.array(cnts), f"em_{geo}_w": np.array(ws),
                    f"em_{geo}_E": np.array(Es)})
    nx, ny = 10, 8
    e1 = np.linspace(0, 1, nx + 1); e2 = np.linspace(0, 2, ny + 1)
    vol = np.diff(e1)[:, None] * np.diff(e2)[None, :]
    Ts, sas, cvs, Ns, cnts, ws, Es = [], [], [], [], [], [], []
    for q in range(6):
        T = 10 ** rng.uniform(-1.5, 0.3, (nx, ny)); sa = 10 ** rng.uniform(-1, 3, (nx, ny))
        cv = 10 ** rng.uniform(-2, 0, (nx, ny))
        beta = 4.0 * 0.01372 * np.maximum(T, 1e-12) ** 3 / cv
        N = int(rng.integers(500, 5000))
        seed_np(600 + q); seed_py(600 + q)
        smp, E = CF2._sample_internal_emission_cf(N, T, 0.01, e1, e2, vol, sa, beta, "xy", False)
        w, d1, d2, t, p1, p2, ci, cj = smp
        flat = ci + nx * cj
        cnt = np.bincount(flat, minlength=nx * ny); wc = np.zeros(nx * ny); wc[flat] = w
        Ts.append(T); sas.append(sa); cvs.append(cv); Ns.append(N); cnts.append(cnt); ws.append(wc); Es.append(E)
    out.update(em_xy_T=np.array(Ts), em_xy_sa=np.array(sas), em_xy_cv=np.array(cvs), em_xy_N=np.array(Ns),
               em_xy_counts=np.array(cnts), em_xy_w=np.array(ws), em_xy_E=np.array(Es))
    return out


CFX = dict(nx=30, ny=3, L=0.3, cv=0.3, T0=0.05, dt=0.01, steps=3, Ntarget=3000, Nboundary=3000, Nmax=12000)


def run_stats_cf(CF1, CF2, seeds=32):
    """Carter-Forest whole steps: a slab Marshak wave (sigma = 100 T^-3, 10 steps) through
    IMC1D_CarterForest.step, and a 30 x 3 XY Marshak wave through IMC2D_CarterForest.step."""
    seed_py, seed_np, _, _ = nb_helpers()
    I = 100
    mesh = np.array([[i * 0.002, (i + 1) * 0.002] for i in range(I)])
    cv = 0.3
    Ts, Trs = [], []
    for s in range(seeds):
        np.random.seed(s); random.seed(s); seed_py(s); seed_np(s)
        st = CF1.init_simulation(2000, np.full(I, 0.001), np.full(I, 0.001), mesh, lambda T: cv * T, lambda e: e / cv)
        for _ in range(10):
            st, info = CF1.step(st, 2000, 2000, 0, 8000, (1.0, 0.0), 0.01, mesh, lambda T: 100.0 * T ** -3,
                                lambda e: e / cv, lambda T: cv + 0 * T, np.zeros(I))
        Ts.append(st.temperature.copy()); Trs.append(st.radiation_temperature.copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    slab = dict(T_mean=Ts.mean(0), T_se=Ts.std(0, ddof=1) / np.sqrt(seeds), Tr_mean=Trs.mean(0),
                Tr_se=Trs.std(0, ddof=1) / np.sqrt(seeds), seeds=seeds, steps=10, A=100.0)
    nx, ny = CFX["nx"], CFX["ny"]
    x_e = np.linspace(0, CFX["L"], nx + 1); y_e = np.linspace(0, 0.1, ny + 1)
    cvx = CFX["cv"]
    Ts, Trs = [], []
    for s in range(seeds):
        np.random.seed(s); random.seed(s); seed_py(s); seed_np(s)
        st = CF2.init_simulation(CFX["Ntarget"], np.full((nx, ny), CFX["T0"]), np.full((nx, ny), CFX["T0"]), x_e, y_e,
                                 lambda T: cvx * T, lambda e: e / cvx, geometry="xy")
        for _ in range(CFX["steps"]):
            st, info = CF2.step(st, CFX["Ntarget"], CFX["Nboundary"], 0, CFX["Nmax"], (1.0, 0.0, 0.0, 0.0), CFX["dt"],
                                x_e, y_e, lambda T: 1.0 * np.maximum(T, 1e-3) ** -3, lambda e: e / cvx,
                                lambda T: cvx + 0 * T, np.zeros((nx, ny)), reflect=(False, False, True, True),
                                geometry="xy")
        Ts.append(st.temperature.copy()); Trs.append(st.radiation_temperature.copy())
    Ts, Trs = np.array(Ts), np.array(Trs)
    xy = dict(T_mean=Ts.mean(0), T_se=Ts.std(0, ddof=1) / np.sqrt(seeds), Tr_mean=Trs.mean(0),
              Tr_se=Trs.std(0, ddof=1) / np.sqrt(seeds), seeds=seeds, **CFX)
    return slab, xy


def main_cf():
    import contextlib
    import io

    t0 = time.time()
    load_reference()
    CF1, CF2 = load_reference_cf()
    with contextlib.redirect_stdout(io.StringIO()):
        pins = gen_cf_pins(CF1, CF2)
    np.savez_compressed(os.path.join(HERE, "cf.npz"), **pins)
    print(f"Carter-Forest pins written ({time.time() - t0:.1f} s)")
    if "--no-stats" not in sys.argv:
        with contextlib.redirect_stdout(io.StringIO()):
            slab, xy = run_stats_cf(CF1, CF2)
        np.savez_compressed(os.path.join(HERE, "stats_cf_slab.npz"), **slab)
        np.savez_compressed(os.path.join(HERE, "stats_cf_xy.npz"), **xy)
        print(f"Carter-Forest statistics written ({time.time() - t0:.1f} s)")


def key_tree(d):
    """Nested key structure of an info dict: {key: subtree or None}."""
    return {k: (key_tree(v) if isinstance(v, dict) else None) for k, v in d.items()}


# small problems for the time-loop fixtures: final_time is not a multiple of dt, so every loop
# ends with a short step, and output_freq = 3 exercises the output cadence
LOOP = dict(dt=0.01, final_time=0.075, output_freq=3, N=300, Nmax=1000, T0=0.01, cv=0.3)


def gen_loops():
    """The reference's run_simulation loops (IMC/IMC1D.py:1127, IMC/IMC2D.py:1900,
    MG_IMC/MG_IMC2D.py:2125, MG_IMC/MG_IMC1D.py:1312, IMC/IMC1D_CarterForest.py:1381,
    IMC/IMC2D_CarterForest.py:1162) on small problems: output times, history shapes and, for
    the loops that return info dicts, their times and key trees; plus the info key tree of one
    step() of every module."""
    IMC1D, IMC2D = load_reference()
    MG2 = load_reference_mg()
    MG1 = load_reference_mg1d()
    CF1, CF2 = load_reference_cf()
    L = LOOP
    cv, N, Nmax, dt, tf, of = L["cv"], L["N"], L["Nmax"], L["dt"], L["final_time"], L["output_freq"]
    eos, inv = (lambda T: cv * T), (lambda e: e / cv)
    cvf = lambda T: cv + 0 * T  # noqa: E731
    sig = lambda T: 10.0 + 0 * T  # noqa: E731
    I = 10
    mesh = np.array([[i * 0.01, (i + 1) * 0.01] for i in range(I)])
    x_e, y_e = np.linspace(0, 0.06, 7), np.linspace(0, 0.05, 6)
    r_e, z_e = np.linspace(0, 0.06, 7), np.linspace(0, 0.05, 6)
    m_e, m_y = np.linspace(0, 0.06, 7), np.array([0.0, 1.0])
    gedges = np.array([1e-2, 0.3, 2.0, 20.0])
    gsig = [lambda T, k=k: (5.0 + 0 * T) * k for k in (1.0, 2.0, 4.0)]
    out = {"problem": L}
    T1 = np.full(I, L["T0"])

    def hist(times, Tr, T):
        return {"times": [float(t) for t in times], "Tr_shape": list(np.shape(Tr)), "T_shape": list(np.shape(T))}

    seed_py, seed_np, _, _ = nb_helpers()

    def seed(s):
        np.random.seed(s); random.seed(s); seed_py(s); seed_np(s)

    seed(1)
    out["imc1d"] = hist(*IMC1D.run_simulation(N, N, 0, Nmax, T1, T1, (1.0, 0.0), dt, mesh, sig, eos, inv, cvf,
                                              np.zeros(I), tf, output_freq=of))
    st = IMC1D.init_simulation(N, T1, T1, mesh, eos, inv)
    _, info = IMC1D.step(st, N, N, 0, Nmax, (1.0, 0.0), dt, mesh, sig, inv, cvf, np.zeros(I))
    out["imc1d"]["info_keys"] = key_tree(info)
    for geo, e1, e2 in (("xy", x_e, y_e), ("rz", r_e, z_e)):
        T2 = np.full((len(e1) - 1, len(e2) - 1), L["T0"])
        seed(2)
        out[f"imc2d_{geo}"] = hist(*IMC2D.run_simulation(N, N, 0, Nmax, T2, T2, (1.0, 0.0, 0.0, 0.0), dt, e1, e2, sig,
                                                         eos, inv, cvf, np.zeros_like(T2), tf, output_freq=of,
                                                         geometry=geo))
        st = IMC2D.init_simulation(N, T2, T2, e1, e2, eos, inv, geometry=geo)
        _, info = IMC2D.step(st, N, N, 0, Nmax, (1.0, 0.0, 0.0, 0.0), dt, e1, e2, sig, inv, cvf, np.zeros_like(T2),
                             geometry=geo)
        out[f"imc2d_{geo}"]["info_keys"] = key_tree(info)
        seed(3)
        out[f"imc2d_cf_{geo}"] = hist(*CF2.run_simulation(N, N, 0, Nmax, T2, T2, (1.0, 0.0, 0.0, 0.0), dt, e1, e2, sig,
                                                          eos, inv, cvf, np.zeros_like(T2), tf, output_freq=of,
                                                          geometry=geo))
        st = CF2.init_simulation(N, T2, T2, e1, e2, eos, inv, geometry=geo)
        _, info = CF2.step(st, N, N, 0, Nmax, (1.0, 0.0, 0.0, 0.0), dt, e1, e2, sig, inv, cvf, np.zeros_like(T2),
                           geometry=geo)
        out[f"imc2d_cf_{geo}"]["info_keys"] = key_tree(info)
    seed(4)
    out["imc1d_cf"] = hist(*CF1.run_simulation(N, N, 0, Nmax, T1, T1, (1.0, 0.0), dt, mesh, sig, eos, inv, cvf,
                                               np.zeros(I), tf, output_freq=of))
    st = CF1.init_simulation(N, T1, T1, mesh, eos, inv)
    _, info = CF1.step(st, N, N, 0, Nmax, (1.0, 0.0), dt, mesh, sig, inv, cvf, np.zeros(I))
    out["imc1d_cf"]["info_keys"] = key_tree(info)
    # multigroup 2-D (xy strip, reflecting in y): (history, state)
    Tm = np.full((len(m_e) - 1, 1), L["T0"])
    seed(5)
    history, _ = MG2.run_simulation(N, N, 0, Nmax, Tm, Tm, (1.0, 0.0, 0.0, 0.0), dt, m_e, m_y, gedges, gsig, eos, inv,
                                    cvf, np.zeros_like(Tm), tf, reflect=(False, False, True, True), output_freq=of)
    out["mg_imc2d"] = {"history_times": [float(h["time"]) for h in history],
                       "history_keys": key_tree(history[-1]), "info_keys": None}
    st = MG2.init_simulation(N, Tm, Tm, m_e, m_y, gedges, eos, inv)
    _, info = MG2.step(st, N, N, 0, Nmax, (1.0, 0.0, 0.0, 0.0), dt, m_e, m_y, gedges, gsig, inv, cvf,
                       np.zeros_like(Tm), reflect=(False, False, True, True))
    out["mg_imc2d"]["info_keys"] = key_tree(info)
    # multigroup sphere: (times, Tr_hist, T_hist, state, history)
    Ts = np.full(6, L["T0"])
    smesh = np.array([[i * 0.01, (i + 1) * 0.01] for i in range(6)])
    seed(6)
    times, Tr, T, _, history = MG1.run_simulation(N, N, 0, Nmax, Ts, Ts, (0.0, 1.0), dt, smesh, gedges, gsig, eos,
                                                  inv, cvf, np.zeros(6), tf, output_freq=of)
    out["mg_imc1d"] = hist(times, Tr, T)
    out["mg_imc1d"]["history_times"] = [float(h["time"]) for h in history]
    st = MG1.init_simulation(N, Ts, Ts, smesh, gedges, eos, inv)
    _, info = MG1.step(st, N, N, 0, Nmax, (0.0, 1.0), dt, smesh, gedges, gsig, inv, cvf, np.zeros(6))
    out["mg_imc1d"]["info_keys"] = key_tree(info)
    return out


def main_stats():
    """Only the multi-seed statistics of the gray slab, RZ crooked pipe and multigroup steps."""
    import contextlib
    import io

    t0 = time.time()
    IMC1D, IMC2D = load_reference()
    for name, fn in (("stats_slab.npz", lambda: run_stats_slab(IMC1D)), ("stats_rz.npz", lambda: run_stats_rz(IMC2D)),
                     ("stats_mg.npz", lambda: run_stats_mg(load_reference_mg()))):
        with contextlib.redirect_stdout(io.StringIO()):
            s = fn()
        np.savez_compressed(os.path.join(HERE, name), **s)
        print(f"{name} written ({time.time() - t0:.1f} s)", flush=True)


def main_loops():
    import contextlib
    import io
    import json

    t0 = time.time()
    with contextlib.redirect_stdout(io.StringIO()):
        loops = gen_loops()
    with open(os.path.join(HERE, "loops.json"), "w") as f:
        json.dump(loops, f, indent=1, sort_keys=True)
    print(f"time-loop fixtures written ({time.time() - t0:.1f} s)")


def main():
    if not REF or not os.path.isdir(REF):
        raise SystemExit("set RADTRANBOOK_REF to the reference checkout")
    if "--mg1d-only" in sys.argv:
        return main_mg1d()
    if "--cf-only" in sys.argv:
        return main_cf()
    if "--loops-only" in sys.argv:
        return main_loops()
    if "--stats-only" in sys.argv:
        return main_stats()
    t0 = time.time()
    IMC1D, IMC2D = load_reference()
    import contextlib
    import io

    with contextlib.redirect_stdout(io.StringIO()):
        ev = gen_events(IMC1D, IMC2D)
        cb = gen_comb(IMC1D, IMC2D)
        sp = gen_samplers(IMC1D, IMC2D)
        so = gen_sources(IMC1D, IMC2D)
    np.savez_compressed(os.path.join(HERE, "events.npz"), **ev)
    np.savez_compressed(os.path.join(HERE, "comb.npz"), **cb)
    np.savez_compressed(os.path.join(HERE, "samplers.npz"), **sp)
    np.savez_compressed(os.path.join(HERE, "sources.npz"), **so)
    print(f"pins written ({time.time() - t0:.1f} s)")
    if "--no-stats" not in sys.argv:
        with contextlib.redirect_stdout(io.StringIO()):
            s1 = run_stats_slab(IMC1D)
        np.savez_compressed(os.path.join(HERE, "stats_slab.npz"), **s1)
        print(f"slab statistics written ({time.time() - t0:.1f} s)")
        with contextlib.redirect_stdout(io.StringIO()):
            s2 = run_stats_rz(IMC2D)
        np.savez_compressed(os.path.join(HERE, "stats_rz.npz"), **s2)
        print(f"rz statistics written ({time.time() - t0:.1f} s)")
    MG_IMC2D = load_reference_mg()
    with contextlib.redirect_stdout(io.StringIO()):
        pl = gen_planck_sampler(MG_IMC2D)
    np.savez_compressed(os.path.join(HERE, "planck.npz"), **pl)
    if "--no-stats" not in sys.argv and "--no-mg-stats" not in sys.argv:
        with contextlib.redirect_stdout(io.StringIO()):
            s3 = run_stats_mg(MG_IMC2D)
        np.savez_compressed(os.path.join(HERE, "stats_mg.npz"), **s3)
        print(f"multigroup statistics written ({time.time() - t0:.1f} s)")
    main_mg1d()
    main_cf()


if __name__ == "__main__":
    main()
