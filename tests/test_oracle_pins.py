"""The FP64 CPU oracle pinned against golden vectors recorded from the reference itself
(tests/golden/make_golden.py): event arithmetic, comb, position samplers and per-cell
source counts.  The reference's Numba / Python random streams were seeded and replayed
when the fixtures were made, so each case carries the exact uniforms the reference drew.

Tolerances: FP64 arithmetic restated in another order agrees to ~1e-12 relative; RZ
positions after a radial crossing differ by the reference's 1e-12 relative face nudge;
integer outputs (event type, face crossed, comb copies, source counts) are exact.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

G = os.path.join(os.path.dirname(__file__), "golden")


def _uniforms(geo, row, r):
    """Map the reference's draws onto the oracle's (u0 distance, u1, u2 direction)."""
    ss, L = row[10], (row[6] - row[5]) if geo in ("slab", "spherical") else min(row[6] - row[5], row[8] - row[7])
    thr = 1e-10 if geo in ("slab", "spherical") else 1e-12
    if ss * L > 10000.0:
        return [1.0 - r[1], r[2], r[3]]
    if ss > thr:
        return [1.0 - r[0], r[1], r[2]]
    return [0.5, r[0], r[1]]


@pytest.mark.parametrize("geo,key", [("slab", "slab"), ("spherical", "sphere"), ("xy", "xy"), ("rz", "rz")])
def test_event_matches_reference(geo, key):
    d = np.load(os.path.join(G, "events.npz"))
    ins, rs, outs = d[f"{key}_in"], d[f"{key}_r"], d[f"{key}_out"]
    n_checked = 0
    for row, r, ref in zip(ins, rs, outs):
        got = O.event(geo, list(row) + _uniforms(geo, row, r))
        assert int(got[9]) == int(ref[9]), (geo, row, got, ref)          # event type
        assert int(got[8]) == int(ref[8]), (geo, row, got, ref)          # face crossed
        tau = row[9] * max(row[11] - ref[7], 0.0)  # optical depth of the flight amplifies distance rounding
        np.testing.assert_allclose(got[0], ref[0], rtol=1e-12 * (1.0 + 10.0 * tau), atol=1e-300)  # weight
        np.testing.assert_allclose(got[7], ref[7], rtol=1e-9, atol=1e-14)    # census distance
        # deposits: w - w e^{-sigma s} cancels for small sigma s in both codes, so the
        # absolute tolerance is a few ulps of the weight (per unit length in 1-D)
        vol = (row[6] - row[5]) if geo == "slab" else 1.0
        if geo == "spherical":
            vol = 4.0 / 3.0 * np.pi * (row[6] ** 3 - row[5] ** 3)
        ulp_w = 64 * np.finfo(float).eps * row[0] / vol
        np.testing.assert_allclose(got[5], ref[5], rtol=1e-9, atol=ulp_w)    # deposited weight
        sa_thr = 1e-10 if geo in ("slab", "spherical") else 1e-12
        ulp_i = ulp_w / row[9] if row[9] > sa_thr else ulp_w
        np.testing.assert_allclose(got[6], ref[6], rtol=1e-9, atol=ulp_i)    # path-length intensity
        np.testing.assert_allclose(got[1], ref[1], rtol=1e-9, atol=1e-10)    # direction 1
        np.testing.assert_allclose(got[3], ref[3], rtol=1e-10, atol=1e-12)   # position 1 (nudges: 1e-12 rel)
        if geo in ("xy", "rz"):
            np.testing.assert_allclose(got[2], ref[2], rtol=1e-9, atol=1e-10)
            np.testing.assert_allclose(got[4], ref[4], rtol=1e-10, atol=1e-12)
        n_checked += 1
    assert n_checked > 0.95 * len(ins)
    # every event kind is exercised
    assert set(np.unique(outs[:, 9]).astype(int)) == {0, 1, 2}


def test_comb_1d_matches_reference():
    d = np.load(os.path.join(G, "comb.npz"))
    n = len(d["c1_w"])
    e = np.linspace(0, 1, 41)
    o = O.Oracle("slab", e, [0.0, 1.0], np.diff(e), 1)
    o.set_bank(d["c1_w"], d["c1_mu"], np.zeros(n), d["c1_t"], d["c1_x"], np.zeros(n), d["c1_cell"])
    disc = o.comb_with_xi(int(d["c1_nmax"]), d["c1_xi"])
    b = o.get_bank()
    assert len(b["weight"]) == len(d["c1_out_w"])
    np.testing.assert_array_equal(b["cell"], d["c1_out_cell"])
    np.testing.assert_allclose(b["weight"], d["c1_out_w"], rtol=1e-14)
    np.testing.assert_array_equal(b["pos1"], d["c1_out_x"])
    np.testing.assert_array_equal(b["dir1"], d["c1_out_mu"])
    np.testing.assert_allclose(disc, d["c1_disc"], atol=1e-12 * d["c1_w"].sum())


def test_comb_2d_matches_reference():
    d = np.load(os.path.join(G, "comb.npz"))
    nx, ny = int(d["c2_nx"]), int(d["c2_ny"])
    n = len(d["c2_w"])
    e1, e2 = np.linspace(0, 1, nx + 1), np.linspace(0, 1, ny + 1)
    o = O.Oracle("xy", e1, e2, np.ones(nx * ny), 1)
    cell = d["c2_ci"] + nx * d["c2_cj"]
    o.set_bank(d["c2_w"], d["c2_d1"], d["c2_d2"], np.zeros(n), d["c2_p1"], d["c2_p2"], cell)
    disc = o.comb_with_xi(int(d["c2_nmax"]), d["c2_xi"])
    b = o.get_bank()
    assert len(b["weight"]) == len(d["c2_out_w"])
    np.testing.assert_array_equal(b["cell"], d["c2_out_ci"] + nx * d["c2_out_cj"])
    np.testing.assert_allclose(b["weight"], d["c2_out_w"], rtol=1e-14)
    np.testing.assert_array_equal(b["pos1"], d["c2_out_p1"])
    np.testing.assert_allclose(disc, d["c2_disc"], atol=1e-12 * d["c2_w"].sum())


def test_position_samplers_match_reference():
    d = np.load(os.path.join(G, "samplers.npz"))
    lib = O.load()
    for (dx, s, T, xi), ref in zip(d["slab_linear_in"], d["slab_linear_out"]):
        np.testing.assert_allclose(lib.orc_slab_linear(dx, s, T, xi), ref, rtol=1e-11, atol=1e-15 * dx)
    for (r0, r1, a, M, xi), (ref_s, ref_c) in zip(d["cdf_in"], d["cdf_out"]):
        np.testing.assert_allclose(lib.orc_sphere_cdf(r0, r1, a, M, xi), ref_s, rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(lib.orc_rz_r_cdf(r0, r1, a, M, xi), ref_c, rtol=1e-12, atol=1e-15)


def test_emission_counts_match_reference_slab():
    d = np.load(os.path.join(G, "sources.npz"))
    T, sa = d["e1d_T"], d["e1d_sa"]
    I = len(T)
    e = np.linspace(0, 0.01 * I, I + 1)
    e = np.array([i * 0.01 for i in range(I)] + [I * 0.01])
    o = O.Oracle("slab", e, [0.0, 1.0], np.array([0.01] * I), 1)
    o.transport(T, sa, np.full(I, 1.0), None, 0, float(d["e1d_dt"]), 0.0, int(d["e1d_N"]), 0, 0, [None, None],
                (False, False), sources_only=True)
    b = o.get_bank()
    np.testing.assert_array_equal(np.bincount(b["cell"], minlength=I), d["e1d_counts"])
    w = np.array([b["weight"][b["cell"] == i][0] for i in range(I)])
    np.testing.assert_allclose(w, d["e1d_w"], rtol=1e-12)


def test_rz_linear_source_counts_match_reference():
    d = np.load(os.path.join(G, "sources.npz"))
    r_e, z_e = d["rz_r_edges"], d["rz_z_edges"]
    nx, ny = len(r_e) - 1, len(z_e) - 1
    vol = O.flat2d(np.pi * (r_e[1:] ** 2 - r_e[:-1] ** 2)[:, None] * np.diff(z_e)[None, :])
    o = O.Oracle("rz", r_e, z_e, vol, 1)
    T = O.flat2d(d["rz_T"])
    o.transport(T, np.ones(nx * ny), np.ones(nx * ny), O.flat2d(d["rz_src"]), 0, float(d["rz_dt"]), 1.0, 0, 0,
                int(d["rz_N"]), [None] * 4, (False,) * 4, rz_linear_source=True, sources_only=True)
    b = o.get_bank()
    np.testing.assert_array_equal(np.bincount(b["cell"], minlength=nx * ny), d["rz_counts"])
    w = np.zeros(nx * ny)
    for c in range(nx * ny):
        if d["rz_counts"][c]:
            w[c] = b["weight"][b["cell"] == c][0]
    np.testing.assert_allclose(w, d["rz_w"], rtol=1e-12)
    # positions stay inside their cells and follow the T^4 tilt (sampled from the same CDF)
    c = b["cell"]
    assert np.all(b["pos1"] >= r_e[c % nx] - 1e-12) and np.all(b["pos1"] <= r_e[c % nx + 1] + 1e-12)
