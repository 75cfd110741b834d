"""GPU parity: the CUDA path (through the C ABI) against the FP64 CPU oracle on the same
inputs and the same Philox streams.

Tolerances (FP32 tracking vs FP64 oracle, stated per quantity):
  - integer work (source counts per cell, cells of sampled particles, comb copies from an
    identical bank): exact;
  - per-particle sampled positions/directions/weights: FP32 rounding (rel 2e-6);
  - per-cell tallies after one transport step from an identical bank: relative L1 error
    over cells <= 2e-4 (FP32 geometry; a history whose event order flips on a near-tie
    diverges from the oracle's, which the L1 bound absorbs);
  - event statistics: relative 1e-3;
  - energy ledger of the CUDA path: |closure| / total <= 1e-12 per step.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200 import _lib, problems
from radtranbook_b200.engine import Engine

pytestmark = pytest.mark.gpu

SEED = 0x5EED0001


def _rz_small():
    p = problems.crooked_pipe(scale=0.01, nr=30, nz=105)
    return p


def _engine_and_oracle(geometry, e1, e2, vol, seed=SEED):
    eng = Engine(geometry, e1, e2, vol, seed=seed)
    orc = O.Oracle(geometry, e1, e2, vol, seed)
    return eng, orc


def _vol2d(e1, e2, geometry):
    if geometry == "xy":
        v = np.diff(e1)[:, None] * np.diff(e2)[None, :]
    else:
        v = np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :]
    return O.flat2d(v)


def _bank_to_oracle(eng, orc):
    b = eng.bank
    orc.set_bank(*(b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")),
                 b.view("cell").cpu().numpy())


def test_philox_device_matches_oracle(cuda):
    lib = _lib.load()
    rng = np.random.default_rng(1)
    ctr = rng.integers(0, 2**32, size=(257, 4), dtype=np.uint64).astype(np.uint32)
    key = (0xA4093822, 0x299F31D0)
    d_ctr = torch.as_tensor(ctr.view(np.int32), device=cuda)
    d_out = torch.zeros_like(d_ctr)
    _lib.check("imc_philox", lib.imc_philox(d_ctr.data_ptr(), key[0], key[1], d_out.data_ptr(), len(ctr),
                                            torch.cuda.current_stream().cuda_stream))
    got = d_out.cpu().numpy().view(np.uint32)
    for q in range(len(ctr)):
        np.testing.assert_array_equal(got[q], O.philox(ctr[q], key))
    # Random123 known-answer vector
    one = torch.as_tensor(np.array([[0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344]], dtype=np.uint32).view(np.int32), device=cuda)
    o1 = torch.zeros_like(one)
    lib.imc_philox(one.data_ptr(), key[0], key[1], o1.data_ptr(), 1, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert list(o1.cpu().numpy().view(np.uint32)[0]) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("geometry", ["slab", "spherical", "xy", "rz"])
def test_initial_census_matches_oracle(cuda, geometry):
    if geometry in ("slab", "spherical"):
        e1 = np.linspace(0.0 if geometry == "slab" else 0.05, 0.2, 41)
        e2 = np.array([0.0, 1.0])
        vol = np.diff(e1) if geometry == "slab" else 4 / 3 * np.pi * np.diff(e1 ** 3)
        tr = np.linspace(0.2, 1.0, 40)
    else:
        e1 = np.linspace(0.0, 1.0, 13)
        e2 = np.linspace(0.0, 2.0, 21)
        vol = _vol2d(e1, e2, geometry)
        tr = O.flat2d(np.outer(np.linspace(0.1, 1.0, 12), np.linspace(1.0, 0.3, 20)))
    eng, orc = _engine_and_oracle(geometry, e1, e2, vol)
    n_gpu = eng.init_census(torch.as_tensor(tr, device=cuda), 5000)
    n_orc = orc.init_ic(tr, 5000)
    assert n_gpu == n_orc
    ob = orc.get_bank()
    gb = {k: eng.bank.view(k).cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2", "cell")}
    np.testing.assert_array_equal(gb["cell"], ob["cell"])
    np.testing.assert_allclose(gb["weight"], ob["weight"], rtol=1e-7)
    np.testing.assert_allclose(gb["pos1"], ob["pos1"], rtol=2e-6, atol=1e-7)
    np.testing.assert_allclose(gb["dir1"], ob["dir1"], rtol=2e-6, atol=1e-6)
    if geometry in ("xy", "rz"):
        np.testing.assert_allclose(gb["pos2"], ob["pos2"], rtol=2e-6, atol=1e-7)
        np.testing.assert_allclose(gb["dir2"], ob["dir2"], rtol=2e-6, atol=1e-6)


def _one_step_compare(geometry, e1, e2, vol, T, sigma, cv, face_T, reflect, Ntarget, Nboundary, max_events, cuda,
                      source=None, Nsource=0, ic=4000, rz_linear=True):
    eng, orc = _engine_and_oracle(geometry, e1, e2, vol)
    dev = lambda a: None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64), device=cuda)  # noqa: E731
    eng.init_census(dev(T), ic)
    _bank_to_oracle(eng, orc)
    res = eng.transport(dev(T), dev(sigma), dev(cv), dev(source), 3, 0.01, 1.0, Ntarget, Nboundary, Nsource,
                        [dev(f) for f in face_T], reflect, max_events=max_events, rz_linear_source=rz_linear)
    ro = orc.transport(T, sigma, cv, source, 3, 0.01, 1.0, Ntarget, Nboundary, Nsource, face_T, reflect,
                       max_events=max_events, rz_linear_source=rz_linear)
    rep = res.report
    assert rep.n_transported == ro["n_transported"]
    stats, esc = eng.host_stats()
    dep = eng.dep.cpu().numpy()
    si = eng.si.cpu().numpy()
    # identical issued source energy (integer counts, FP32 weights)
    np.testing.assert_allclose(rep.boundary_emission, ro["boundary_emission"], rtol=1e-7)
    np.testing.assert_allclose(eng.emitted.cpu().numpy(), ro["emitted"], rtol=1e-7, atol=1e-300)
    l1 = lambda a, b: np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)  # noqa: E731
    assert l1(dep, ro["dep"]) < 2e-4, l1(dep, ro["dep"])
    assert l1(si, ro["si"]) < 2e-4, l1(si, ro["si"])
    np.testing.assert_allclose(esc[:4].sum(), ro["escaped"].sum(), rtol=2e-4, atol=1e-12 * max(rep.boundary_emission, 1e-30))
    np.testing.assert_allclose(stats[0], ro["stats"][0], rtol=1e-3)
    return eng, orc, res, ro


def test_transport_slab_matches_oracle(cuda):
    p = problems.marshak_slab()
    e1 = np.concatenate([p["mesh"][:, 0], p["mesh"][-1:, 1]])
    T = np.linspace(0.9, 0.02, 100)
    _one_step_compare("slab", e1, np.array([0.0, 1.0]), np.diff(e1), T, 300 * T ** -3.0, np.full(100, 0.3),
                      [np.array([1.0]), None], (False, False), 3000, 3000, 0, cuda)


def test_transport_sphere_matches_oracle(cuda):
    e1 = np.linspace(0.0, 0.5, 51)
    T = np.linspace(0.6, 0.05, 50)
    _one_step_compare("spherical", e1, np.array([0.0, 1.0]), 4 / 3 * np.pi * np.diff(e1 ** 3), T, 5.0 / T,
                      np.full(50, 0.1), [None, np.array([0.8])], (True, False), 3000, 3000, 0, cuda)


def test_transport_xy_matches_oracle(cuda):
    e1 = np.linspace(0.0, 1.0, 17)
    e2 = np.linspace(0.0, 1.0, 17)
    vol = _vol2d(e1, e2, "xy")
    T = O.flat2d(np.outer(np.linspace(0.5, 0.05, 16), np.ones(16)))
    _one_step_compare("xy", e1, e2, vol, T, 20.0 / T, np.full(256, 0.1), [np.full(16, 1.0), None, None, None],
                      (False, False, True, True), 3000, 3000, 1_000_000, cuda)


def test_transport_rz_crooked_pipe_matches_oracle(cuda):
    p = _rz_small()
    e1, e2 = p["edges1"], p["edges2"]
    vol = _vol2d(e1, e2, "rz")
    T = O.flat2d(p["Tinit"])
    rc = 0.5 * (e1[:-1] + e1[1:])
    face = [None, None, np.where(rc < 0.5, 0.5, 0.0), None]
    _one_step_compare("rz", e1, e2, vol, T, O.flat2d(p["sigma_host"](p["Tinit"])), O.flat2d(p["cv_host"](p["Tinit"])),
                      face, p["reflect"], 6000, 3000, 1_000_000, cuda)


def test_comb_matches_oracle_on_identical_bank(cuda):
    e1 = np.linspace(0.0, 1.0, 9)
    e2 = np.linspace(0.0, 1.0, 9)
    vol = _vol2d(e1, e2, "xy")
    eng, orc = _engine_and_oracle("xy", e1, e2, vol)
    rng = np.random.default_rng(7)
    n = 20000
    # FP32-exact weights so both sides comb the same numbers
    w = rng.uniform(0.1, 2.0, n).astype(np.float32).astype(np.float64)
    cell = rng.integers(0, 64, n).astype(np.int32)
    f = lambda: rng.uniform(0, 1, n).astype(np.float32).astype(np.float64)  # noqa: E731
    d1, d2, p1, p2 = f(), f(), f(), f()
    eng.bank.load(w, d1, d2, np.zeros(n), p1, p2, cell)
    orc.set_bank(w, d1, d2, np.zeros(n), p1, p2, cell)
    rep = eng.comb(5000, 11)
    disc_o = orc.comb(5000, 11)
    ob = orc.get_bank()
    assert rep.n_out == len(ob["weight"])
    np.testing.assert_array_equal(eng.bank.view("cell").cpu().numpy(), ob["cell"])
    np.testing.assert_allclose(eng.bank.view("weight").cpu().numpy(), ob["weight"], rtol=1e-7)
    np.testing.assert_array_equal(eng.bank.view("pos1").cpu().numpy(), ob["pos1"].astype(np.float32))
    np.testing.assert_allclose(eng.disc.cpu().numpy(), disc_o, atol=1e-4 * w.sum() / 64)


def test_crooked_pipe_ledger_closes(cuda):
    """Five drop-in steps of a reduced crooked pipe: FP64 energy closure <= 1e-12."""
    from radtranbook_b200 import imc2d

    p = problems.crooked_pipe(scale=0.02)
    st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                               p["inv_eos_dev"], geometry="rz")
    for _ in range(5):
        st, info = imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"],
                              p["edges1"], p["edges2"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"],
                              reflect=p["reflect"], geometry="rz", boundary_source_func=p["boundary_source_func"])
        assert abs(info["ledger"]["relative_closure"]) < 1e-12, info["ledger"]
        assert info["profiling"]["transport_events"]["total"] > 0
    assert np.all(np.isfinite(info["temperature"]))
