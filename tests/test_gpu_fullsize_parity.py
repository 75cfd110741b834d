"""GPU against the FP64 oracle at the workloads' stated sizes.

Each single-problem workload runs a few drop-in steps on the GPU (device material callables)
until its census is established, then the census is copied into the oracle and ONE transport
step (sources + tracking, the same Philox streams) runs on both sides from that identical
bank:

  - slab Marshak wave: 100 cells, 20k emission + 20k boundary particles per step, NMax 80k,
    after 20 steps;
  - RZ crooked pipe: 60 x 210 cells, 2e6 source particles per step (1,333,334 emission +
    666,666 surface), Nmax 6.67e6, after 5 steps (census about 6.7e6);
  - multigroup Marshak wave: 200 cells x 10 groups, 1e6 source particles per step, Nmax
    1.33e6, after 8 steps;
  - differentiable step: 128 x 128 random-opacity XY field, 4e6 boundary histories, the
    deposition of the forward step and the vector-Jacobian product for the unit cotangent
    against the oracle's FP64 adjoint of the same estimator.

Tolerances (FP32 tracking against FP64, stated per quantity, the same as the reduced-size
parity tests): transported entries exact; issued boundary energy and emitted energy per cell
to FP32 weight rounding (rtol 1e-7); per-cell deposition and intensity relative L1 <= 2e-4
(gray) / 5e-4 (multigroup); escaped energy relative 2e-4 / 5e-4 of the energy in play; event
count relative 1e-3; adjoint gradient relative L1 <= 2e-3.  The oracle runs with every host
thread (about 1-3 s per step on the GPU host).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200 import adjoint, imc1d, imc2d, mg_imc2d, problems

pytestmark = pytest.mark.gpu

L1 = lambda a, b: np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)  # noqa: E731


def _oracle_from_engine(eng):
    orc = O.Oracle(eng.geometry, eng.e1.cpu().numpy(), eng.e2.cpu().numpy(), eng.vol.cpu().numpy(), eng.seed,
                   n_groups=eng.ng)
    b = eng.bank
    fields = [b.view(k).double().cpu().numpy() for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")]
    orc.set_bank(*fields, b.view("cell").cpu().numpy(), b.view("group").cpu().numpy() if eng.ng > 1 else None)
    return orc


def _dev(a, cuda):
    return None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=cuda)


def _compare(eng, res, ro, tol, energy_in):
    rep = res.report
    assert rep.n_transported == ro["n_transported"]
    np.testing.assert_allclose(rep.boundary_emission, ro["boundary_emission"], rtol=1e-7)
    np.testing.assert_allclose(eng.emitted.cpu().numpy(), ro["emitted"], rtol=1e-7, atol=1e-300)
    dep, si = eng.dep.cpu().numpy(), eng.si.cpu().numpy()
    assert L1(dep, ro["dep"]) <= tol, L1(dep, ro["dep"])
    assert L1(si, ro["si"]) <= tol, L1(si, ro["si"])
    stats, esc = eng.host_stats()
    assert abs(esc[:4].sum() - ro["escaped"].sum()) <= tol * energy_in
    np.testing.assert_allclose(stats[0], ro["stats"][0], rtol=1e-3)
    return L1(dep, ro["dep"])


def test_slab_marshak_full_size_step_matches_oracle(cuda):
    p = problems.marshak_slab()
    st = imc1d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["mesh"], p["eos_dev"], p["inv_eos_dev"],
                               seed=0xF5A1)
    for _ in range(20):
        st, _ = imc1d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], p["mesh"],
                           p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"])
    eng = st._engine
    assert eng.bank.size > 0.9 * p["Nmax"]
    orc = _oracle_from_engine(eng)
    T = st._T.cpu().numpy()
    sig, cv = 300.0 * T ** -3.0, np.full_like(T, 0.3)
    face = [np.array([1.0]), None]
    res = eng.transport(_dev(T, cuda), _dev(sig, cuda), _dev(cv, cuda), None, st.count, p["dt"], 1.0, p["Ntarget"],
                        p["Nboundary"], 0, [_dev(f, cuda) for f in face], (False, False))
    ro = orc.transport(T, sig, cv, None, st.count, p["dt"], 1.0, p["Ntarget"], p["Nboundary"], 0, face,
                       (False, False))
    _compare(eng, res, ro, 2e-4, ro["boundary_emission"] + float(np.sum(ro["emitted"])))


def test_crooked_pipe_full_size_step_matches_oracle(cuda):
    p = problems.crooked_pipe()
    st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_dev"],
                               p["inv_eos_dev"], geometry="rz", seed=0xF5A2)
    for _ in range(5):
        st, _ = imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], p["edges1"],
                           p["edges2"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"], p["source"], reflect=p["reflect"],
                           geometry="rz", boundary_source_func=p["boundary_source_func"])
    eng = st._engine
    assert eng.bank.size > 0.9 * p["Nmax"]
    orc = _oracle_from_engine(eng)
    T = st._T.cpu().numpy()
    sig = O.flat2d(p["sigma_host"](p["Tinit"]))
    cv = O.flat2d(p["cv_host"](p["Tinit"]))
    rc = 0.5 * (p["edges1"][:-1] + p["edges1"][1:])
    face = [None, None, np.where(rc < 0.5, 0.5, 0.0), None]
    res = eng.transport(_dev(T, cuda), _dev(sig, cuda), _dev(cv, cuda), None, st.count, p["dt"], 1.0, p["Ntarget"],
                        p["Nboundary"], 0, [_dev(f, cuda) for f in face], p["reflect"], max_events=1_000_000)
    ro = orc.transport(T, sig, cv, None, st.count, p["dt"], 1.0, p["Ntarget"], p["Nboundary"], 0, face, p["reflect"],
                       max_events=1_000_000)
    assert ro["stats"][0] > 5e7  # the full-size step: tens of millions of track segments
    _compare(eng, res, ro, 2e-4, ro["boundary_emission"] + float(np.sum(ro["emitted"])))


def test_mg_marshak_full_size_step_matches_oracle(cuda):
    p = problems.marshak_mg()
    st = mg_imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"],
                                  p["energy_edges"], p["eos_dev"], p["inv_eos_dev"], geometry="xy", seed=0xF5A3)
    for _ in range(8):
        st, _ = mg_imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"], p["edges1"],
                              p["edges2"], p["energy_edges"], p["sigma_dev"], p["inv_eos_dev"], p["cv_dev"],
                              p["source"], reflect=p["reflect"], geometry="xy")
    eng = st._engine
    assert eng.bank.size > 0.9 * p["Nmax"]
    orc = _oracle_from_engine(eng)
    T = st._T.cpu().numpy()
    sig = np.stack([h(T) for h in p["sigma_host"]]).reshape(-1)  # [g, c]
    cv = np.full_like(T, 0.3)
    face = [np.array([1.0]), None, None, None]
    res = eng.transport(_dev(T, cuda), _dev(sig, cuda), _dev(cv, cuda), None, st.count, p["dt"], 1.0, p["Ntarget"],
                        p["Nboundary"], 0, [_dev(f, cuda) for f in face], p["reflect"], max_events=1_000_000,
                        rz_linear_source=False)
    ro = orc.transport_mg(T, sig, cv, None, st.count, p["dt"], 1.0, p["Ntarget"], p["Nboundary"], 0, face, p["reflect"],
                          p["energy_edges"], max_events=1_000_000)
    e_in = ro["boundary_emission"] + ro["source_emission"] + ro["emission_total"]
    _compare(eng, res, ro, 5e-4, e_in)
    assert np.abs(eng.escaped_group.cpu().numpy() - ro["esc_by_group"]).sum() <= 1e-3 * e_in


def test_adjoint_full_size_matches_oracle(cuda):
    prob, sigma = adjoint.opacity_field_problem()
    s = prob.setup
    sig = torch.as_tensor(sigma, device=cuda)
    cot = adjoint.unit_cotangent(prob.nc)
    dep = prob.forward(sig).cpu().numpy()
    g = prob.vjp(sig, torch.as_tensor(cot, device=cuda)).cpu().numpy()
    e = s.edges1
    vol = O.flat2d(np.diff(e)[:, None] * np.diff(e)[None, :])
    Tc, cvc = np.full(prob.nc, s.T), np.full(prob.nc, s.cv)
    n = len(e) - 1
    face = [np.full(n, 1.0), None, None, None]
    # forward deposition from the same sources
    o = O.Oracle("xy", e, e, vol, s.seed)
    ro = o.transport(Tc, sigma, cvc, None, s.step, s.dt, s.theta, 0, s.n_boundary, 0, face, s.reflect,
                     max_events=s.max_events, rz_linear_source=False)
    assert ro["n_transported"] == s.n_boundary
    assert L1(dep, ro["dep"]) <= 2e-4, L1(dep, ro["dep"])
    # gradient: the oracle's adjoint replays the same histories in FP64
    o2 = O.Oracle("xy", e, e, vol, s.seed)
    o2.transport(Tc, sigma, cvc, None, s.step, s.dt, s.theta, 0, s.n_boundary, 0, face, s.reflect,
                 max_events=s.max_events, rz_linear_source=False, sources_only=True)
    g_orc = o2.adjoint_vjp(Tc, sigma, cvc, s.step, s.dt, s.theta, s.reflect, cot, max_events=s.max_events)
    assert L1(g, g_orc) <= 2e-3, L1(g, g_orc)
