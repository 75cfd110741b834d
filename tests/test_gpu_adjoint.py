"""GPU adjoint (imc_adjoint_vjp through the C ABI, and the autograd.Function) against the
FP64 oracle adjoint and against central finite differences of the GPU forward step.

Tolerances: GPU vs oracle gradient on the same sources (FP32 vs FP64 tracking of the same
Philox histories): relative L1 over cells <= 2e-3; GPU adjoint vs finite differences with
common random numbers, cold material (implicit-capture term only): relative 2e-3 per cell
for cells whose derivative is above 1e-3 of the largest; autograd backward == vjp up to the
order of FP64 atomic adds.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from radtranbook_b200 import adjoint

pytestmark = pytest.mark.gpu


def _problem(n, T, cv, nb, log_mean, log_std, seed=3):
    edges = np.linspace(0.0, 1.0, n + 1)
    setup = adjoint.AdjointSetup("xy", edges, edges, T=T, cv=cv, face_T=(1.0, 0.0, 0.0, 0.0),
                                 reflect=(False, False, True, False), dt=0.02, n_boundary=nb)
    rng = np.random.default_rng(seed)
    sigma = np.exp(log_mean + log_std * rng.standard_normal(n * n))
    cot = rng.standard_normal(n * n)
    cot /= np.linalg.norm(cot)
    return setup, sigma, cot


@pytest.mark.parametrize("T,cv", [(0.01, 0.1), (0.8, 0.01)])
def test_gpu_adjoint_matches_oracle(cuda, T, cv):
    n = 16
    setup, sigma, cot = _problem(n, T, cv, 40000, np.log(8.0), 0.6)
    prob = adjoint.AdjointProblem(setup)
    g_gpu = prob.vjp(torch.as_tensor(sigma, device=cuda), torch.as_tensor(cot, device=cuda)).cpu().numpy()
    e = setup.edges1
    vol = O.flat2d(np.diff(e)[:, None] * np.diff(e)[None, :])
    o = O.Oracle("xy", e, e, vol, setup.seed)
    Tc, cvc = np.full(n * n, T), np.full(n * n, cv)
    face = [np.full(n, 1.0), None, None, None]
    o.transport(Tc, sigma, cvc, None, 0, setup.dt, 1.0, 0, setup.n_boundary, 0, face, setup.reflect,
                max_events=setup.max_events, sources_only=True)
    g_orc = o.adjoint_vjp(Tc, sigma, cvc, 0, setup.dt, 1.0, setup.reflect, cot, max_events=setup.max_events)
    rel = np.abs(g_gpu - g_orc).sum() / np.abs(g_orc).sum()
    assert rel <= 2e-3, rel


def test_gpu_adjoint_matches_finite_differences(cuda):
    n = 24
    setup, sigma, cot = _problem(n, 0.01, 0.1, 100000, np.log(20.0), 0.8)
    prob = adjoint.AdjointProblem(setup)
    sig = torch.as_tensor(sigma, device=cuda)
    ct = torch.as_tensor(cot, device=cuda)
    g = prob.vjp(sig, ct).cpu().numpy()
    cells = np.argsort(-np.abs(g))[:12]
    fd = adjoint.fd_check(prob, sig, ct, cells, rel=1e-3)
    scale = np.abs(g).max()
    for c, f in zip(cells, fd):
        if abs(f) > 1e-3 * scale:
            assert abs(g[c] - f) <= 2e-3 * abs(f), (c, g[c], f)


def test_autograd_function_backward_is_the_vjp(cuda):
    n = 12
    setup, sigma, cot = _problem(n, 0.3, 0.05, 20000, np.log(5.0), 0.5)
    prob = adjoint.AdjointProblem(setup)
    sig = torch.as_tensor(sigma, device=cuda).requires_grad_(True)
    dep = adjoint.deposition(sig, prob)
    assert dep.shape == (n * n,) and dep.dtype == torch.float64
    ct = torch.as_tensor(cot, device=cuda)
    (dep * ct).sum().backward()
    ref = prob.vjp(sig.detach(), ct)
    # FP64 atomics add the per-cell sums in a run-dependent order
    torch.testing.assert_close(sig.grad, ref, rtol=1e-10, atol=1e-14 * float(ref.abs().max()))
    # the forward is the plain step, the same Philox histories every call
    torch.testing.assert_close(prob.forward(sig.detach()), dep.detach(), rtol=1e-12, atol=0)
