"""Differentiable IMC step: deposition as a function of the per-cell opacity.

`deposition(sigma, problem)` runs one 2-D gray IMC step (the problem's census, sources,
Philox seed and step index) and returns the per-cell FP64 energy deposition per unit
volume; it is a torch.autograd.Function whose backward calls the adjoint kernel
(imc_adjoint_vjp): the step's histories are regenerated from their Philox counters and
replayed twice each, giving the vector-Jacobian product d(g . dep)/d sigma by the
path-length derivative of implicit capture plus the likelihood-ratio derivative of the
effective-scatter sampling, chained through the Fleck factor.  Nothing is stored between
forward and backward except the opacity and the census the step started from.

`opacity_field_problem()` is the 128 x 128 XY benchmark: sigma = exp(g), g a Gaussian
random field (mean ln 50, standard deviation 1, squared-exponential correlation
exp(-r^2 / (2 l^2)) with l = 0.1 cm), 1 keV source on x = 0, vacuum elsewhere, T = 0.01 keV,
cv = 0.1, one 0.02 ns step of 4e6 boundary histories.  At T = 0.01 keV the material
emission of the step is about 2e-4 of the boundary energy and the initial radiation
energy about 1e-7 of it, so the step carries the boundary histories only.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .engine import Engine, require_cuda
from .rng import normals

TAG_GRF = 0x71000000
TAG_COTANGENT = 0x72000000


def gaussian_random_field(n: int = 128, length: float = 1.0, mean: float = float(np.log(50.0)), std: float = 1.0,
                          ell: float = 0.1, seed: int = 0xAD50) -> np.ndarray:
    """Stationary Gaussian field on an n x n cell-centred grid of [0, length]^2 with
    covariance std^2 exp(-r^2 / (2 ell^2)), by circulant embedding on the 2n x 2n torus
    (Dietrich & Newsam 1997): eigenvalues = FFT of the first row of the periodised
    covariance, field = real part of FFT(sqrt(eigenvalues / M) * complex white noise),
    restricted to the n x n corner.  White noise from Philox (seeded, host).  Returns
    g[i, j] (i along x)."""
    m = 2 * n
    h = length / n
    k = np.arange(m)
    dk = np.minimum(k, m - k) * h
    r2 = dk[:, None] ** 2 + dk[None, :] ** 2
    row = std ** 2 * np.exp(-r2 / (2.0 * ell ** 2))
    lam = np.real(np.fft.fft2(row))
    lam = np.maximum(lam, 0.0)  # round-off negatives of a positive-definite embedding
    z = normals(2 * m * m, seed, TAG_GRF).reshape(2, m, m)
    w = (z[0] + 1j * z[1]) * np.sqrt(lam / (m * m))
    f = np.fft.fft2(w)
    return mean + np.real(f)[:n, :n]


def unit_cotangent(nc: int, seed: int = 0xC07A) -> np.ndarray:
    g = normals(nc, seed, TAG_COTANGENT)
    return g / np.linalg.norm(g)


@dataclass
class AdjointSetup:
    geometry: str
    edges1: np.ndarray
    edges2: np.ndarray
    T: float
    cv: float
    face_T: tuple          # per side: temperature (keV) or 0
    reflect: tuple
    dt: float
    n_boundary: int
    seed: int = 0x5EED0005
    step: int = 0
    theta: float = 1.0
    max_events: int = 1_000_000


class AdjointProblem:
    """One differentiable step on the device: forward(sigma) -> dep, vjp(sigma, g) -> grad."""

    def __init__(self, setup: AdjointSetup, device: torch.device | None = None):
        self.setup = setup
        self.device = device or require_cuda()
        e1 = np.asarray(setup.edges1, dtype=np.float64)
        e2 = np.asarray(setup.edges2, dtype=np.float64)
        self.nx, self.ny = len(e1) - 1, len(e2) - 1
        if setup.geometry == "xy":
            vol = np.diff(e1)[:, None] * np.diff(e2)[None, :]
        elif setup.geometry == "rz":
            vol = np.pi * (e1[1:] ** 2 - e1[:-1] ** 2)[:, None] * np.diff(e2)[None, :]
        else:
            raise ValueError("the adjoint covers 2-D gray geometries (xy, rz)")
        self.engine = Engine(setup.geometry, e1, e2, np.ascontiguousarray(vol.T).reshape(-1), seed=setup.seed,
                             capacity=int(setup.n_boundary) * 4 + 1024, device=self.device)
        self.nc = self.nx * self.ny
        dev = self.device
        self.T = torch.full((self.nc,), float(setup.T), dtype=torch.float64, device=dev)
        self.cv = torch.full((self.nc,), float(setup.cv), dtype=torch.float64, device=dev)
        self.faces = []
        for q in range(4):
            Tq = setup.face_T[q] if q < len(setup.face_T) else 0.0
            n = self.ny if q < 2 else self.nx
            self.faces.append(torch.full((n,), float(Tq), dtype=torch.float64, device=dev) if Tq > 0 else None)
        self.refl = tuple(bool(r) for r in setup.reflect) + (False,) * (4 - len(setup.reflect))
        self.lib = _lib.load()
        self.forward_ms = self.backward_ms = None

    def _check_sigma(self, sigma: torch.Tensor) -> torch.Tensor:
        if sigma.shape != (self.nc,):
            raise ValueError(f"sigma must have shape ({self.nc},), cells flattened i + nx*j")
        return sigma.detach().to(self.device, torch.float64).contiguous()

    def forward(self, sigma: torch.Tensor) -> torch.Tensor:
        s = self.setup
        sig = self._check_sigma(sigma)
        eng = self.engine
        eng.bank.size = 0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.transport(self.T, sig, self.cv, None, s.step, s.dt, s.theta, 0, s.n_boundary, 0, self.faces, self.refl,
                      max_events=s.max_events, rz_linear_source=False)
        e1.record()
        e1.synchronize()
        self.forward_ms = e0.elapsed_time(e1)
        return eng.dep[: self.nc].clone()

    def vjp(self, sigma: torch.Tensor, cotangent: torch.Tensor) -> torch.Tensor:
        s = self.setup
        sig = self._check_sigma(sigma)
        cot = cotangent.detach().to(self.device, torch.float64).contiguous()
        eng = self.engine
        eng.bank.size = 0
        grad = torch.zeros(self.nc, dtype=torch.float64, device=self.device)
        mat = _lib.ImcMaterial(self.T.data_ptr(), sig.data_ptr(), self.cv.data_ptr(), None)
        par = eng._params(s.step, s.dt, s.theta, 0, s.n_boundary, 0, self.faces, self.refl, s.max_events, False, 0.0)
        bound = int(self.lib.imc_source_bound(ctypes.byref(eng.cmesh), ctypes.byref(par)))
        eng.bank.ensure(bound + 16)
        wsp, wsn = eng._ws(eng.bank.capacity)
        cb = eng.bank.c()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.check("imc_adjoint_vjp", self.lib.imc_adjoint_vjp(
            ctypes.byref(eng.cmesh), ctypes.byref(mat), ctypes.byref(par), ctypes.byref(cb), cot.data_ptr(),
            grad.data_ptr(), ctypes.byref(eng.ctal), wsp, wsn, eng._stream()))
        e1.record()
        e1.synchronize()
        self.backward_ms = e0.elapsed_time(e1)
        return grad


class IMCDeposition(torch.autograd.Function):
    """dep = IMCDeposition.apply(sigma, problem); backward gives d(g . dep)/d sigma."""

    @staticmethod
    def forward(ctx, sigma: torch.Tensor, problem: AdjointProblem) -> torch.Tensor:
        ctx.problem = problem
        ctx.save_for_backward(sigma)
        return problem.forward(sigma)

    @staticmethod
    def backward(ctx, grad_dep: torch.Tensor):
        (sigma,) = ctx.saved_tensors
        g = ctx.problem.vjp(sigma, grad_dep)
        return g.to(sigma.dtype), None


def deposition(sigma: torch.Tensor, problem: AdjointProblem) -> torch.Tensor:
    return IMCDeposition.apply(sigma, problem)


def opacity_field_problem(n: int = 128, n_histories: int = 4_000_000, device=None) -> tuple[AdjointProblem, np.ndarray]:
    """The 128 x 128 random-opacity benchmark.  Returns (problem, sigma[c]) with cells
    flattened c = i + n*j."""
    edges = np.linspace(0.0, 1.0, n + 1)
    setup = AdjointSetup("xy", edges, edges, T=0.01, cv=0.1, face_T=(1.0, 0.0, 0.0, 0.0),
                         reflect=(False, False, False, False), dt=0.02, n_boundary=int(n_histories))
    g = gaussian_random_field(n)
    sigma = np.exp(g).T.reshape(-1)  # [i, j] -> c = i + n*j
    return AdjointProblem(setup, device), sigma


def fd_check(problem: AdjointProblem, sigma: torch.Tensor, cot: torch.Tensor, cells, rel: float = 1e-3) -> np.ndarray:
    """Central differences of cot . dep with common random numbers (same seed and step)."""
    out = []
    for c in cells:
        h = rel * float(sigma[c])
        sp = sigma.clone(); sp[c] += h
        sm = sigma.clone(); sm[c] -= h
        fp = float(cot @ problem.forward(sp))
        fm = float(cot @ problem.forward(sm))
        out.append((fp - fm) / (2.0 * h))
    return np.array(out)
