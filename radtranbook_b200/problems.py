"""Benchmark workloads of the IMC engine, as reference-style problem definitions.

Each function returns a dict with the mesh, material callables (host NumPy versions, as a
reference driver writes them, and device versions) and the step parameters, so the same
problem can be run through the drop-in API, the device engine or the CPU oracle.

  marshak_slab   1-D gray slab Marshak wave: 0.20 cm, 100 cells, sigma = 300 T^-3,
                 cv = 0.3, 1 keV left face, T0 = 1e-3 keV, dt 0.01 ns x 100
                 (IMC/MarshakWave.py setup; 20k emission + 20k boundary / step, NMax 80k)
  crooked_pipe   2-D RZ crooked pipe: r in [0,2], z in [0,7] on 60x210; pipe sigma 0.2,
                 cv 0.001; wall sigma 2000, cv 0.5; 0.5 keV on z=0 for r<0.5; reflect r=0;
                 T0 = 0.05 keV; dt 0.01 ns x 100; 2e6 source particles per step split 2:1
                 emission:boundary, Nmax 6.67e6 (IMC/CrookedPipe2D.py geometry)
  mg_crooked_pipe  2-D RZ multigroup crooked pipe (MG_IMC/problems/crooked_pipe_multigroup_imc.py
                 with its command-line defaults; see the function)
  marshak_mg     multigroup Marshak wave, 200 cells x 10 groups, 1e6 particles per step, on the
                 2-D multigroup step (MG_IMC/problems/test_marshak_wave_multigroup_powerlaw.py
                 set-up with sigma_g clamped to [1e-2, 1e6]; see the function)
"""
from __future__ import annotations

import numpy as np
import torch

from .materials import Constant, GroupedOpacity, GroupPowerLawOpacity, LinearEOS, PowerLawOpacity, device_callable


def marshak_slab(scale: float = 1.0) -> dict:
    I = 100
    L = 0.20
    mesh = np.array([[i * L / I, (i + 1) * L / I] for i in range(I)])
    cv_val = 0.3

    def sigma_host(T):
        return 300.0 * np.power(T, -3.0)

    # device versions: parametric materials the step evaluates on the device itself
    eos = LinearEOS(cv_val)
    return dict(
        name="1-D gray slab Marshak wave (100 cells, sigma=300 T^-3)",
        geometry="slab", mesh=mesh, dim=1,
        Tinit=np.full(I, 0.001), Tr_init=np.full(I, 0.001),
        sigma_host=sigma_host, sigma_dev=PowerLawOpacity(300.0, 3.0),
        cv_host=lambda T: np.full_like(T, cv_val), cv_dev=eos.cv,
        eos_host=lambda T: cv_val * T, inv_eos_host=lambda e: e / cv_val,
        eos_dev=eos.eos, inv_eos_dev=eos.inv_eos,
        Ntarget=int(20000 * scale), Nboundary=int(20000 * scale), Nsource=0, Nmax=int(80000 * scale),
        T_boundary=(1.0, 0.0), reflect=(False, False), dt=0.01, n_steps=100, source=np.zeros(I),
    )


def crooked_pipe_thin(r: np.ndarray, z: np.ndarray) -> np.ndarray:
    """Pipe (optically thin) region map, evaluated at cell centres."""
    return (((r < 0.5) & (z >= 0.0) & (z <= 3.0))
            | ((r >= 0.5) & (r < 1.5) & (z >= 2.5) & (z <= 3.0))
            | ((r >= 1.0) & (r <= 1.5) & (z >= 3.0) & (z <= 4.0))
            | ((r >= 0.5) & (r < 1.5) & (z >= 4.0) & (z <= 4.5))
            | ((r < 0.5) & (z >= 4.0) & (z <= 7.0)))


def crooked_pipe(scale: float = 1.0, nr: int = 60, nz: int = 210) -> dict:
    r_edges = np.linspace(0.0, 2.0, nr + 1)
    z_edges = np.linspace(0.0, 7.0, nz + 1)
    rc = 0.5 * (r_edges[:-1] + r_edges[1:])
    zc = 0.5 * (z_edges[:-1] + z_edges[1:])
    R, Z = np.meshgrid(rc, zc, indexing="ij")
    thin = crooked_pipe_thin(R, Z)
    sig = np.where(thin, 0.2, 2000.0)
    cvg = np.where(thin, 0.001, 0.5)
    # device versions: parametric materials (per-cell constants, linear EOS) the step
    # evaluates on the device itself
    eos = LinearEOS(cvg)
    sigma_dev, cv_dev, eos_dev, inv_eos_dev = Constant(sig), eos.cv, eos.eos, eos.inv_eos

    def bsf(r, z, side):
        return 0.5 if (side == "zmin" and r < 0.5) else 0.0

    n_src = int(round(2e6 * scale))
    n_bnd = n_src // 3
    return dict(
        name="2-D RZ gray crooked pipe (60x210)",
        geometry="rz", dim=2, edges1=r_edges, edges2=z_edges,
        Tinit=np.full((nr, nz), 0.05), Tr_init=np.full((nr, nz), 0.05),
        sigma_host=lambda T: sig.copy(), sigma_dev=sigma_dev,
        cv_host=lambda T: cvg.copy(), cv_dev=cv_dev,
        eos_host=lambda T: cvg * T, inv_eos_host=lambda e: e / cvg,
        eos_dev=eos_dev, inv_eos_dev=inv_eos_dev,
        Ntarget=n_src - n_bnd, Nboundary=n_bnd, Nsource=0, Nmax=int(round(6.67e6 * scale)),
        T_boundary=(0.0, 0.0, 0.0, 0.0), reflect=(True, False, False, False), boundary_source_func=bsf,
        dt=0.01, n_steps=100, source=np.zeros((nr, nz)), thin=thin,
        fiducials={"r=0,z=0.25": (0.0, 0.25), "r=0,z=2.75": (0.0, 2.75), "r=1.25,z=3.5": (1.25, 3.5),
                   "r=0,z=4.25": (0.0, 4.25), "r=0,z=6.75": (0.0, 6.75)},
    )


def mg_crooked_pipe_thick(r: np.ndarray, z: np.ndarray) -> np.ndarray:
    """Wall (optically thick) map of the multigroup crooked pipe, at cell centres
    (MG_IMC/problems/crooked_pipe_multigroup_imc.py:185-208)."""
    thin = (((r < 0.5) & ((z < 3.0) | (z > 4.0))) | ((r < 1.5) & (z > 2.5) & (z < 3.0))
            | ((r < 1.5) & (z > 4.0) & (z < 4.5)) | ((r >= 1.0) & (r < 1.5) & (z > 2.5) & (z < 4.5)))
    return ~thin


def mg_crooked_pipe(n_groups: int = 10, nr: int = 60, nz: int = 210, mode: str = "standard",
                    bc_T: float = 0.5) -> dict:
    """The multigroup crooked pipe of MG_IMC/problems/crooked_pipe_multigroup_imc.py with its
    command-line defaults: r in [0,2] x z in [0,7] cm, wall density 2, pipe density 0.1 g/cm^3,
    e = 0.05 rho T, sigma_g(T) = sqrt(sigma(T, E_g) sigma(T, E_g+1)) with
    sigma(T, E) = min(10 rho max(T, 0.01)^-1/2 E^-3, 1e14), groups log-spaced on [0.01, 10] keV,
    T0 = 0.05 keV, a 0.5 keV blackbody surface source on z = 0 for r < 0.5, reflecting axis,
    emission only from cells above 0.075 keV, dt from 1e-4 ns growing by 1.1 to 0.01 ns, and the
    driver's particle presets ('quick' 20k + 20k per step, Nmax 1e5 + 1e4 per step to 5e5;
    'standard' 200k + 200k, Nmax 1e6 + 5e4 per step to 5e6)."""
    r_edges = np.linspace(0.0, 2.0, nr + 1)
    z_edges = np.linspace(0.0, 7.0, nz + 1)
    rc = 0.5 * (r_edges[:-1] + r_edges[1:])
    zc = 0.5 * (z_edges[:-1] + z_edges[1:])
    R, Z = np.meshgrid(rc, zc, indexing="ij")
    rho = np.where(mg_crooked_pipe_thick(R, Z), 2.0, 0.1)
    cvg = 0.05 * rho
    edges = np.logspace(np.log10(1e-2), np.log10(10.0), n_groups + 1)
    cache = {}

    def dev(a, T):
        key = (id(a), T.device)
        if key not in cache:
            cache[key] = torch.as_tensor(a, dtype=torch.float64, device=T.device)
        return cache[key]

    def opacity(g):
        lo, hi = float(edges[g]), float(edges[g + 1])

        def host(T):
            Ts = np.maximum(T, 1e-2) ** -0.5
            return np.sqrt(np.minimum(10.0 * rho * Ts * lo ** -3, 1e14) * np.minimum(10.0 * rho * Ts * hi ** -3, 1e14))

        @device_callable
        def device(T):
            Ts = torch.pow(torch.clamp(T, min=1e-2), -0.5)
            rh = dev(rho, T)
            return torch.sqrt(torch.clamp(10.0 * rh * Ts * lo ** -3, max=1e14)
                              * torch.clamp(10.0 * rh * Ts * hi ** -3, max=1e14))
        return host, device

    ops = [opacity(g) for g in range(n_groups)]
    # On the device: 10 rho max(T, 0.01)^-1/2 (E_g E_g+1)^-3/2, the same function as the
    # geometric mean above wherever the 1e14 cap does not bind, which is everywhere on this
    # problem (10 rho max(T, 0.01)^-1/2 E^-3 <= 10 * 2 * 10 * 0.01^-3 = 2e8); a material law
    # the multigroup step evaluates in its material update kernel.
    sigma_dev = GroupPowerLawOpacity(10.0, 0.5, (edges[:-1] * edges[1:]) ** -1.5, scale=rho, T_floor=1e-2)
    eos = LinearEOS(cvg)
    presets = {"quick": (20_000, 20_000, 100_000, 10_000, 500_000),
               "standard": (200_000, 200_000, 1_000_000, 50_000, 5_000_000)}
    nt, nb, nmax, ngrow, nfin = presets[mode]

    def bsf(r, z, side):
        return bc_T if (side == "zmin" and r < 0.5) else 0.0

    return dict(
        name=f"2-D RZ multigroup crooked pipe ({nr}x{nz}, {n_groups} groups)",
        geometry="rz", dim=2, edges1=r_edges, edges2=z_edges, energy_edges=edges, rho=rho,
        Tinit=np.full((nr, nz), 0.05), Tr_init=np.full((nr, nz), 0.05),
        sigma_host=[h for h, _ in ops], sigma_dev=sigma_dev, sigma_dev_callables=[d for _, d in ops],
        cv_host=lambda T: cvg.copy(), cv_dev=eos.cv,
        eos_host=lambda T: cvg * T, inv_eos_host=lambda e: e / cvg,
        eos_dev=eos.eos, inv_eos_dev=eos.inv_eos,
        Ntarget=nt, Nboundary=nb, Nsource=0, Nmax=nmax, Nmax_growth=ngrow, Nmax_final=nfin,
        T_boundary=(0.0, 0.0, 0.0, 0.0), reflect=(True, False, False, False), boundary_source_func=bsf,
        T_emit_floor=0.075, dt_initial=1e-4, dt_max=0.01, dt_growth=1.1, source=np.zeros((nr, nz)),
        fiducials={"r=0,z=0.25": (0.0, 0.25), "r=0,z=2.75": (0.0, 2.75), "r=1.25,z=3.5": (1.25, 3.5),
                   "r=0,z=4.25": (0.0, 4.25), "r=0,z=6.75": (0.0, 6.75)},
    )


def marshak_mg(scale: float = 1.0) -> dict:
    """1-D multigroup Marshak wave run through the 2-D multigroup step (MG_IMC2D on an XY strip,
    reflecting in y): slab 0.5 cm in 200 cells, 10 groups with edges log-spaced on [1e-4, 20]
    keV, sigma_g(T) = clamp(10 nu_g^-3 T^-1/2, 1e-2, 1e6) with nu_g the arithmetic group
    midpoint, cv = 0.3, a 1 keV source on the left face, T0 = 0.001 keV, dt = 0.005 ns,
    1e6 particles per step split 2:1 between emission and the boundary, Nmax 1.33e6."""
    nx = 200
    e1 = np.linspace(0.0, 0.5, nx + 1)
    e2 = np.array([0.0, 1.0])
    edges = np.logspace(-4, np.log10(20.0), 11)
    nu = 0.5 * (edges[:-1] + edges[1:])
    cv_val = 0.3

    def one(g):
        k = 10.0 * nu[g] ** -3

        def host(T):
            return np.clip(k * np.power(T, -0.5), 1e-2, 1e6)

        @device_callable
        def dev(T):
            return torch.clamp(k * torch.pow(T, -0.5), min=1e-2, max=1e6)
        return host, dev

    ops = [one(g) for g in range(10)]
    # on the device as a material law the multigroup step evaluates in its material update
    # kernel: clamp(10 T^-1/2 nu_g^-3, 1e-2, 1e6), the host callables' function (the products
    # in another order, so equal to rounding)
    sigma_dev = GroupPowerLawOpacity(10.0, 0.5, nu ** -3, lo=1e-2, hi=1e6)
    eos = LinearEOS(cv_val)

    return dict(
        name="multigroup Marshak wave (200 cells, 10 groups) on the 2-D multigroup step",
        geometry="xy", dim=2, edges1=e1, edges2=e2, energy_edges=edges,
        Tinit=np.full((nx, 1), 0.001), Tr_init=np.full((nx, 1), 0.001),
        sigma_host=[h for h, _ in ops], sigma_dev=sigma_dev, sigma_dev_callables=[d for _, d in ops],
        cv_host=lambda T: np.full_like(T, cv_val), cv_dev=eos.cv,
        eos_host=lambda T: cv_val * T, inv_eos_host=lambda e: e / cv_val,
        eos_dev=eos.eos, inv_eos_dev=eos.inv_eos,
        Ntarget=int(666667 * scale), Nboundary=int(333333 * scale), Nsource=0, Nmax=int(1330000 * scale),
        T_boundary=(1.0, 0.0, 0.0, 0.0), reflect=(False, False, True, True), dt=0.005, n_steps=200,
        source=np.zeros((nx, 1)),
    )
