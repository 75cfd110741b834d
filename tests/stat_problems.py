"""Shared setups for the statistical parity tests: the same reduced problems the golden
generator ran through the reference (tests/golden/make_golden.py: run_stats_slab,
run_stats_rz), expressed for the oracle and for the GPU drop-in API."""
import numpy as np

# the number of steps of each run is read from its fixture ("steps")
SLAB = dict(I=100, dx=0.002, cv=0.3, Ntarget=2000, Nboundary=2000, NMax=8000, dt=0.01, T0=0.001)
RZ = dict(nr=30, nz=105, Ntarget=6000, Nboundary=3000, Nmax=30000, dt=0.01, T0=0.05)


def slab_mesh():
    I, dx = SLAB["I"], SLAB["dx"]
    return np.array([[i * dx, (i + 1) * dx] for i in range(I)])


def rz_setup():
    nr, nz = RZ["nr"], RZ["nz"]
    r_e = np.linspace(0, 2, nr + 1)
    z_e = np.linspace(0, 7, nz + 1)
    rc = 0.5 * (r_e[:-1] + r_e[1:])
    zc = 0.5 * (z_e[:-1] + z_e[1:])
    R, Z = np.meshgrid(rc, zc, indexing="ij")
    thin = (((R < 0.5) & (Z <= 3.0)) | ((R >= 0.5) & (R < 1.5) & (Z >= 2.5) & (Z <= 3.0))
            | ((R >= 1.0) & (R <= 1.5) & (Z >= 3.0) & (Z <= 4.0)) | ((R >= 0.5) & (R < 1.5) & (Z >= 4.0) & (Z <= 4.5))
            | ((R < 0.5) & (Z >= 4.0)))
    sig = np.where(thin, 0.2, 2000.0)
    cvg = np.where(thin, 0.001, 0.5)
    face = np.where(rc < 0.5, 0.5, 0.0)
    return r_e, z_e, sig, cvg, face


def compare_means(mean_a, se_a, mean_b, se_b, roi, z_max=4.5, frac_3sigma=0.08):
    """Two independent Monte Carlo estimates agree cell by cell within combined errors."""
    se = np.sqrt(se_a ** 2 + se_b ** 2) + 1e-300
    z = np.abs(mean_a - mean_b)[roi] / se[roi]
    assert roi.sum() >= 5, "too few cells in the region of interest"
    assert np.max(z) < z_max, (np.max(z), np.argmax(z))
    assert np.mean(z > 3.0) <= frac_3sigma, np.mean(z > 3.0)
    return z
