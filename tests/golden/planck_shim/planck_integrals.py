"""Stand-in for the external `planck_integrals` extension imported by MG_IMC/MG_IMC2D.py:62
(not part of the reference tree), used only when recording golden fixtures from the
reference: group Planck integrals by adaptive quadrature (SciPy), so the reference runs
with real Planck group fractions instead of its equal-split fallback.  The reference only
uses ratios B_g / sum_g B_g, so the common normalisation a c / (4 pi) is kept."""
import numpy as np
from scipy.integrate import quad

_C = 29.98 * 0.01372 / (4.0 * np.pi)
_cache = {}


def _frac(x0, x1):
    key = (float(x0), float(x1))
    if key not in _cache:
        f = lambda t: t ** 3 / np.expm1(t) if t > 0 else 0.0  # noqa: E731
        _cache[key] = 15.0 / np.pi ** 4 * quad(f, x0, x1, epsabs=0.0, epsrel=1e-12, limit=200)[0]
    return _cache[key]


def Bg(E_low, E_high, T):
    T = np.asarray(T, dtype=np.float64)
    out = np.zeros_like(T)
    it = np.nditer(T, flags=["multi_index"])
    for t in it:
        t = float(t)
        if t > 0:
            out[it.multi_index] = _C * t ** 4 * _frac(E_low / t, E_high / t) * np.pi ** 4 / 15.0
    return out if out.ndim else float(out)


def dBgdT(E_low, E_high, T, h=1e-6):
    T = np.asarray(T, dtype=np.float64)
    return (Bg(E_low, E_high, T * (1 + h)) - Bg(E_low, E_high, T * (1 - h))) / (2 * h * T)


def Bg_multigroup(energy_edges, T):
    return np.array([Bg(energy_edges[g], energy_edges[g + 1], T) for g in range(len(energy_edges) - 1)])


def dBgdT_multigroup(energy_edges, T):
    return np.array([dBgdT(energy_edges[g], energy_edges[g + 1], T) for g in range(len(energy_edges) - 1)])
