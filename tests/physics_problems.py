"""Set-ups of the analytic gray benchmarks, shared by the oracle (CPU) and GPU tests.

Su–Olson non-equilibrium slab (the reference's IMC/SuOlson.py set-up, run with IMC1D step
semantics): sigma = 1, e = a T^4 (cv = 4 a T^3), source a c for x <= 0.5, reflecting left
face, vacuum right face, slab length 1.5 (0.5 + tau), 50 cells, dt = 0.0005 ns, 10^4
emission and 2x10^4 source particles per step; T^4 and Tr^4 are the normalised material and
radiation energy densities of the analytic solution.

0-D equilibration (IMC/0-DTests.py set-up): one reflecting cell, sigma = 1, cv = 0.01,
T0 = 0.4 keV, Tr0 = 1 keV; the exact solution is the exchange ODE
d(a Tr^4)/dt = -a c sigma (Tr^4 - T^4) = -d(cv T)/dt.
"""
import ast
import os

import numpy as np

A_RAD, C_LIGHT = 0.01372, 29.98
SU_OLSON_TAUS = [0.1, 0.31623, 1.0, 3.16228, 10.0, 31.62278, 100.0]


def su_olson(tau=1.0):
    L = 1.5 * (0.5 + tau)
    e1 = np.linspace(0.0, L, 51)
    mid = 0.5 * (e1[:-1] + e1[1:])
    return dict(edges=e1, mid=mid, T0=np.full(50, 1e-8), source=np.where(mid <= 0.5, A_RAD * C_LIGHT, 0.0),
                dt=0.0005, steps=int(round(tau / C_LIGHT / 0.0005)), Ntarget=10000, Nsource=20000, Nmax=200000,
                sigma=lambda T: 1.0 + 0.0 * T, eos=lambda T: A_RAD * T ** 4,
                inv_eos=lambda u: (np.maximum(u, 0.0) / A_RAD) ** 0.25, cv=lambda T: 4.0 * A_RAD * T ** 3)


def su_olson_tables(ref_root):
    """(radiation, material) analytic tables from the reference checkout: rows x, columns
    SU_OLSON_TAUS (IMC/SuOlson.py:22-38 and IMC/Su_Olson_Material.csv)."""
    src = open(os.path.join(ref_root, "IMC", "SuOlson.py")).read()
    rad = None
    for node in ast.parse(src).body:
        if (isinstance(node, ast.Assign) and getattr(node.targets[0], "id", "") == "rad_data"
                and isinstance(node.value, ast.List)):
            rad = np.array(ast.literal_eval(node.value), dtype=np.float64)
            break
    mat = np.loadtxt(os.path.join(ref_root, "IMC", "Su_Olson_Material.csv"), delimiter=",")
    return rad, mat


def zero_d(dt=0.002, t_final=0.375):
    cv = 0.01
    return dict(edges=np.array([0.0, 0.1]), T0=0.4, Tr0=1.0, cv=cv, dt=dt, steps=int(round(t_final / dt)),
                Ntarget=4000, Nmax=20000, sigma=lambda T: 1.0 + 0.0 * T, eos=lambda T: cv * T,
                inv_eos=lambda u: u / cv, cvf=lambda T: cv + 0.0 * T)


def zero_d_exact(p, times):
    from scipy.integrate import solve_ivp

    cv = p["cv"]

    def rhs(t, y):
        T = y[1] / cv
        Tr4 = max(y[0], 0.0) / A_RAD
        em = A_RAD * C_LIGHT * (Tr4 - T ** 4)
        return [-em, em]

    sol = solve_ivp(rhs, [0.0, times[-1] * (1 + 1e-12)], [A_RAD * p["Tr0"] ** 4, cv * p["T0"]], t_eval=times,
                    rtol=1e-10, atol=1e-14)
    return sol.y[1] / cv, (sol.y[0] / A_RAD) ** 0.25


def zero_d_mg_exact(edges, sigmas, cv, T0, Tr0, times):
    """0-D multigroup exchange: dE_g/dt = c sigma_g (a T^4 b_g(T) - E_g), cv dT/dt = -sum_g of
    the same, with b_g the normalised Planck fractions over the groups (as the MG step emits)
    and E_g(0) = a Tr0^4 b_g(Tr0).  Returns T(t), Tr(t) = (sum_g E_g / a)^(1/4)."""
    from scipy.integrate import solve_ivp

    from radtranbook_b200.mg_imc2d import planck_fractions

    sig = np.asarray(sigmas, dtype=np.float64)
    G = len(sig)

    def rhs(t, y):
        T = y[G] / cv
        b = planck_fractions(edges, np.array([T])).reshape(G)
        ex = C_LIGHT * sig * (A_RAD * T ** 4 * b - y[:G])
        return np.concatenate([ex, [-ex.sum()]])

    b0 = planck_fractions(edges, np.array([Tr0])).reshape(G)
    y0 = np.concatenate([A_RAD * Tr0 ** 4 * b0, [cv * T0]])
    sol = solve_ivp(rhs, [0.0, times[-1] * (1 + 1e-12)], y0, t_eval=times, rtol=1e-9, atol=1e-14, method="LSODA")
    return sol.y[G] / cv, (np.clip(sol.y[:G].sum(0), 0.0, None) / A_RAD) ** 0.25


def marshak_self_similar(x, t, T_bc=1.0, cv=0.3, sigma_coef=300.0):
    """Self-similar Marshak wave for sigma = sigma_coef T^-3, e = cv T (IMC/MarshakWave2D.py:
    187-209; profile constants xi_max = 1.11305, omega = 0.05989)."""
    xi_max, omega = 1.11305, 0.05989
    K = 8.0 * A_RAD * C_LIGHT / (7.0 * 3.0 * sigma_coef * T_bc ** -3 * cv)
    xi = np.asarray(x) / np.sqrt(K * max(float(t), 1e-30))
    return np.where(xi < xi_max, T_bc * np.power(np.maximum((1.0 - xi / xi_max) * (1.0 + omega * xi / xi_max), 1e-30),
                                                  1.0 / 6.0), 0.0)
