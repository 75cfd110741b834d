"""The FP64 oracle of the adjoint (d(g . dep)/d sigma) checked against finite differences
of the oracle's own forward step, and the random opacity field / cotangent generators.

  * implicit-capture (path-length) part: with effective scatter negligible (cold material,
    Fleck factor ~1) central differences with common random numbers differentiate the same
    histories, so adjoint and FD agree to round-off: relative 1e-4;
  * likelihood-ratio (effective scatter) part: FD with common random numbers and the
    adjoint are different unbiased estimators of the same derivative; their means over
    independent seeds agree within 4 combined standard errors.
"""
import numpy as np

from oracle import oracle as O


def _setup(n, T, cv, log_mean, log_std, seed=5):
    e1 = np.linspace(0, 1, n + 1)
    e2 = np.linspace(0, 1, n + 1)
    vol = O.flat2d(np.diff(e1)[:, None] * np.diff(e2)[None, :])
    rng = np.random.default_rng(seed)
    sigma = np.exp(log_mean + log_std * rng.standard_normal(n * n))
    cot = rng.standard_normal(n * n)
    cot /= np.linalg.norm(cot)
    return e1, e2, vol, sigma, np.full(n * n, T), np.full(n * n, cv), cot


def _runner(e1, e2, vol, T, cv, n, NB):
    face = [np.full(n, 1.0), None, None, None]
    refl = (False, False, False, False)

    def fwd(sig, seed):
        o = O.Oracle("xy", e1, e2, vol, seed)
        return o.transport(T, sig, cv, None, 0, 0.02, 1.0, 0, NB, 0, face, refl, max_events=1_000_000)["dep"]

    def adj(sig, cot, seed):
        o = O.Oracle("xy", e1, e2, vol, seed)
        o.transport(T, sig, cv, None, 0, 0.02, 1.0, 0, NB, 0, face, refl, max_events=1_000_000, sources_only=True)
        return o.adjoint_vjp(T, sig, cv, 0, 0.02, 1.0, refl, cot, max_events=1_000_000)

    return fwd, adj


def test_oracle_adjoint_matches_fd_pathwise():
    n = 8
    e1, e2, vol, sigma, T, cv, cot = _setup(n, 0.01, 0.1, np.log(5.0), 0.5)
    fwd, adj = _runner(e1, e2, vol, T, cv, n, 20000)
    g = adj(sigma, cot, 77)
    big = 0
    for j in (0, 3, 9, 18, 27, 36, 50):
        h = 1e-4 * sigma[j]
        sp, sm = sigma.copy(), sigma.copy()
        sp[j] += h
        sm[j] -= h
        fd = (cot @ fwd(sp, 77) - cot @ fwd(sm, 77)) / (2 * h)
        if abs(fd) > 1e-9:
            big += 1
            assert abs(g[j] - fd) <= 1e-4 * abs(fd), (j, g[j], fd)
    assert big >= 5


def test_oracle_adjoint_scatter_term_is_unbiased():
    n = 6
    e1, e2, vol, sigma, T, cv, cot = _setup(n, 0.8, 0.01, np.log(3.0), 0.3)
    fwd, adj = _runner(e1, e2, vol, T, cv, n, 8000)
    cells = [0, 7, 20]
    M = 16
    A, F = [], []
    for s in range(M):
        A.append(adj(sigma, cot, 9000 + s)[cells])
        row = []
        for j in cells:
            h = 1e-2 * sigma[j]
            sp, sm = sigma.copy(), sigma.copy()
            sp[j] += h
            sm[j] -= h
            row.append((cot @ fwd(sp, 9000 + s) - cot @ fwd(sm, 9000 + s)) / (2 * h))
        F.append(row)
    A, F = np.array(A), np.array(F)
    for q in range(len(cells)):
        se = np.hypot(A[:, q].std(ddof=1), F[:, q].std(ddof=1)) / np.sqrt(M)
        assert abs(A[:, q].mean() - F[:, q].mean()) <= 4 * se, (cells[q], A[:, q].mean(), F[:, q].mean(), se)


def test_random_opacity_field_and_cotangent():
    from radtranbook_b200 import adjoint

    g = adjoint.gaussian_random_field()
    assert g.shape == (128, 128)
    np.testing.assert_array_equal(g, adjoint.gaussian_random_field())  # seeded
    # one realisation of a field with 0.1 cm correlation: mean within ~3 standard errors of
    # ln 50, spread near 1, correlation at one correlation length near exp(-1/2)
    assert abs(g.mean() - np.log(50.0)) < 0.75
    assert 0.6 < g.std() < 1.4
    lag = 13  # cells of 1/128 cm ~ 0.1 cm
    c = np.mean((g[:-lag] - g.mean()) * (g[lag:] - g.mean())) / g.var()
    assert abs(c - np.exp(-((lag / 128) ** 2) / (2 * 0.01))) < 0.15
    u = adjoint.unit_cotangent(128 * 128)
    assert abs(np.linalg.norm(u) - 1.0) < 1e-12
    np.testing.assert_array_equal(u, adjoint.unit_cotangent(128 * 128))
