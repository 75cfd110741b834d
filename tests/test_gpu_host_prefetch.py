"""Host material callables in the gray 2-D drop-in step: the next step's opacity and heat
capacity are evaluated at the new temperature while the comb runs, and a step that passes the
same callables takes them.  Results must equal a run that evaluates them at every step start
(assigning state.temperature drops the prefetched values), and a step that passes another
callable must use that one.  Counts match exactly, temperatures to 1e-12 (deposition is an
integer tally; only the FP64 atomic order of a few per-cell sums differs between runs)."""
import numpy as np
import pytest

from radtranbook_b200 import imc2d, problems

pytestmark = pytest.mark.gpu


def _run(p, n, refresh, sigma_of_step=None):
    st = imc2d.init_simulation(p["Ntarget"], p["Tinit"], p["Tr_init"], p["edges1"], p["edges2"], p["eos_host"],
                               p["inv_eos_host"], geometry="rz", seed=0xAB1)
    out = []
    for k in range(n):
        sig = p["sigma_host"] if sigma_of_step is None else sigma_of_step(k)
        st, info = imc2d.step(st, p["Ntarget"], p["Nboundary"], 0, p["Nmax"], p["T_boundary"], p["dt"],
                              p["edges1"], p["edges2"], sig, p["inv_eos_host"], p["cv_host"], p["source"],
                              reflect=p["reflect"], geometry="rz", boundary_source_func=p["boundary_source_func"])
        out.append((np.array(info["temperature"]), np.array(info["radiation_temperature"]), info["N_particles"],
                    info["profiling"]["transport_events"]["total"]))
        if refresh:
            st.temperature = np.array(st.temperature)  # drops the prefetched opacity
        else:
            assert "_host_next" in st.__dict__
    return out


def _same_runs(a, b):
    # counts exactly; temperatures to 1e-12 (deposition is an integer tally, only the FP64
    # atomic order of a few per-cell sums differs between runs)
    for (T1, Tr1, n1, e1), (T2, Tr2, n2, e2) in zip(a, b):
        np.testing.assert_allclose(T1, T2, rtol=1e-12)
        np.testing.assert_allclose(Tr1, Tr2, rtol=1e-12)
        assert n1 == n2 and e1 == e2


def test_prefetched_host_materials_match_fresh_evaluation(cuda):
    p = problems.crooked_pipe(scale=0.01, nr=30, nz=105)
    _same_runs(_run(p, 4, refresh=False), _run(p, 4, refresh=True))


def test_a_new_opacity_callable_is_used(cuda):
    p = problems.crooked_pipe(scale=0.01, nr=30, nz=105)
    base = p["sigma_host"]
    thick = lambda T: 3.0 * base(T)  # noqa: E731

    def sig(k):
        return base if k < 2 else thick

    got = _run(p, 4, refresh=False, sigma_of_step=sig)
    ref = _run(p, 4, refresh=True, sigma_of_step=sig)
    _same_runs(got, ref)
    plain = _run(p, 4, refresh=True)
    assert not np.array_equal(got[3][0], plain[3][0])  # the opacity change took effect
