"""The device loop's time-step schedule (no GPU): IMC/CrookedPipe2D.py:887-1007 grows dt by a
factor up to dt_max and shortens the step that would pass an unsaved output time so that it
lands on it (and does not grow dt after that step)."""
import numpy as np

from radtranbook_b200.driver import adaptive_schedule


def test_schedule_lands_on_output_times_and_grows_geometrically():
    steps, nxt = adaptive_schedule(0.0, [0.01, 0.03], dt_initial=0.001, dt_max=0.004, growth=1.5)
    dts = [dt for dt, _ in steps]
    t = np.cumsum(dts)
    outs = [(k, o) for k, (_, o) in enumerate(steps) if o is not None]
    assert [o for _, o in outs] == [0.01, 0.03]
    for k, o in outs:
        assert abs(t[k] - o) < 1e-12
    # geometric growth 0.001, 0.0015, 0.00225, 0.003375, then capped at 0.004
    np.testing.assert_allclose(dts[:4], [0.001, 0.0015, 0.00225, 0.003375], rtol=1e-15)
    assert max(dts) <= 0.004 + 1e-15
    # the step that was cut to land on 0.01 does not grow dt: the next one starts from the same dt
    k0 = outs[0][0]
    assert dts[k0] < 0.004 and abs(dts[k0 + 1] - 0.004) < 1e-15
    assert abs(t[-1] - 0.03) < 1e-12 and nxt == 0.004


def test_schedule_resumes_with_saved_outputs():
    """A restart passes the outputs already saved; the schedule continues to the last one."""
    steps, _ = adaptive_schedule(0.01, [0.01, 0.02], dt_initial=0.004, dt_max=0.004, growth=1.1, saved={0.01})
    t = 0.01 + np.cumsum([dt for dt, _ in steps])
    assert abs(t[-1] - 0.02) < 1e-12 and steps[-1][1] == 0.02
