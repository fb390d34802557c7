"""Failure detection on the device without a fault: the fused band sweep's
bounded waits.  A test-only entry point makes CTA 0 withhold one staged row
and shortens the wait limit, so the wait for that row runs out; the kernel
sets MQV_ERR_TIMEOUT, lets its issued copies land and returns.  The call
that reads the device status reports TIMEOUT, the handle then refuses
compute until its state is set again, and after that it runs sweeps equal
to the oracle's.  Nothing waits without a bound, nothing faults."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_band_wait_timeout_is_reported_and_recovered(orc):
    import marqov_b200 as M
    from marqov_b200 import _lib
    L, beta, seed = 8192, 0.44068679, 31
    cfg = M.Config(seed=seed, repid=0, ncluster=0, nmetro=1)
    with M.makeCore(M.RegularHypercubic(L, 2), cfg, M.Ising(-1.0), beta) as c:
        c.init()
        s0 = c.state
        _lib.check(c._lib.mqv_selftest_inject_timeout(c.handle, 3, 200_000))  # 200 us
        with pytest.raises(M.MarqovError) as ei:
            c.emcs(1, ncluster=0, nmetro=1)
        assert ei.value.status == _lib.ERR_TIMEOUT
        with pytest.raises(M.MarqovError) as ei:
            c.emcs(1, ncluster=0, nmetro=1)
        assert ei.value.status == _lib.ERR_STATE
        with pytest.raises(M.MarqovError):
            _ = c.state
        # recovery: the state set again, the sweeps go on from the counters
        c.state = s0
        sweep, _ = c.counters
        assert "ising2d_band" in c.describe()
        obs, _ = c.emcs(2, ncluster=0, nmetro=1)
        final = c.state
    s = s0.copy()
    for t in range(2):
        orc.ising2d_sweep(L, -1.0, s, beta, seed, 0, sweep + t)
    assert (final == s).all()
    assert np.isfinite(obs).all()


def test_injection_needs_the_band_path():
    import marqov_b200 as M
    from marqov_b200 import _lib
    with M.makeCore(M.RegularHypercubic(64, 2), M.Config(seed=1), M.Ising(-1.0), 0.4) as c:
        assert c._lib.mqv_selftest_inject_timeout(c.handle, 3, 1000) == _lib.ERR_UNSUPPORTED_TERM
