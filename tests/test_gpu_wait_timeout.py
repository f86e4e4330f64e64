"""The failure path of the bounded waits: every TMA-fed kernel waits on its copies through a
bounded mbarrier wait that, when it runs out, raises a device flag the host turns into
BD_ERR_TIMEOUT. Here a wait on a barrier that nothing completes runs out (after a short, fixed
number of polls) and the status comes back; the control case completes; and the context stays
usable: a normal stencil call afterwards gives the same result as before."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stencil(gpu):
    rng = np.random.default_rng(3)
    n = (8, 10, 16)
    T0 = 25 + 40 * rng.random(n); Q = rng.random(n) * 1e-3
    K = 1e-4 + 5e-4 * rng.random(n); R = 2e-3 + 2e-3 * rng.random(n)
    return gpu.run_thermal3d_substeps_gpu(T0, Q, K, R, *n, 0.015, 0.015, 0.015, 5e-5, 4, h_eff=2e-5,
                                          t_ambient=25.0, is_active=1)


def test_bounded_wait_times_out_and_the_context_survives(gpu):
    from bug_defense_b200 import _lib
    before = _stencil(gpu)
    t0 = time.perf_counter()
    with pytest.raises(_lib.BugdefError) as exc:
        _lib.call("bd_selftest_wait_timeout", 2000, 0, _lib.stream_ptr())
    assert exc.value.code == _lib.BD_ERR_TIMEOUT
    assert "gave up" in str(exc.value)
    assert time.perf_counter() - t0 < 10.0
    _lib.call("bd_selftest_wait_timeout", 2000, 1, _lib.stream_ptr())   # completed barrier: no timeout
    with pytest.raises(ValueError):
        _lib.call("bd_selftest_wait_timeout", 0, 0, _lib.stream_ptr())
    after = _stencil(gpu)
    assert np.array_equal(before, after)
