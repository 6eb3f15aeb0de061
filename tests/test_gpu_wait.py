"""The bounded device-side wait gives up cleanly.

Every mbarrier wait in the pipelined kernels is bounded (time limit and poll
count); when it runs out the kernel sets a status bit and returns instead of
spinning. Here one warp waits on a barrier that nothing completes, with a
short limit and no copy in flight: the call must return LK_ERR_DEVICE_TIMEOUT
with the timeout bit set, and the device must stay usable (a completed
barrier and an ordinary search run normally afterwards)."""

from __future__ import annotations

import ctypes
import time

import numpy as np
import pytest

from conftest import series
from oracle import lko

pytestmark = pytest.mark.gpu


def _wait(limit_us: int, complete: bool):
    from loki_b200 import _capi as C

    st = ctypes.c_uint32(0)
    t0 = time.perf_counter()
    rc = C.lib().lk_wait_check(limit_us, 1 if complete else 0, ctypes.byref(st), None)
    return rc, st.value, time.perf_counter() - t0


def test_wait_gives_up_and_device_stays_usable(cuda):
    from loki_b200 import _capi as C
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA

    rc, st, _ = _wait(20_000, True)
    assert rc == C.LK_OK and st == 0
    rc, st, secs = _wait(20_000, False)
    assert rc == C.LK_ERR_DEVICE_TIMEOUT
    assert st & 1  # timeout bit
    assert st & (1 << 7)  # set by the check's wait site
    assert "wait gave up" in C.lib().lk_last_error().decode()
    assert secs < 5.0
    # the context is intact: a completed wait and a search still work
    rc, st, _ = _wait(20_000, True)
    assert rc == C.LK_OK and st == 0
    nsamps, nbins, widths = 1 << 16, 32, [1, 2, 3, 4]
    cfg = PulsarSearchConfig(nsamps, 1e-3, nbins, 1.0, np.array([[5.0, 8.0]]), use_fourier=False,
                             score_widths=widths)
    e, v = series(nsamps, 3)
    got = FFACUDA(cfg).scores(e, v)
    op = lko.plan_create(lko.make_cfg(nsamps, 1e-3, nbins, 1.0, [[5.0, 8.0]]))
    want = lko.snr_boxcar_3d(lko.ffa(op, e, v), np.array(widths, np.uint64), nbins).ravel()
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_wait_limit_is_checked(cuda):
    from loki_b200 import _capi as C

    rc, _, _ = _wait(10, False)  # below 1 ms: rejected before any launch
    assert rc == C.LK_ERR_INVALID_ARG
