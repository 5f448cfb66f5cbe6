"""The device-side failure path, exercised without a fault.

Every mbarrier wait of the split-precision kernel is bounded in time; on
expiry the kernel records SHT_ERR_DEVICE_TIMEOUT in the plan's device error
word and unwinds, and the C-ABI reports the word after the call.  Making a
tensor-core commit never arrive would need a broken program, so
sht_selftest_device_timeout runs the same bounded wait on a shared-memory
barrier that nothing arrives at.  These tests check that the wait gives up
after its limit, that the status comes back through the C-ABI with its
message, that the word is cleared, and that the plan and the context stay
usable."""
import ctypes
import time

import numpy as np
import pytest

from conftest import pkg, relerr

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_reports():
    P = pkg()
    lib = P.load_library()
    s = P.SpmlUtil(64, 32, 1, 21)
    try:
        x = np.random.default_rng(1).standard_normal((3, 32, 64))
        w_before = s.wa_xya(x)
        for limit_ms in (5, 50):
            t0 = time.perf_counter()
            st = lib.sht_selftest_device_timeout(s._h, limit_ms)
            dt = time.perf_counter() - t0
            assert st == 7, (st, lib.sht_last_error())
            assert b"timed out" in lib.sht_last_error()
            assert dt >= limit_ms * 1e-3 * 0.9, dt      # the wait ran to its limit
            assert dt < limit_ms * 1e-3 + 5.0, dt        # and then gave up
            # the word is cleared: the next calls succeed, on both precisions
            assert lib.sht_synchronize(s._h) == 0
            assert np.array_equal(s.wa_xya(x), w_before)
            s.set_precision(P.SHT_PREC_SPLIT)
            assert relerr(s.wa_xya(x), w_before) < 1e-11
            s.set_precision(P.SHT_PREC_FP64)
    finally:
        s.final()


def test_selftest_arguments():
    P = pkg()
    lib = P.load_library()
    s = P.SpmlUtil(64, 32, 1, 21)
    try:
        assert lib.sht_selftest_device_timeout(s._h, 0) == 1
        assert lib.sht_selftest_device_timeout(s._h, 1001) == 1
    finally:
        s.final()
