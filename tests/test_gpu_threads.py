"""Concurrent host threads, as the reference issues its per-level calls from
OpenMP threads (e.g. HBEBaroc_hspm_vfvm_mod.f90:388, SpmlUtil_mod.f90:360-366):
the C-ABI is re-entrant, calls on one plan are serialised by the plan, calls
on different plans run side by side, and each thread keeps its own last error.

Each thread transforms single levels through the host-pointer entry points
(ctypes releases the interpreter lock during the call); the results are
compared with the oracle at the FP64 tolerance, 1e-11 per field.
"""
import ctypes
import threading

import numpy as np
import pytest

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _run_threads(fns):
    errors = []

    def wrap(fn):
        try:
            fn()
        except BaseException as e:  # noqa: BLE001 - reported below
            errors.append(e)

    ts = [threading.Thread(target=wrap, args=(f,)) for f in fns]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in ts), "a thread did not finish"
    if errors:
        raise errors[0]


def test_per_level_calls_from_many_threads_on_one_plan():
    W = workloads()
    I, J, N = W.GRIDS["T42"]
    sp = pkg().SpmlUtil(I, J, 24, N)
    ora = O.OraclePlan(I, J, N)
    try:
        K = 24
        w = W.seeded_spectra(N, K, 1.5, seed=41)
        ref_g = ora.xya_wa(w)
        ref_w = ora.wa_xya(ref_g)
        out_g = np.zeros((K, J, I))
        out_w = np.zeros((K, sp.lm))

        def worker(t):
            def run():
                for rep in range(3):
                    for k in range(t, K, 8):
                        out_g[k] = sp.xy_w(w[k])
                        out_w[k] = sp.w_xy(out_g[k])
            return run

        _run_threads([worker(t) for t in range(8)])
        assert relerr(out_g, ref_g) < TOL
        assert relerr(out_w, ref_w) < TOL
    finally:
        sp.final()


def test_threads_on_different_plans_and_private_errors():
    W = workloads()
    P = pkg()
    grids = [W.GRIDS["T21"], W.GRIDS["T42"], W.GRIDS["T85"]]
    plans = [P.SpmlUtil(I, J, 8, N) for I, J, N in grids]
    lib = P.load_library()
    try:
        results = {}
        ws = [W.seeded_spectra(N, 8, 2.0, seed=50 + i) for i, (I, J, N) in enumerate(grids)]
        refs = [O.OraclePlan(I, J, N).xya_wa(w) for (I, J, N), w in zip(grids, ws)]

        def good(i):
            def run():
                for _ in range(4):
                    g = plans[i].xya_wa(ws[i])
                    back = plans[i].wa_xya(g)
                results[i] = (relerr(back, ws[i]), relerr(g, refs[i]))
            return run

        def bad():
            buf = (ctypes.c_double * 8)()
            for _ in range(50):
                assert lib.sht_wa_xya(plans[0]._h, buf, -1, buf) == 1  # SHT_ERR_INVALID_ARG
                assert b"nb" in lib.sht_last_error()

        before = lib.sht_last_error()
        _run_threads([good(0), good(1), good(2), bad])
        for i in range(3):
            rt, vs_oracle = results[i]
            assert rt < TOL and vs_oracle < TOL, (grids[i], rt, vs_oracle)
        # the failing thread's message did not reach this thread
        assert lib.sht_last_error() == before
    finally:
        for p in plans:
            p.final()
