"""The allocation-free analysis entry point, sht_wa_xya_dev_noalloc.

It serves callers that must not allocate device memory while they run.  Those
are hosts whose GPU memory belongs to another pool allocator, time loops that
cannot take the synchronisation cudaMalloc may cause, and hosts that forbid
allocation after start-up.  Its output must match the ordinary device entry
point, sht_wa_xya_dev, and the oracle's analysis on two calls in a row.  Two calls matter because the
fixed scratch array keeps the first call's data.  A batch larger than the
fixed scratch must be refused cleanly.

This file is collected last so that a run stopping at the first failure has
already run every other test.  It builds its own plan and inputs, so it also
passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11
VP = ctypes.c_void_p


def _lib():
    lib = pkg().load_library()
    lib.sht_wa_xya_dev_noalloc.argtypes = [VP, VP, ctypes.c_int, VP]
    lib.sht_wa_xya_dev_noalloc.restype = ctypes.c_int
    lib.sht_noalloc_scratch_bytes.restype = ctypes.c_ulonglong
    return lib


def test_noalloc_matches_device_entry_point_twice():
    import torch

    P, W = pkg(), workloads()
    lib = _lib()
    I, J, N = W.GRIDS["T85"]
    nb = 48
    sht = P.SpmlUtil(I, J, nb, N, None, 6.371e6)
    try:
        stream = torch.cuda.current_stream()
        assert lib.sht_set_stream(sht._h, VP(stream.cuda_stream)) == 0
        for call, seed in enumerate((101, 202)):
            w = torch.from_numpy(W.seeded_spectra(N, nb, 2.0, seed=seed)).cuda()
            grid = sht.xya_wa(w)  # device grid from the ordinary synthesis
            ref = torch.empty((nb, (N + 1) ** 2), dtype=torch.float64, device="cuda")
            out = torch.full_like(ref, float("nan"))
            assert lib.sht_wa_xya_dev(sht._h, VP(grid.data_ptr()), nb, VP(ref.data_ptr())) == 0
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            st = lib.sht_wa_xya_dev_noalloc(sht._h, VP(grid.data_ptr()), nb, VP(out.data_ptr()))
            assert st == 0, lib.sht_last_error()
            torch.cuda.synchronize()
            if call == 1:
                # the call's whole contract: no device memory is taken (the
                # first call may still load the module that holds the array)
                assert torch.cuda.mem_get_info()[0] == free_before, "the call allocated device memory"
            o, r = out.cpu().numpy(), ref.cpu().numpy()
            assert np.isfinite(o).all(), f"call {call}: non-finite output"
            assert relerr(o, r) < TOL, f"call {call}: {relerr(o, r)}"
            assert relerr(o, w.cpu().numpy()) < TOL, f"call {call}: round trip"
            # and against the oracle's analysis of the same grid
            assert relerr(o, O.OraclePlan(I, J, N, 6.371e6).wa_xya(grid.cpu().numpy())) < TOL, f"call {call}: oracle"
    finally:
        sht.final()


def test_noalloc_setup_call_with_no_field_levels():
    """A call with nb = 0 only looks up the scratch array (loading its module
    on the device's first lookup), so a host can make it at start-up, before
    another pool takes the GPU's memory; after it, a real call takes no memory."""
    import torch

    P, W = pkg(), workloads()
    lib = _lib()
    I, J, N = W.GRIDS["T42"]
    nb = 16
    sht = P.SpmlUtil(I, J, nb, N, None, 1.0)
    try:
        stream = torch.cuda.current_stream()
        assert lib.sht_set_stream(sht._h, VP(stream.cuda_stream)) == 0
        assert lib.sht_wa_xya_dev_noalloc(sht._h, None, 0, None) == 0
        w = torch.from_numpy(W.seeded_spectra(N, nb, 1.5, seed=11)).cuda()
        grid = sht.xya_wa(w)
        out = torch.full((nb, (N + 1) ** 2), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        assert lib.sht_wa_xya_dev_noalloc(sht._h, VP(grid.data_ptr()), nb, VP(out.data_ptr())) == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before
        assert relerr(out.cpu().numpy(), w.cpu().numpy()) < TOL
    finally:
        sht.final()


def test_noalloc_rejects_batches_beyond_the_fixed_scratch():
    import torch

    P, W = pkg(), workloads()
    lib = _lib()
    I, J, N = W.GRIDS["T85"]
    limit = int(lib.sht_noalloc_scratch_bytes())
    per = 16 * ((N + 1) * J + (N + 1) * (N + 4) // 2)
    nb = limit // per + 8  # certainly too large
    sht = P.SpmlUtil(I, J, 1, N, None, 1.0)
    try:
        grid = torch.zeros((nb, J, I), dtype=torch.float64, device="cuda")
        out = torch.zeros((nb, (N + 1) ** 2), dtype=torch.float64, device="cuda")
        st = lib.sht_wa_xya_dev_noalloc(sht._h, VP(grid.data_ptr()), nb, VP(out.data_ptr()))
        assert st == 8  # SHT_ERR_TOO_LARGE
        assert b"limit" in lib.sht_last_error()
    finally:
        sht.final()


def test_noalloc_split_precision_needs_tables_built_elsewhere():
    """In split precision the digit tables are allocated by the plan's first
    split call of an ordinary entry point; before that the allocation-free
    entry point refuses instead of allocating them, and afterwards it matches
    the ordinary entry point on two calls in a row."""
    import torch

    P, W = pkg(), workloads()
    lib = _lib()
    I, J, N = W.GRIDS["T42"]
    nb = 20
    sht = P.SpmlUtil(I, J, nb, N, None, 1.0)
    try:
        stream = torch.cuda.current_stream()
        assert lib.sht_set_stream(sht._h, VP(stream.cuda_stream)) == 0
        w = torch.from_numpy(W.seeded_spectra(N, nb, 1.5, seed=7)).cuda()
        grid = sht.xya_wa(w)
        out = torch.zeros((nb, (N + 1) ** 2), dtype=torch.float64, device="cuda")
        sht.set_precision(P.SHT_PREC_SPLIT)
        st = lib.sht_wa_xya_dev_noalloc(sht._h, VP(grid.data_ptr()), nb, VP(out.data_ptr()))
        assert st == 1 and b"digit tables" in lib.sht_last_error()
        ref = torch.empty_like(out)
        for _ in range(2):
            out.fill_(float("nan"))
            assert lib.sht_wa_xya_dev(sht._h, VP(grid.data_ptr()), nb, VP(ref.data_ptr())) == 0
            assert lib.sht_wa_xya_dev_noalloc(sht._h, VP(grid.data_ptr()), nb, VP(out.data_ptr())) == 0
            torch.cuda.synchronize()
            assert relerr(out.cpu().numpy(), ref.cpu().numpy()) < TOL
    finally:
        sht.set_precision(P.SHT_PREC_FP64)
        sht.final()
