"""The single-kernel small-grid transforms (SHT_OPT_LEGENDRE_KERNEL = 4):
longitude FFT, Legendre contraction and SPML layout conversion of a group of
field-levels in one thread block, for im <= 128.

They must give what the batched four-kernel path gives (1e-13: the same
products, summed in another order) and what the oracle gives (1e-11), on odd
and even truncations, latitude counts whose last row tile is partial, and
batches whose last group of levels is partial; fall back to the batched path
for every other operator, precision and grid; and launch one kernel per call.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11
SMALL = [(32, 16, 10), (64, 32, 21), (64, 48, 20), (128, 64, 42), (128, 64, 41), (64, 32, 15)]


@pytest.fixture(scope="module")
def plans():
    cache = {}

    def get(I, J, N, a=1.0):
        key = (I, J, N, a)
        if key not in cache:
            cache[key] = (pkg().SpmlUtil(I, J, 1, N, None, a), O.OraclePlan(I, J, N, a))
        return cache[key]

    yield get
    for g, _ in cache.values():
        g.final()


def _inputs(I, J, N, nb, seed):
    rng = np.random.default_rng(seed)
    w = workloads().seeded_spectra(N, nb, 1.5, rng=rng)
    return w, rng.standard_normal((nb, J, I))


def _with_kernel(gpu, kern, fn):
    P = pkg()
    gpu.set_option(P.SHT_OPT_LEGENDRE_KERNEL, kern)
    try:
        return fn()
    finally:
        gpu.set_option(P.SHT_OPT_LEGENDRE_KERNEL, 0)


@pytest.mark.parametrize("grid", SMALL)
@pytest.mark.parametrize("nb", [1, 6, 37])
def test_small_matches_batched_and_oracle(grid, nb, plans):
    I, J, N = grid
    gpu, ora = plans(I, J, N)
    w, x = _inputs(I, J, N, nb, seed=31 + nb)
    # the per-band kernel family (1) keeps the batched path on every grid
    ref = _with_kernel(gpu, 1, lambda: (gpu.xya_wa(w), gpu.wa_xya(x)))
    got = _with_kernel(gpu, 4, lambda: (gpu.xya_wa(w), gpu.wa_xya(x)))
    assert relerr(got[0], ref[0]) < 1e-13
    assert relerr(got[1], ref[1]) < 1e-13
    assert relerr(got[0], ora.xya_wa(w)) < TOL
    assert relerr(got[1], ora.wa_xya(x)) < TOL
    # the round trip returns the spectrum
    back = _with_kernel(gpu, 4, lambda: gpu.wa_xya(got[0]))
    assert relerr(back, w) < TOL


@pytest.mark.parametrize("grid", [(64, 32, 21), (128, 64, 42)])
def test_small_device_pointers_one_launch(grid, plans):
    """Device-pointer calls: one kernel per direction, results equal to the
    host-pointer calls of the same path bit for bit."""
    P = pkg()
    I, J, N = grid
    gpu, _ = plans(I, J, N)
    w, x = _inputs(I, J, N, 23, seed=5)
    wd, xd = torch.from_numpy(w).cuda(), torch.from_numpy(x).cuda()
    gpu.set_option(P.SHT_OPT_LEGENDRE_KERNEL, 4)
    try:
        host = (gpu.xya_wa(w), gpu.wa_xya(x))
        torch.cuda.synchronize()
        n0 = P.launch_count()
        g = gpu.xya_wa(wd)
        n1 = P.launch_count()
        s = gpu.wa_xya(xd)
        n2 = P.launch_count()
        torch.cuda.synchronize()
        assert n1 - n0 == 1 and n2 - n1 == 1
        assert np.array_equal(g.cpu().numpy(), host[0])
        assert np.array_equal(s.cpu().numpy(), host[1])
    finally:
        gpu.set_option(P.SHT_OPT_LEGENDRE_KERNEL, 0)


def test_small_falls_back_elsewhere(plans):
    """Other operators, split precision and grids outside the small-grid range
    take the batched path under the option: results equal the automatic
    choice's bit for bit."""
    P = pkg()
    # other operators on a small grid
    gpu, _ = plans(64, 32, 21)
    w, x = _inputs(64, 32, 21, 9, seed=8)
    ops = lambda: (gpu.xya_GradMu_wa(w), gpu.wa_DivMu_xya(x), gpu.xya_GradLon_wa(w), gpu.wa_AlphaOptr_xya(x, x))
    a, b = _with_kernel(gpu, 0, ops), _with_kernel(gpu, 4, ops)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    # split precision keeps the tensor-core path
    gpu.set_precision(P.SHT_PREC_SPLIT)
    try:
        a = _with_kernel(gpu, 0, lambda: (gpu.xya_wa(w), gpu.wa_xya(x)))
        b = _with_kernel(gpu, 4, lambda: (gpu.xya_wa(w), gpu.wa_xya(x)))
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    finally:
        gpu.set_precision(P.SHT_PREC_FP64)
    # grids the single kernel does not take: T85, a longitude count with a
    # factor of 3, and a grid whose Fourier arrays exceed a block's shared memory
    for I, J, N in ((256, 128, 85), (96, 48, 31), (128, 128, 63)):
        gpu, _ = plans(I, J, N)
        w, x = _inputs(I, J, N, 4, seed=9)
        a = _with_kernel(gpu, 0, lambda: (gpu.xya_wa(w), gpu.wa_xya(x)))
        b = _with_kernel(gpu, 4, lambda: (gpu.xya_wa(w), gpu.wa_xya(x)))
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (I, J, N)


def test_small_in_multi_instance_batches(plans):
    """Multi-instance groups of small plans run the single kernel when the
    plans ask for it: each instance equals its single-plan transform."""
    P, W = pkg(), workloads()
    grids = {"T21": W.GRIDS["T21"], "T42": W.GRIDS["T42"]}
    own = {k: P.SpmlUtil(*g[:2], 1, g[2]) for k, g in grids.items()}
    rng = np.random.default_rng(41)
    insts = []
    try:
        for k, p in own.items():
            p.set_option(P.SHT_OPT_LEGENDRE_KERNEL, 4)
            for nb in (5, 33):
                w = W.seeded_spectra(p.nm, nb, 1.5, rng=rng)
                insts.append(dict(plan=p, w=w,
                                  wa=torch.zeros((nb, p.lm), dtype=torch.float64, device="cuda"),
                                  xya=torch.zeros((nb, p.jm, p.im), dtype=torch.float64, device="cuda")))
        m = P.MultiTransform()
        try:
            for x in insts:
                m.add(x["plan"], x["wa"], x["xya"])
            m.build(autotune=False)
            for x in insts:
                x["wa"].copy_(torch.from_numpy(x["w"]))
            torch.cuda.synchronize()
            assert all(g["legendre_kernel"] == 4 for g in m.groups())
            m.run(P.SHT_MULTI_ROUND_TRIP)
            m.synchronize()
            for x in insts:
                ref = x["plan"].xya_wa(x["w"])
                assert relerr(x["xya"].cpu().numpy(), ref) < 1e-12
                assert relerr(x["wa"].cpu().numpy(), x["w"]) < TOL
        finally:
            m.close()
    finally:
        for p in own.values():
            p.final()


def test_small_is_the_automatic_choice_at_im_32(plans):
    """im = 32 (T10) takes the single kernel by default: one launch per call."""
    P = pkg()
    gpu, ora = plans(32, 16, 10)
    w, x = _inputs(32, 16, 10, 12, seed=3)
    wd = torch.from_numpy(w).cuda()
    torch.cuda.synchronize()
    n0 = P.launch_count()
    g = gpu.xya_wa(wd)
    torch.cuda.synchronize()
    assert P.launch_count() - n0 == 1
    assert relerr(g.cpu().numpy(), ora.xya_wa(w)) < TOL
