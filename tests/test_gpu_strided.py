"""Analysis and synthesis of haloed arrays through leading dimensions
(sht_analysis / sht_synthesis and their _dev forms).

The model holds each field as xyz(IA, JA, KA) with one-point halos
(IHALO = JHALO = 1, util/grid/DOGCM_GaussSpmVFvmGrid_mod.f90:158-183) and
hands SpmlUtil the (IS:IE, JS:JE) section of every level
(HBEBaroc_hspm_vfvm_mod.f90:160-172).  These tests pass the whole haloed
array with its leading dimensions and check that

- the section's transform matches the oracle to 1e-11 per field (the FP64
  bar of every operator) and the contiguous entry points bit for bit;
- halos and spectral padding are neither read (NaN there would reach the
  result) nor written (a sentinel there survives);
- the per-call precision mode applies to that call only.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import pkg, relerr

pytestmark = pytest.mark.gpu

TOL = 1e-11
SENTINEL = 7.25
GRIDS = [(64, 32, 21), (256, 128, 85), (512, 256, 170)]


@pytest.fixture(scope="module")
def plans():
    cache = {}

    def get(I, J, N):
        key = (I, J, N)
        if key not in cache:
            cache[key] = (pkg().SpmlUtil(I, J, 1, N), O.OraclePlan(I, J, N))
        return cache[key]

    yield get
    for g, _ in cache.values():
        g.final()


def _haloed(x, hi=1, hj=1, fill=np.nan):
    """(nb, J, I) -> (nb, J + 2 hj, I + 2 hi) with the halo set to fill."""
    nb, J, I = x.shape
    h = np.full((nb, J + 2 * hj, I + 2 * hi), fill)
    h[:, hj:hj + J, hi:hi + I] = x
    return h


def _padded(w, pad=3, fill=np.nan):
    h = np.full((w.shape[0], w.shape[1] + pad), fill)
    h[:, :w.shape[1]] = w
    return h


@pytest.mark.parametrize("I,J,N", GRIDS)
def test_haloed_host_vs_oracle(I, J, N, plans):
    g, ora = plans(I, J, N)
    nb = 6
    rng = np.random.default_rng(N)
    x = rng.standard_normal((nb, J, I))
    w = rng.standard_normal((nb, g.lm))
    # analysis of the interior of a NaN-haloed array into padded rows
    wout = _padded(np.zeros((nb, g.lm)), fill=SENTINEL)
    g.analysis(_haloed(x), 1, 1, out=wout)
    assert relerr(wout[:, :g.lm], ora.wa_xya(x)) < TOL
    assert np.array_equal(wout[:, :g.lm], g.w_xy(x))
    assert np.all(wout[:, g.lm:] == SENTINEL)
    # synthesis from NaN-padded rows into the interior of a haloed array
    xout = _haloed(np.zeros((nb, J, I)), fill=SENTINEL)
    g.synthesis(_padded(w), xout, 1, 1)
    assert relerr(xout[:, 1:-1, 1:-1], ora.xya_wa(w)) < TOL
    assert np.array_equal(xout[:, 1:-1, 1:-1], g.xy_w(w))
    halo = np.ones(xout.shape, bool)
    halo[:, 1:-1, 1:-1] = False
    assert np.all(xout[halo] == SENTINEL)


@pytest.mark.parametrize("I,J,N", GRIDS[:2])
def test_haloed_device_vs_oracle(I, J, N, plans):
    g, ora = plans(I, J, N)
    nb = 5
    rng = np.random.default_rng(N + 1)
    x = rng.standard_normal((nb, J, I))
    w = rng.standard_normal((nb, g.lm))
    dev = torch.device("cuda:0")
    # odd offsets: the section does not start on a 16-byte boundary
    xh = torch.from_numpy(_haloed(x, hi=3, hj=2)).to(dev)
    wout = torch.from_numpy(_padded(np.zeros((nb, g.lm)), pad=5, fill=SENTINEL)).to(dev)
    g.analysis(xh, 3, 2, out=wout)
    wo = wout.cpu().numpy()
    assert relerr(wo[:, :g.lm], ora.wa_xya(x)) < TOL
    assert np.array_equal(wo[:, :g.lm], g.w_xy(torch.from_numpy(x).to(dev)).cpu().numpy())
    assert np.all(wo[:, g.lm:] == SENTINEL)
    xout = torch.from_numpy(_haloed(np.zeros((nb, J, I)), hi=3, hj=2, fill=SENTINEL)).to(dev)
    g.synthesis(torch.from_numpy(_padded(w, pad=5)).to(dev), xout, 3, 2)
    xo = xout.cpu().numpy()
    assert relerr(xo[:, 2:-2, 3:-3], ora.xya_wa(w)) < TOL
    halo = np.ones(xo.shape, bool)
    halo[:, 2:-2, 3:-3] = False
    assert np.all(xo[halo] == SENTINEL)
    # contiguous arrays take the ordinary device path
    wc = g.analysis(torch.from_numpy(x).to(dev))
    assert np.array_equal(wc.cpu().numpy(), wo[:, :g.lm])


def test_mode_applies_to_one_call(plans):
    I, J, N = 256, 128, 85
    g, ora = plans(I, J, N)
    P = pkg()
    assert g.get_precision() == P.SHT_PREC_FP64
    rng = np.random.default_rng(5)
    x = rng.standard_normal((4, J, I))
    ws = g.analysis(_haloed(x), 1, 1, mode=P.SHT_PREC_SPLIT)
    assert g.get_precision() == P.SHT_PREC_FP64
    assert relerr(ws, ora.wa_xya(x)) < TOL
    w = rng.standard_normal((4, g.lm))
    xs = g.synthesis(w, _haloed(np.zeros((4, J, I))), 1, 1, mode=P.SHT_PREC_SPLIT)
    assert relerr(xs[:, 1:-1, 1:-1], ora.xya_wa(w)) < TOL
    assert g.get_precision() == P.SHT_PREC_FP64
    # FP64 forced on a split plan
    g.set_precision(P.SHT_PREC_SPLIT)
    try:
        wf = g.analysis(_haloed(x), 1, 1, mode=P.SHT_PREC_FP64)
        assert g.get_precision() == P.SHT_PREC_SPLIT
    finally:
        g.set_precision(P.SHT_PREC_FP64)
    assert np.array_equal(wf, g.w_xy(x))


def test_zonal_haloed():
    """im = 1: one longitude per row, rows of IA = 3 values."""
    z = pkg().SpmlUtil(1, 64, 1, -1)
    try:
        rng = np.random.default_rng(9)
        x = rng.standard_normal((7, 64, 1))
        w = z.analysis(_haloed(x), 1, 1)
        assert np.array_equal(w, z.wa_xya(x))
        xo = z.synthesis(w, _haloed(np.zeros((7, 64, 1)), fill=SENTINEL), 1, 1)
        assert np.array_equal(xo[:, 1:-1, 1:-1], z.xya_wa(w))
        assert np.all(xo[:, 0] == SENTINEL) and np.all(xo[:, :, 0] == SENTINEL)
    finally:
        z.final()


def test_strided_argument_errors(plans):
    g, _ = plans(64, 32, 21)
    lib = pkg().load_library()
    x = np.zeros((2, 34, 66))
    w = np.zeros((2, g.lm))
    ptr = x.ctypes.data + 8 * (66 + 1)
    # leading dimensions below the grid, unknown mode, null arrays
    assert lib.sht_analysis(g._h, ptr, 63, 34, 2, w.ctypes.data, g.lm, -1) == 1
    assert lib.sht_analysis(g._h, ptr, 66, 31, 2, w.ctypes.data, g.lm, -1) == 1
    assert lib.sht_analysis(g._h, ptr, 66, 34, 2, w.ctypes.data, g.lm - 1, -1) == 1
    assert lib.sht_analysis(g._h, ptr, 66, 34, 2, w.ctypes.data, g.lm, 5) == 1
    assert lib.sht_synthesis(g._h, None, g.lm, 2, ptr, 66, 34, -1) == 1
    assert lib.sht_analysis(g._h, ptr, 66, 34, -1, w.ctypes.data, g.lm, -1) == 1
    # an empty batch is a no-op, even with null arrays
    assert lib.sht_analysis(g._h, None, 66, 34, 0, None, g.lm, -1) == 0
    with pytest.raises(pkg().SpmlError):
        g.analysis(np.zeros((2, 32, 66)), 1, 1)        # section leaves the array
