"""Split-precision Legendre contraction (signed 8-bit digit products on
tcgen05, exact integer level sums, FP64 recombination) through the C-ABI,
against the CPU oracle and the FP64 path.

Tolerance: 1e-11 per-field normwise relative error, the same bar as the plain
FP64 path (the digits keep 46 bits per operand below its row or column bound).
"""
import numpy as np
import pytest

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11
GRIDS = [(64, 32, 21), (128, 64, 42), (256, 128, 85), (512, 256, 170)]


@pytest.fixture(scope="module")
def plan_cache():
    cache = {}

    def get(I, J, N, a=1.0):
        key = (I, J, N, a)
        if key not in cache:
            cache[key] = (pkg().SpmlUtil(I, J, 1, N, None, a), O.OraclePlan(I, J, N, a))
        return cache[key]

    yield get
    for g, _ in cache.values():
        g.final()


@pytest.mark.parametrize("grid", GRIDS)
def test_split_round_trip_vs_oracle(grid, plan_cache):
    P, W = pkg(), workloads()
    I, J, N = grid
    gpu, ora = plan_cache(I, J, N)
    rng = np.random.default_rng(5)
    w = W.seeded_spectra(N, 70, 2.0, rng=rng)      # 70 columns: a ragged 64-column tile
    x = rng.standard_normal((70, J, I))
    gpu.set_precision(P.SHT_PREC_SPLIT)
    try:
        g_split = gpu.xya_wa(w)
        w_split = gpu.wa_xya(x)
        gpu.synchronize()  # also reads the device error word of the bounded waits
    finally:
        gpu.set_precision(P.SHT_PREC_FP64)
    assert relerr(g_split, ora.xya_wa(w)) < TOL
    assert relerr(w_split, ora.wa_xya(x)) < TOL
    assert relerr(g_split, gpu.xya_wa(w)) < TOL


@pytest.mark.parametrize("grid", GRIDS)
def test_split_derivatives_vs_oracle(grid, plan_cache):
    P, W = pkg(), workloads()
    I, J, N = grid
    a = 6.371e6
    gpu, ora = plan_cache(I, J, N, a)
    w = W.seeded_spectra(N, 9, 2.0, seed=3) / a
    w2 = W.seeded_spectra(N, 9, 2.0, seed=4) / a
    gpu.set_precision(P.SHT_PREC_SPLIT)
    try:
        u, v = gpu.calc_VorDiv2UV(w, w2)
        cs = np.cos(gpu.y_Lat)[None, :, None]
        vo, di = gpu.calc_UVCosLat2VorDiv(u * cs, v * cs)
        gpu.synchronize()
    finally:
        gpu.set_precision(P.SHT_PREC_FP64)
    uo, vvo = ora.vordiv2uv(w, w2)
    vr, dr = ora.uvcoslat2vordiv(u * cs, v * cs)
    assert relerr(u, uo) < TOL and relerr(v, vvo) < TOL
    assert relerr(vo, vr) < TOL and relerr(di, dr) < TOL


def test_split_t85_full_batch_round_trip(plan_cache):
    """The benchmark batch (480 field-levels at T85) survives a split round trip."""
    P, W = pkg(), workloads()
    I, J, N = W.GRIDS["T85"]
    gpu, _ = plan_cache(I, J, N)
    w = W.seeded_spectra(N, 480, 2.0)
    gpu.set_precision(P.SHT_PREC_SPLIT)
    try:
        out = gpu.wa_xya(gpu.xya_wa(w))
        gpu.synchronize()
    finally:
        gpu.set_precision(P.SHT_PREC_FP64)
    assert relerr(out, w) < TOL


def test_split_t341_matches_fp64(plan_cache):
    """T341 (segments of the output dimension, 256-term exact level sums)
    against the FP64 GPU path and as a round trip."""
    P, W = pkg(), workloads()
    I, J, N = W.GRIDS["T341"]
    gpu, _ = plan_cache(I, J, N)
    w = W.seeded_spectra(N, 24, 2.0, seed=9)
    g64 = gpu.xya_wa(w)
    gpu.set_precision(P.SHT_PREC_SPLIT)
    try:
        g = gpu.xya_wa(w)
        back = gpu.wa_xya(g)
        gpu.synchronize()
    finally:
        gpu.set_precision(P.SHT_PREC_FP64)
    assert relerr(g, g64) < TOL
    assert relerr(back, w) < TOL


def test_split_many_latitudes_vs_oracle(plan_cache):
    """512 half-latitudes: the analysis contraction runs over eight K chunks,
    with the column exponents from a first pass over all of them."""
    P, W = pkg(), workloads()
    gpu, ora = plan_cache(64, 1024, 21)
    rng = np.random.default_rng(12)
    w = W.seeded_spectra(21, 6, 1.5, rng=rng)
    x = rng.standard_normal((6, 1024, 64))
    gpu.set_precision(P.SHT_PREC_SPLIT)
    try:
        g = gpu.xya_wa(w)
        back = gpu.wa_xya(x)
        gpu.synchronize()
    finally:
        gpu.set_precision(P.SHT_PREC_FP64)
    assert relerr(g, ora.xya_wa(w)) < TOL
    assert relerr(back, ora.wa_xya(x)) < TOL


def _trel(a, b) -> float:
    """relerr of two device tensors, on the device (fields = leading axis)."""
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    den = b.abs().amax(dim=1)
    den = den.masked_fill(den == 0, 1.0)
    return float(((a - b).abs().amax(dim=1) / den).max())


def _config_results(gpu, w, coef):
    """Every C2/C4 quantity of one precision, on device arrays: synthesis,
    analysis round trip, both gradients, AlphaOptr of two grids, and the
    backward-Euler diffusion round trip."""
    import torch
    g = gpu.xya_wa(w)
    back = gpu.wa_xya(g)
    glon, glat = gpu.xy_HGrad_w(w)
    alpha = gpu.wa_AlphaOptr_xya(g, glat)
    d = g.clone()
    gpu.roundtrip_diffuse_(d, coef, 1.0)
    torch.cuda.synchronize()
    return dict(g=g, back=back, glon=glon, glat=glat, alpha=alpha, diffused=d)


@pytest.mark.parametrize("cfg", ["C2", "C4"])
def test_config_full_batch_split_vs_fp64(cfg):
    """C2 (T170, 60 x 12, p = 1.5) and C4 (T341, 60 x 16, p = 2, Ord-8
    diffusion with dt nu = 1e-3): the whole batch in split precision against
    the FP64 GPU path, which the oracle pins at these truncations on small
    batches; the round trip against the identity."""
    import torch
    P, W = pkg(), workloads()
    c = W.CONFIGS[cfg]
    I, J, N = W.GRIDS[c["grid"]]
    nb = c["levels"] * c["fields"]
    dev = torch.device("cuda")
    gpu = P.SpmlUtil(I, J, 1, N, None, 6.371e6)
    try:
        w = W.seeded_spectra_torch(N, nb, c["power"], dev)
        coef = torch.from_numpy(W.diffusion_coef(N, 8, 1e-3)).to(dev)
        ref = _config_results(gpu, w, coef)
        gpu.set_precision(P.SHT_PREC_SPLIT)
        try:
            got = _config_results(gpu, w, coef)
        finally:
            gpu.set_precision(P.SHT_PREC_FP64)
        for k in ref:
            assert _trel(got[k], ref[k]) < TOL, k
        assert _trel(got["back"], w) < TOL and _trel(ref["back"], w) < TOL
    finally:
        gpu.final()


def test_per_direction_precision(plan_cache):
    """SHT_PREC_AUTO: split precision for a contraction of at least 128 terms
    (the analysis at jm/2 >= 128, the synthesis at (nm+3)/2 >= 128), FP64 for
    the others.  T85: both directions as FP64, bit for bit; T170: the analysis
    as split, the synthesis as FP64, bit for bit, and both against the oracle."""
    P, W = pkg(), workloads()
    for I, J, N in ((256, 128, 85), (512, 256, 170)):
        gpu, ora = plan_cache(I, J, N)
        rng = np.random.default_rng(N)
        w = W.seeded_spectra(N, 9, 2.0, rng=rng)
        x = rng.standard_normal((9, J, I))
        out = {}
        try:
            for mode in (P.SHT_PREC_FP64, P.SHT_PREC_SPLIT, P.SHT_PREC_AUTO):
                gpu.set_precision(mode)
                assert gpu.get_precision() == mode
                out[mode] = (gpu.xya_wa(w), gpu.wa_xya(x))
        finally:
            gpu.set_precision(P.SHT_PREC_FP64)
        syn_split, ana_split = (N + 3) // 2 >= 128, J // 2 >= 128
        assert np.array_equal(out[P.SHT_PREC_AUTO][0], out[P.SHT_PREC_SPLIT if syn_split else P.SHT_PREC_FP64][0])
        assert np.array_equal(out[P.SHT_PREC_AUTO][1], out[P.SHT_PREC_SPLIT if ana_split else P.SHT_PREC_FP64][1])
        assert relerr(out[P.SHT_PREC_AUTO][0], ora.xya_wa(w)) < TOL
        assert relerr(out[P.SHT_PREC_AUTO][1], ora.wa_xya(x)) < TOL
    with pytest.raises(P.SpmlError):
        gpu.set_precision(3)
