"""GPU parity: every SpmlUtil operator through the C-ABI against the CPU oracle
and the golden vectors.

Tolerance: the plain FP64 path must match within 1e-11 per-field normwise
relative error (max|gpu - ref| / max|ref| per field-level), the bound the
transform is specified to.
"""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden, pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11
GRIDS = [(32, 16, 10), (64, 32, 21), (128, 64, 42), (256, 128, 85), (512, 256, 170)]


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


def _inputs(I, J, N, nb, seed=11, a=1.0):
    rng = np.random.default_rng(seed)
    W = workloads()
    w = W.seeded_spectra(N, nb, 1.5, rng=rng)
    w2 = W.seeded_spectra(N, nb, 2.0, rng=rng)
    grid = rng.standard_normal((nb, J, I))
    return w, w2, grid


@pytest.mark.parametrize("tag", ["T21", "T10"])
def test_golden(tag, plans):
    g = load_golden(tag)
    gpu, _ = plans(int(g["I"]), int(g["J"]), int(g["N"]), float(g["radius"]))
    cs = np.cos(np.arcsin(g["mu"]))[None, :, None]
    res = {
        "xy_w": relerr(gpu.xya_wa(g["w"]), g["xy_w"]),
        "w_xy_rand": relerr(gpu.wa_xya(g["grid_rand"]), g["w_xy_rand"]),
        "gradlambda": relerr(gpu.xya_GradLambda_wa(g["w"]), g["gradlambda"]),
        "gradmu": relerr(gpu.xya_GradMu_wa(g["w"]), g["gradmu"]),
        "gradlon": relerr(gpu.xya_GradLon_wa(g["w"]), g["gradlon"]),
        "gradlat": relerr(gpu.xya_GradLat_wa(g["w"]), g["gradlat"]),
        "divlambda": relerr(gpu.wa_DivLambda_xya(g["divA"]), g["divlambda"]),
        "divmu": relerr(gpu.wa_DivMu_xya(g["divB"]), g["divmu"]),
        "w_alpha": relerr(gpu.wa_AlphaOptr_xya(g["divA"], g["divB"]), g["w_alpha"]),
        "xy_alpha": relerr(gpu.xya_AlphaOptr_wa(g["w"], g["w2"]), g["xy_alpha"]),
        "avr": relerr(gpu.AvrLonLat_xy(g["xy_w"]), g["avr"]),
    }
    u, v = gpu.calc_VorDiv2UV(g["w"], g["w2"])
    res["U"], res["V"] = relerr(u, g["U"]), relerr(v, g["V"])
    vo, di = gpu.calc_UVCosLat2VorDiv(g["U"] * cs, g["V"] * cs)
    res["vor"], res["div"] = relerr(vo, g["vor"]), relerr(di, g["div"])
    bad = {k: v for k, v in res.items() if v > TOL}
    assert not bad, bad


@pytest.mark.parametrize("grid", GRIDS)
def test_analysis_synthesis_vs_oracle(grid, plans):
    I, J, N = grid
    gpu, ora = plans(I, J, N)
    w, w2, x = _inputs(I, J, N, 5)
    assert relerr(gpu.xya_wa(w), ora.xya_wa(w)) < TOL
    assert relerr(gpu.wa_xya(x), ora.wa_xya(x)) < TOL


@pytest.mark.parametrize("grid", GRIDS)
def test_derivatives_vs_oracle(grid, plans):
    I, J, N = grid
    a = 6.371e6
    gpu, ora = plans(I, J, N, a)
    w, w2, x = _inputs(I, J, N, 4, seed=12)
    cs2 = np.cos(gpu.y_Lat)[None, :, None] ** 2
    A, B = ora.xya_wa(w) * cs2, ora.xya_wa(w2) * cs2  # U cos phi-like, vanish at the poles
    res = {
        "gradlambda": relerr(gpu.xya_GradLambda_wa(w), ora.xya_gradlambda_wa(w)),
        "gradmu": relerr(gpu.xya_GradMu_wa(w), ora.xya_gradmu_wa(w)),
        "gradlon": relerr(gpu.xya_GradLon_wa(w), ora.xya_gradlon_wa(w)),
        "gradlat": relerr(gpu.xya_GradLat_wa(w), ora.xya_gradlat_wa(w)),
        "divlambda": relerr(gpu.wa_DivLambda_xya(A), ora.wa_divlambda_xya(A)),
        "divmu": relerr(gpu.wa_DivMu_xya(B), ora.wa_divmu_xya(B)),
        "w_alpha": relerr(gpu.wa_AlphaOptr_xya(A, B), ora.wa_alphaoptr_xya(A, B)),
        "xy_alpha": relerr(gpu.xya_AlphaOptr_wa(w, w2), ora.xya_alphaoptr_wa(w, w2)),
        "lapla": relerr(gpu.w_Lapla_w(w), ora.wa_lapla_wa(w)),
        "laplainv": relerr(gpu.w_LaplaInv_w(w), ora.wa_laplainv_wa(w)),
    }
    u, v = gpu.calc_VorDiv2UV(w / a, w2 / a)
    uo, vo = ora.vordiv2uv(w / a, w2 / a)
    res["U"], res["V"] = relerr(u, uo), relerr(v, vo)
    vg, dg = gpu.calc_UVCosLat2VorDiv(A, B)
    vr, dr = ora.uvcoslat2vordiv(A, B)
    res["vor"], res["div"] = relerr(vg, vr), relerr(dg, dr)
    bad = {k: v for k, v in res.items() if v > TOL}
    assert not bad, bad


def test_reductions_vs_oracle(plans):
    gpu, ora = plans(128, 64, 42)
    _, _, x = _inputs(128, 64, 42, 3)
    # the means of random data cancel: measure the error against the data scale
    scale = np.abs(x).mean()
    assert np.abs(gpu.AvrLonLat_xy(x) - ora.avrlonlat(x)).max() / scale < 1e-14
    assert np.abs(gpu.IntLonLat_xy(x) - ora.intlonlat(x)).max() / (4 * np.pi * scale) < 1e-14
    assert np.abs(gpu.ya_AvrLon_xya(x) - ora.ya_avrlon(x)).max() / scale < 1e-14
    assert np.abs(gpu.ya_IntLon_xya(x) - ora.ya_intlon(x)).max() / (2 * np.pi * scale) < 1e-14


def test_grid_info_matches_oracle(plans):
    gpu, ora = plans(256, 128, 85)
    xl, yl, xw, yw = ora.grid_info()
    assert np.abs(gpu.y_Lat - yl).max() < 1e-14
    assert np.abs(gpu.y_Lat_Weight - yw).max() < 1e-15
    assert np.abs(gpu.x_Lon - xl).max() == 0.0
    assert abs(gpu.y_Lat_Weight.sum() - 2.0) < 1e-14
    assert np.allclose(gpu.rn, ora.rn(), rtol=0, atol=0)


def test_config_c0_full(plans):
    """C0: T21, 20 levels x 3 fields: round trip plus gradient/divergence/vorticity."""
    W = workloads()
    c = W.CONFIGS["C0"]
    I, J, N = W.GRIDS[c["grid"]]
    nb = c["levels"] * c["fields"]
    gpu, ora = plans(I, J, N, 6.371e6)
    w = W.seeded_spectra(N, nb, c["power"])
    g = gpu.xya_wa(w)
    assert relerr(g, ora.xya_wa(w)) < TOL
    assert relerr(gpu.wa_xya(g), w) < TOL
    u, v = gpu.calc_VorDiv2UV(w / 6.371e6, w[::-1] / 6.371e6)
    uo, vo = ora.vordiv2uv(w / 6.371e6, w[::-1] / 6.371e6)
    assert relerr(u, uo) < TOL and relerr(v, vo) < TOL
    cs = np.cos(gpu.y_Lat)[None, :, None]
    vg, dg = gpu.calc_UVCosLat2VorDiv(u * cs, v * cs)
    vr, dr = ora.uvcoslat2vordiv(u * cs, v * cs)
    assert relerr(vg, vr) < TOL and relerr(dg, dr) < TOL


def test_config_c1_tendency(plans):
    """C1 pattern at T85 (HBEBaroc_HTRCRHS, HBEBaroc_hspm_vfvm_mod.f90:160-172): U,V from
    vor/div, tracer gradients, grid products, analysed back by w_AlphaOptr_xy; 12 levels."""
    W = workloads()
    a = 6.371e6
    I, J, N = W.GRIDS["T85"]
    nb = 12
    gpu, ora = plans(I, J, N, a)
    vor = W.seeded_spectra(N, nb, 2.0, seed=1) / a
    div = W.seeded_spectra(N, nb, 2.0, seed=2) / a
    T = W.seeded_spectra(N, nb, 1.5, seed=3)
    U, V = gpu.calc_VorDiv2UV(vor, div)
    Uo, Vo = ora.vordiv2uv(vor, div)
    Tg = gpu.xya_wa(T)
    cs = np.cos(gpu.y_Lat)[None, :, None]
    out = gpu.wa_AlphaOptr_xya(Tg * U * cs, Tg * V * cs)
    ref = ora.wa_alphaoptr_xya(Tg * Uo * cs, Tg * Vo * cs)
    assert relerr(U, Uo) < TOL and relerr(V, Vo) < TOL
    assert relerr(out, ref) < TOL


@pytest.mark.parametrize("grid", [(1024, 512, 341), (512, 256, 170)])
def test_round_trip_property_large(grid, plans):
    """Band-limited spectra survive synthesis + analysis (exact with J > N Gauss rows)."""
    I, J, N = grid
    gpu, _ = plans(I, J, N)
    w = workloads().seeded_spectra(N, 8, 2.0)
    assert relerr(gpu.wa_xya(gpu.xya_wa(w)), w) < TOL


def test_largest_grid_properties():
    """The largest longitude count a plan takes (im = 2048: the 1024-point
    complex FFT) with 512 half-latitudes (beyond the paired and chunked
    Legendre kernels, so the per-band ones run): a band-limited round trip is
    the identity, and d/dlambda of a spectrum equals the synthesis of i m times
    it.  The oracle is too slow at T682, so these are properties."""
    N = 682
    gpu = pkg().SpmlUtil(2048, 1024, 1, N)
    try:
        w = workloads().seeded_spectra(N, 2, 2.0, seed=5)
        assert relerr(gpu.wa_xya(gpu.xya_wa(w)), w) < TOL
        im_w = np.zeros_like(w)
        for n in range(1, N + 1):
            m = np.arange(1, n + 1)
            c, s_ = n * (n + 1) + m, n * (n + 1) - m
            im_w[:, c] = -m * w[:, s_]
            im_w[:, s_] = m * w[:, c]
        assert relerr(gpu.xya_GradLambda_wa(w), gpu.xya_wa(im_w)) < TOL
    finally:
        gpu.final()


def test_device_pointer_path_matches_host(plans):
    import torch
    I, J, N = 256, 128, 85
    gpu, _ = plans(I, J, N, 6.371e6)
    w, w2, x = _inputs(I, J, N, 6)
    wd = torch.from_numpy(w).cuda()
    xd = torch.from_numpy(x).cuda()
    assert np.array_equal(gpu.xya_wa(wd).cpu().numpy(), gpu.xya_wa(w))
    assert np.array_equal(gpu.wa_xya(xd).cpu().numpy(), gpu.wa_xya(x))
    u1, v1 = gpu.calc_VorDiv2UV(wd, torch.from_numpy(w2).cuda())
    u2, v2 = gpu.calc_VorDiv2UV(w, w2)
    assert np.array_equal(u1.cpu().numpy(), u2) and np.array_equal(v1.cpu().numpy(), v2)


def test_single_level_and_odd_batches(plans):
    gpu, ora = plans(128, 64, 42)
    w, _, x = _inputs(128, 64, 42, 37)
    assert relerr(gpu.xy_w(w[0])[None], ora.xya_wa(w[:1])) < TOL
    assert relerr(gpu.wa_xya(x), ora.wa_xya(x)) < TOL  # 37 columns: ragged column tiles


def test_diffusion_epilogue(plans):
    import torch
    W = workloads()
    I, J, N = 256, 128, 85
    gpu, ora = plans(I, J, N)
    w = W.seeded_spectra(N, 4, 2.0)
    coef = W.diffusion_coef(N, 8, 1e-3)
    out = gpu.diffuse(w, coef, 1.0)
    assert relerr(out, ora.diffuse(w, coef, 1.0)) < 1e-15
    g = torch.from_numpy(gpu.xya_wa(w)).cuda().contiguous()
    gpu.roundtrip_diffuse_(g, torch.from_numpy(coef).cuda(), 1.0)
    ref = ora.xya_wa(ora.diffuse(ora.wa_xya(gpu.xya_wa(w)), coef, 1.0))
    assert relerr(g.cpu().numpy(), ref) < TOL


def test_error_paths(plans):
    P = pkg()
    gpu, _ = plans(64, 32, 21)
    with pytest.raises(P.SpmlError):
        gpu.xya_wa(np.zeros((2, 17)))
    with pytest.raises(P.SpmlError):
        gpu.set_precision(7)
    g2 = P.SpmlUtil(64, 32, 1, 21, None, 1.0)
    g2.final()
    assert not g2.isInitialzed()
    lib = P.load_library()
    import ctypes
    buf = (ctypes.c_double * 8)()
    assert lib.sht_wa_xya(None, buf, 1, buf) == 3
    # an empty batch is a no-op on a live plan, even with null arrays
    assert lib.sht_wa_xya(gpu._h, None, 0, None) == 0
    assert lib.sht_xya_wa_dev(gpu._h, None, 0, None) == 0
    assert lib.sht_wa_alphaoptr_prod_xya(gpu._h, None, None, None, 0, None) == 0
    # negative counts and null arrays with work to do are rejected
    assert lib.sht_xya_wa(gpu._h, buf, -3, buf) == 1
    assert lib.sht_xya_hgrad_wa(gpu._h, buf, 1, buf, None) == 1


@pytest.mark.parametrize("grid", [(64, 32, 21), (128, 64, 42), (256, 128, 85), (256, 128, 84), (32, 32, 10),
                                  (512, 256, 170), (512, 256, 169), (1024, 512, 341)])
def test_legendre_kernel_variants_agree(grid, plans):
    """The per-band kernel (1), the persistent paired-band kernel (2, grids up
    to T85) and the latitude-chunked paired kernel (3, jm/2 a multiple of 16)
    give the same transforms: odd and even N, ragged column tiles.  A variant
    that does not cover a grid falls back, so every setting must agree."""
    P = pkg()
    I, J, N = grid
    gpu, ora = plans(I, J, N)
    nb = 37 if N < 300 else 19
    w, w2, x = _inputs(I, J, N, nb, seed=21)
    out = {}
    for variant in (1, 2, 3):
        gpu.set_option(P.SHT_OPT_LEGENDRE_KERNEL, variant)
        out[variant] = (gpu.xya_wa(w), gpu.wa_xya(x), gpu.xya_GradMu_wa(w2))
    gpu.set_option(P.SHT_OPT_LEGENDRE_KERNEL, 0)
    for v in (2, 3):
        for k in range(3):
            assert relerr(out[v][k], out[1][k]) < 1e-13, (v, k)
    if N <= 170:
        assert relerr(out[3][0], ora.xya_wa(w)) < TOL
        assert relerr(out[3][1], ora.wa_xya(x)) < TOL


@pytest.mark.parametrize("grid", [(64, 32, 21), (256, 128, 85), (512, 256, 170), (1024, 512, 341)])
def test_legendre_tiles_agree(grid, plans):
    """Every tile of the paired kernel (8 or 16 analysis columns per item) and
    of the chunked kernel (16 or 32 latitudes per chunk) gives the same
    results bit for bit, and matches the oracle; a tile a kernel cannot take
    falls back to its automatic one."""
    P = pkg()
    I, J, N = grid
    gpu, ora = plans(I, J, N)
    nb = 37 if N < 300 else 11
    w, w2, x = _inputs(I, J, N, nb, seed=23)
    try:
        for kern in (2, 3):
            gpu.set_option(P.SHT_OPT_LEGENDRE_KERNEL, kern)
            out = {}
            for tile in (0, 8, 16, 32):
                gpu.set_option(P.SHT_OPT_LEGENDRE_TILE, tile)
                assert gpu.get_option(P.SHT_OPT_LEGENDRE_TILE) == tile
                out[tile] = (gpu.wa_xya(x), gpu.xya_wa(w), gpu.wa_DivMu_xya(x))
            for tile in (8, 16, 32):
                for k in range(3):
                    assert np.array_equal(out[tile][k], out[0][k]), (kern, tile, k)
            if N <= 170:
                assert relerr(out[0][0], ora.wa_xya(x)) < TOL
                assert relerr(out[0][1], ora.xya_wa(w)) < TOL
        with pytest.raises(P.SpmlError):
            gpu.set_option(P.SHT_OPT_LEGENDRE_TILE, 12)
    finally:
        gpu.set_option(P.SHT_OPT_LEGENDRE_TILE, 0)
        gpu.set_option(P.SHT_OPT_LEGENDRE_KERNEL, 0)


@pytest.mark.parametrize("grid", [(96, 48, 31), (192, 96, 63), (320, 160, 106)])
@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_longitude_counts_with_factors_3_and_5(grid, prec, plans):
    """im = 96, 192 and 320 (2^5 x 3, 2^6 x 3, 2^6 x 5): dogcm derives
    nm = (im - 1)/3 from any im (DOGCM_GaussSpmVFvmGrid_mod.f90:209-211), so
    these grids take the direct longitude transform; every operator against
    the oracle in both precisions."""
    P = pkg()
    I, J, N = grid
    a = 6.371e6
    gpu, ora = plans(I, J, N, a)
    w, w2, x = _inputs(I, J, N, 6, seed=21)
    gpu.set_precision(P.SHT_PREC_SPLIT if prec == "split" else P.SHT_PREC_FP64)
    try:
        assert relerr(gpu.xya_wa(w), ora.xya_wa(w)) < TOL
        assert relerr(gpu.wa_xya(x), ora.wa_xya(x)) < TOL
        assert relerr(gpu.xya_GradLon_wa(w), ora.xya_gradlon_wa(w)) < TOL
        assert relerr(gpu.xya_GradLat_wa(w), ora.xya_gradlat_wa(w)) < TOL
        u, v = gpu.calc_VorDiv2UV(w / a, w2 / a)
        uo, vo = ora.vordiv2uv(w / a, w2 / a)
        assert relerr(u, uo) < TOL and relerr(v, vo) < TOL
        cs = np.cos(gpu.y_Lat)[None, :, None]
        vg, dg = gpu.calc_UVCosLat2VorDiv(u * cs, v * cs)
        vr, dr = ora.uvcoslat2vordiv(u * cs, v * cs)
        assert relerr(vg, vr) < TOL and relerr(dg, dr) < TOL
        gpu.synchronize()
    finally:
        gpu.set_precision(P.SHT_PREC_FP64)


def test_default_truncation_of_a_factor_3_grid():
    """nm = -1 picks the model's default truncation (im - 1)/3 on a
    96-longitude grid, and the round trip of band-limited spectra holds."""
    P, W = pkg(), workloads()
    gpu = P.SpmlUtil(96, 48, 1, -1)
    try:
        assert gpu.nm == 31
        w = W.seeded_spectra(31, 4, 2.0, seed=3)
        assert relerr(gpu.wa_xya(gpu.xya_wa(w)), w) < TOL
    finally:
        gpu.final()
