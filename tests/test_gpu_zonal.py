"""Axisymmetric plans (iMax = 1): the DOGCM_MODE_AXISYM transform of SPMODEL's
wa_zonal_module (SpmlUtil_mod.f90:30-35, 210-211; lm = nm + 1, only m = 0),
the mode of the shipped experiments (exp/APEOGCirc/APEOGCircExp.nml:6-8:
IM = 1, JM = 64, KM = 60).

Oracle: the same CPU restatement on a 3-D grid, fed with longitude-constant
fields and m = 0 spectra; the m = 0 entries (l = n(n+1)) of its results are
the zonal transform.  Tolerance 1e-11 per field, as for the 3-D plans.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11
A = 6.371e6


def _embed(N, w):
    """zonal spectra (nb, N+1) -> full SPML layout (nb, (N+1)^2)."""
    full = np.zeros((w.shape[0], (N + 1) ** 2))
    n = np.arange(N + 1)
    full[:, n * (n + 1)] = w
    return full


def _extract(N, full):
    n = np.arange(N + 1)
    return full[:, n * (n + 1)]


def _zonal_spectra(N, nb, seed, power=1.5):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nb, N + 1)) * (np.arange(N + 1) + 1.0) ** -power


@pytest.fixture(scope="module")
def zplans():
    cache = {}

    def get(J, nm, a=1.0):
        key = (J, nm, a)
        if key not in cache:
            z = pkg().SpmlUtil(1, J, 1, nm, None, a)
            io = 16
            while io < 2 * z.nm + 2:
                io *= 2
            cache[key] = (z, O.OraclePlan(io, J, z.nm, a), io)
        return cache[key]

    yield get
    for z, _, _ in cache.values():
        z.final()


def test_zonal_defaults_and_index_map(zplans):
    z, _, _ = zplans(64, -1)
    assert z.zonal and z.im == 1 and z.nm == 42 and z.lm == 43   # (2 jm - 1) / 3
    assert z.l_nm(0, 0) == 1 and z.l_nm(42, 0) == 43
    assert z.l_nm(3, 1) == 0 and z.l_nm(43, 0) == 0
    assert z.nm_l(5) == (4, 0)
    assert np.allclose(z.rn, -np.arange(43) * np.arange(1, 44))


@pytest.mark.parametrize("J,nm", [(64, -1), (32, 10), (128, 84), (256, -1)])
def test_zonal_transforms_vs_oracle(J, nm, zplans):
    z, ora, io = zplans(J, nm)
    N = z.nm
    w = _zonal_spectra(N, 11, seed=J)
    x = np.random.default_rng(J + 1).standard_normal((11, J, 1))
    # synthesis, analysis, derivatives
    assert relerr(z.xya_wa(w), ora.xya_wa(_embed(N, w))[:, :, :1]) < TOL
    assert relerr(z.wa_xya(x), _extract(N, ora.wa_xya(np.repeat(x, io, axis=2)))) < TOL
    assert relerr(z.xya_GradMu_wa(w), ora.xya_gradmu_wa(_embed(N, w))[:, :, :1]) < TOL
    assert relerr(z.xya_GradLat_wa(w), ora.xya_gradlat_wa(_embed(N, w))[:, :, :1]) < TOL
    assert relerr(z.wa_DivMu_xya(x), _extract(N, ora.wa_divmu_xya(np.repeat(x, io, axis=2)))) < TOL
    assert np.abs(z.xya_GradLambda_wa(w)).max() == 0.0
    assert relerr(z.wa_Lapla_wa(w), _extract(N, ora.wa_lapla_wa(_embed(N, w)))) < TOL
    # the round trip is the identity on band-limited spectra
    assert relerr(z.wa_xya(z.xya_wa(w)), w) < TOL


@pytest.mark.parametrize("J,nm", [(64, -1), (128, 84)])
def test_zonal_vector_operators_vs_oracle(J, nm, zplans):
    z, ora, io = zplans(J, nm, A)
    N = z.nm
    vor = _zonal_spectra(N, 7, seed=3, power=2.0) / A
    div = _zonal_spectra(N, 7, seed=4, power=2.0) / A
    vor[:, 0] = div[:, 0] = 0.0
    u, v = z.calc_VorDiv2UV(vor, div)
    uo, vo = ora.vordiv2uv(_embed(N, vor), _embed(N, div))
    assert relerr(u, uo[:, :, :1]) < TOL and relerr(v, vo[:, :, :1]) < TOL
    cs = np.cos(z.y_Lat)[None, :, None]
    ov, od = z.calc_UVCosLat2VorDiv(u * cs, v * cs)
    rv, rd = ora.uvcoslat2vordiv(np.repeat(u * cs, io, axis=2), np.repeat(v * cs, io, axis=2))
    assert relerr(ov, _extract(N, rv)) < TOL and relerr(od, _extract(N, rd)) < TOL
    assert relerr(ov, vor) < TOL and relerr(od, div) < TOL
    xa = np.random.default_rng(5).standard_normal((7, J, 1))
    xb = np.random.default_rng(6).standard_normal((7, J, 1))
    ra = ora.wa_alphaoptr_xya(np.repeat(xa, io, axis=2), np.repeat(xb, io, axis=2))
    assert relerr(z.wa_AlphaOptr_xya(xa, xb), _extract(N, ra)) < TOL
    assert relerr(z.AvrLonLat_xy(xa[0]), ora.avrlonlat(np.repeat(xa[:1], io, axis=2))[0]) < 1e-13


def test_zonal_legendre_variants_and_split_agree(zplans):
    P = pkg()
    z, _, _ = zplans(64, -1)
    w = _zonal_spectra(z.nm, 60 * 8, seed=9)          # the shipped case: KM = 60 levels x 8 fields
    ref = z.xya_wa(w)
    for variant in (1, 2, 3):
        z.set_option(P.SHT_OPT_LEGENDRE_KERNEL, variant)
        assert relerr(z.xya_wa(w), ref) < 1e-13
    z.set_option(P.SHT_OPT_LEGENDRE_KERNEL, 0)
    z.set_precision(P.SHT_PREC_SPLIT)
    try:
        g = z.xya_wa(w)
        back = z.wa_xya(g)
        z.synchronize()
    finally:
        z.set_precision(P.SHT_PREC_FP64)
    assert relerr(g, ref) < TOL and relerr(back, w) < TOL


def test_zonal_plan_in_a_batch(zplans):
    """A zonal plan and a 3-D plan side by side in one multi-instance step."""
    P, W = pkg(), workloads()
    z, _, _ = zplans(64, -1)
    g3 = P.SpmlUtil(128, 64, 1, 42)
    try:
        wz = _zonal_spectra(z.nm, 40, seed=12)
        w3 = W.seeded_spectra(42, 24, 1.5, seed=13)
        bufs = [(z, torch.zeros((40, z.lm), dtype=torch.float64, device="cuda"),
                 torch.zeros((40, 64, 1), dtype=torch.float64, device="cuda"), wz),
                (g3, torch.zeros((24, g3.lm), dtype=torch.float64, device="cuda"),
                 torch.zeros((24, 64, 128), dtype=torch.float64, device="cuda"), w3)]
        m = P.MultiTransform()
        for p, wa, xya, _ in bufs:
            m.add(p, wa, xya)
        m.build(autotune=True)
        for _, wa, _, w in bufs:
            wa.copy_(torch.from_numpy(w))
        m.run(P.SHT_MULTI_SYNTHESIS)
        m.synchronize()
        for p, _, xya, w in bufs:
            assert relerr(xya.cpu().numpy(), p.xya_wa(w)) < 1e-12
        m.close()
    finally:
        g3.final()
