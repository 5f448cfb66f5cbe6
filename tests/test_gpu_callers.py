"""Batched callers (dennou-ogcm_b200/callers.py): the spectral parts of the
per-level loops of HBEBaroc_HTRCRHS (HBEBaroc_hspm_vfvm_mod.f90:160-172),
HBEBaroc_MOMRHS_VorDivForm (:430-441) and HBEDiagnose_VorDiv
(HBEDiagnose_hspm_vfvm_mod.f90:276-284) as calls over all levels.

Oracle: the loops' formulas composed from the CPU restatement's operators as
the reference writes them (w_AlphaOptr_xy(B, -A) for the divergence
tendency, not the calc_UVCosLat2VorDiv identity the batched form uses).
The level-by-level form through the library must agree with the batched one.
Tolerance 1e-11 per field, as for every FP64 operator.
"""
import importlib

import numpy as np
import pytest
import torch

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11
A = 6.371e6


def callers():
    return importlib.import_module("dennou-ogcm_b200.callers")


@pytest.fixture(scope="module")
def t42():
    I, J, N = workloads().GRIDS["T42"]
    sp = pkg().SpmlUtil(I, J, 12, N, None, A)
    yield sp, O.OraclePlan(I, J, N, A)
    sp.final()


def _grids(K, J, I, n, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((K, J, I)) for _ in range(n)]


def test_htrc_rhs_batched_vs_oracle_and_per_level(t42):
    sp, ora = t42
    C = callers()
    K = 12
    u, v, tmp, vflx, hphys = _grids(K, sp.jm, sp.im, 5, seed=1)
    n = np.floor(np.sqrt(np.arange(sp.lm)))
    filt = np.exp(-((n / sp.nm) ** 8))  # an AdvFilter-like spectral taper
    w = ora.wa_xya(vflx) - ora.wa_alphaoptr_xya(u * tmp, v * tmp)
    ref = ora.xya_wa(w * filt[None, :]) + hphys
    d = [torch.from_numpy(x).cuda() for x in (u, v, tmp, vflx)]
    f, hp = torch.from_numpy(filt).cuda(), torch.from_numpy(hphys).cuda()
    out = C.htrc_rhs(sp, *d, f, hp)
    lvl = C.per_level(C.htrc_rhs, sp, *d, f, hp)
    torch.cuda.synchronize()
    assert relerr(out.cpu().numpy(), ref) < TOL
    assert relerr(lvl.cpu().numpy(), out.cpu().numpy()) < 1e-13


def test_momrhs_vordiv_batched_vs_oracle_and_per_level(t42):
    sp, ora = t42
    C = callers()
    K = 12
    a, b, c = _grids(K, sp.jm, sp.im, 3, seed=2)
    cs = np.cos(sp.y_Lat)[None, :, None]
    a, b = a * cs, b * cs  # xy_A and xy_B carry cos(phi)
    vor_rhs = -ora.wa_alphaoptr_xya(a, b)
    div_rhs = ora.wa_alphaoptr_xya(b, -a) - ora.wa_lapla_wa(ora.wa_xya(c))
    ur, vr = ora.vordiv2uv(vor_rhs, div_rhs)
    d = [torch.from_numpy(x).cuda() for x in (a, b, c)]
    u, v = C.momrhs_vordiv(sp, *d)
    ul, vl = C.per_level(C.momrhs_vordiv, sp, *d)
    torch.cuda.synchronize()
    assert relerr(u.cpu().numpy(), ur) < TOL and relerr(v.cpu().numpy(), vr) < TOL
    assert relerr(ul.cpu().numpy(), u.cpu().numpy()) < 1e-13
    assert relerr(vl.cpu().numpy(), v.cpu().numpy()) < 1e-13


def test_momrhs_vordiv_fma_vs_oracle(t42):
    """Products formed in the load: A = cos(phi)(Vor U + za), B = cos(phi)(Vor V + zb)."""
    sp, ora = t42
    C = callers()
    K = 12
    u, v, vor, za, zb, c = _grids(K, sp.jm, sp.im, 6, seed=4)
    cs = np.cos(sp.y_Lat)[None, :, None]
    a, b = cs * (vor * u + za), cs * (vor * v + zb)
    vor_rhs = -ora.wa_alphaoptr_xya(a, b)
    div_rhs = ora.wa_alphaoptr_xya(b, -a) - ora.wa_lapla_wa(ora.wa_xya(c))
    ur, vr = ora.vordiv2uv(vor_rhs, div_rhs)
    d = [torch.from_numpy(x).cuda() for x in (u, v, vor, za, zb, c)]
    gu, gv = C.momrhs_vordiv_fma(sp, *d)
    torch.cuda.synchronize()
    assert relerr(gu.cpu().numpy(), ur) < TOL and relerr(gv.cpu().numpy(), vr) < TOL


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("with_sums", [True, False])
def test_uvcoslat2vordiv_fma_vs_oracle(t42, where, with_sums):
    """The fused entry point against calc_UVCosLat2VorDiv of the products, both
    array kinds, with and without the added terms."""
    sp, ora = t42
    u, v, q, za, zb = _grids(5, sp.jm, sp.im, 5, seed=5)
    if not with_sums:
        za = zb = None
    cs = np.cos(sp.y_Lat)[None, :, None]
    a = cs * (u * q + (za if with_sums else 0.0))
    b = cs * (v * q + (zb if with_sums else 0.0))
    rv, rd = ora.uvcoslat2vordiv(a, b)
    xs = [u, v, q, za, zb]
    if where == "device":
        xs = [None if x is None else torch.from_numpy(x).cuda() for x in xs]
    gv, gd = sp.calc_UVCosLat2VorDiv_fma(*xs)
    if where == "device":
        torch.cuda.synchronize()
        gv, gd = gv.cpu().numpy(), gd.cpu().numpy()
    assert relerr(gv, rv) < TOL and relerr(gd, rd) < TOL


def test_uvcoslat2vordiv_fma_split_and_zonal():
    """Split precision at T42, and the zonal plan (im = 1) against a 3-D oracle
    plan of longitude-constant grids (its m = 0 coefficients)."""
    P, W = pkg(), workloads()
    I, J, N = W.GRIDS["T42"]
    sp = P.SpmlUtil(I, J, 1, N, None, A)
    ora = O.OraclePlan(I, J, N, A)
    try:
        sp.set_precision(P.SHT_PREC_SPLIT)
        u, v, q, za, zb = _grids(6, J, I, 5, seed=6)
        cs = np.cos(sp.y_Lat)[None, :, None]
        rv, rd = ora.uvcoslat2vordiv(cs * (u * q + za), cs * (v * q + zb))
        gv, gd = sp.calc_UVCosLat2VorDiv_fma(*(torch.from_numpy(x).cuda() for x in (u, v, q, za, zb)))
        torch.cuda.synchronize()
        assert relerr(gv.cpu().numpy(), rv) < TOL and relerr(gd.cpu().numpy(), rd) < TOL
    finally:
        sp.final()
    z = P.SpmlUtil(1, 64, 1, -1, None, A)
    try:
        io = 16
        while io < 2 * z.nm + 2:
            io *= 2
        full = O.OraclePlan(io, 64, z.nm, A)
        u, v, q, za, zb = _grids(7, 64, 1, 5, seed=8)
        cs = np.cos(z.y_Lat)[None, :, None]
        rep = lambda x: np.repeat(x, io, axis=2)
        rv, rd = full.uvcoslat2vordiv(rep(cs * (u * q + za)), rep(cs * (v * q + zb)))
        n = np.arange(z.nm + 1)
        gv, gd = z.calc_UVCosLat2VorDiv_fma(u, v, q, za, zb)
        assert relerr(gv, rv[:, n * (n + 1)]) < TOL and relerr(gd, rd[:, n * (n + 1)]) < TOL
    finally:
        z.final()


def test_uvcoslat2vordiv_fma_rejects_one_sum(t42):
    sp, _ = t42
    u, v, q, za = _grids(2, sp.jm, sp.im, 4, seed=7)
    with pytest.raises(pkg().SpmlError):
        sp.calc_UVCosLat2VorDiv_fma(u, v, q, za, None)


def test_diagnose_vordiv_batched_vs_oracle_and_per_level(t42):
    sp, ora = t42
    C = callers()
    u, v = _grids(12, sp.jm, sp.im, 2, seed=3)
    cs = np.cos(sp.y_Lat)[None, :, None]
    wv, wd = ora.uvcoslat2vordiv(u * cs, v * cs)
    rv, rd = ora.xya_wa(wv), ora.xya_wa(wd)
    du, dv = torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()
    gv, gd = C.diagnose_vordiv(sp, du, dv)
    lv, ld = C.per_level(C.diagnose_vordiv, sp, du, dv)
    torch.cuda.synchronize()
    assert relerr(gv.cpu().numpy(), rv) < TOL and relerr(gd.cpu().numpy(), rd) < TOL
    assert relerr(lv.cpu().numpy(), gv.cpu().numpy()) < 1e-13
    assert relerr(ld.cpu().numpy(), gd.cpu().numpy()) < 1e-13
