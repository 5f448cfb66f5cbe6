"""Fused clients of the transform: the grid-space product epilogue and the
horizontal-gradient composites.

- w_AlphaOptrProd_xy(A, B, Q) = w_AlphaOptr_xy(A Q, B Q), the tracer flux
  divergence of HBEBaroc_hspm_vfvm_mod.f90:160-165 (Q = H cos(phi) T), with
  the products formed inside the longitude transform;
- xy_HGrad_w(w) = (xy_GradLon_w(w), xy_GradLat_w(w)) in one synthesis;
- xy_HGrad_xy(T) = the same of w_xy(T), the Redi/GM tracer gradients of
  physics/lphys/LPhys_RediGM_hspm_vfvm_mod.f90:432-440 (before 1/radius);
- xy_FluxDiv_xy(A, B) = xy_w(w_AlphaOptr_xy(A, B)), the Redi/GM flux
  divergence of the same file, :350-355.

Oracle: the CPU restatement, with the products formed in numpy and the
gradients composed from its single operators.  Tolerance 1e-11 per field, as
for every FP64 operator.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11
A = 6.371e6
# (I, J, N): T21, T85, T170, T341 -- the factor tile is staged in shared
# memory beside the data tile where both fit, else read from global memory
GRIDS = [(64, 32, 21), (256, 128, 85), (512, 256, 170), (1024, 512, 341)]


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


def _io(nm):
    """Longitude count of the 3-D oracle plan that stands in for a zonal one."""
    io = 16
    while io < 2 * nm + 2:
        io *= 2
    return io


def _grids(nb, J, I, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((nb, J, I))
    b = rng.standard_normal((nb, J, I))
    q = 1.0 + 0.5 * rng.standard_normal((nb, J, I))
    return a, b, q


@pytest.mark.parametrize("grid", GRIDS)
def test_alphaoptr_prod_vs_oracle(grid, plans):
    I, J, N = grid
    gpu, ora = plans(I, J, N, A)
    nb = 5 if N < 300 else 2
    a, b, q = _grids(nb, J, I, seed=N)
    ref = ora.wa_alphaoptr_xya(a * q, b * q)
    assert relerr(gpu.w_AlphaOptrProd_xy(a, b, q), ref) < TOL
    # the unfused composition through the library agrees as well
    assert relerr(gpu.w_AlphaOptr_xy(a * q, b * q), ref) < TOL


def test_alphaoptr_prod_device_pipelined_and_split(plans):
    gpu, ora = plans(128, 64, 42, A)
    P = pkg()
    nb = 100  # the host path runs as a pipeline of two chunks
    a, b, q = _grids(nb, 64, 128, seed=3)
    ref = ora.wa_alphaoptr_xya(a * q, b * q)
    assert relerr(gpu.w_AlphaOptrProd_xy(a, b, q), ref) < TOL
    ta, tb, tq = (torch.from_numpy(x).cuda() for x in (a, b, q))
    out = gpu.w_AlphaOptrProd_xy(ta, tb, tq)
    torch.cuda.synchronize()
    assert relerr(out.cpu().numpy(), ref) < TOL
    gpu.set_precision(P.SHT_PREC_SPLIT)
    try:
        w = gpu.w_AlphaOptrProd_xy(ta, tb, tq)
        torch.cuda.synchronize()
    finally:
        gpu.set_precision(P.SHT_PREC_FP64)
    assert relerr(w.cpu().numpy(), ref) < TOL


def test_alphaoptr_prod_one_level_and_zonal(plans):
    gpu, ora = plans(64, 32, 21, A)
    a, b, q = _grids(1, 32, 64, seed=7)
    assert relerr(gpu.w_AlphaOptrProd_xy(a[0], b[0], q[0]), ora.wa_alphaoptr_xya(a * q, b * q)[0]) < TOL
    z = pkg().SpmlUtil(1, 64, 1, -1, None, A)
    try:
        za, zb, zq = _grids(9, 64, 1, seed=8)
        io = _io(z.nm)
        full = O.OraclePlan(io, 64, z.nm, A)
        rep = lambda x: np.repeat(x, io, axis=2)
        ref = full.wa_alphaoptr_xya(rep(za * zq), rep(zb * zq))
        n = np.arange(z.nm + 1)
        assert relerr(z.w_AlphaOptrProd_xy(za, zb, zq), ref[:, n * (n + 1)]) < TOL
    finally:
        z.final()


def test_alphaoptr_prod_rejects_mismatched_shapes(plans):
    gpu, _ = plans(64, 32, 21)
    a, b, q = _grids(3, 32, 64, seed=9)
    with pytest.raises(pkg().SpmlError):
        gpu.w_AlphaOptrProd_xy(a, b, q[:2])


@pytest.mark.parametrize("grid", GRIDS)
def test_hgrad_vs_oracle(grid, plans):
    I, J, N = grid
    gpu, ora = plans(I, J, N)
    nb = 6 if N < 300 else 2
    w = workloads().seeded_spectra(N, nb, 1.5, seed=N)
    lon, lat = gpu.xy_HGrad_w(w)
    assert relerr(lon, ora.xya_gradlon_wa(w)) < TOL
    assert relerr(lat, ora.xya_gradlat_wa(w)) < TOL
    # the fused synthesis reproduces the two single operators
    assert relerr(lon, gpu.xy_GradLon_w(w)) < 1e-13 and relerr(lat, gpu.xy_GradLat_w(w)) < 1e-13
    x = np.random.default_rng(N + 1).standard_normal((nb, J, I))
    glon, glat = gpu.xy_HGrad_xy(x)
    wx = ora.wa_xya(x)
    assert relerr(glon, ora.xya_gradlon_wa(wx)) < TOL
    assert relerr(glat, ora.xya_gradlat_wa(wx)) < TOL


def test_hgrad_device_and_pipelined(plans):
    gpu, ora = plans(128, 64, 42)
    nb = 120
    x = np.random.default_rng(21).standard_normal((nb, 64, 128))
    wx = ora.wa_xya(x)
    rlon, rlat = ora.xya_gradlon_wa(wx), ora.xya_gradlat_wa(wx)
    lon, lat = gpu.xy_HGrad_xy(x)  # host arrays: a pipeline of two chunks
    assert relerr(lon, rlon) < TOL and relerr(lat, rlat) < TOL
    tlon, tlat = gpu.xy_HGrad_xy(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert relerr(tlon.cpu().numpy(), rlon) < TOL and relerr(tlat.cpu().numpy(), rlat) < TOL
    w = workloads().seeded_spectra(42, nb, 1.5, seed=22)
    slon, slat = gpu.xy_HGrad_w(torch.from_numpy(w).cuda())
    torch.cuda.synchronize()
    assert relerr(slon.cpu().numpy(), ora.xya_gradlon_wa(w)) < TOL
    assert relerr(slat.cpu().numpy(), ora.xya_gradlat_wa(w)) < TOL


def test_hgrad_zonal():
    z = pkg().SpmlUtil(1, 64, 1, -1)
    try:
        io = _io(z.nm)
        full = O.OraclePlan(io, 64, z.nm)
        n = np.arange(z.nm + 1)
        x = np.random.default_rng(5).standard_normal((4, 64, 1))
        wx = full.wa_xya(np.repeat(x, io, axis=2))
        lon, lat = z.xy_HGrad_xy(x)
        assert np.abs(lon).max() == 0.0
        assert relerr(lat, full.xya_gradlat_wa(wx)[:, :, :1]) < TOL
        w = np.zeros((4, (z.nm + 1) ** 2))
        w[:, n * (n + 1)] = z.w_xy(x)
        assert relerr(z.xy_HGrad_w(z.w_xy(x))[1], full.xya_gradlat_wa(w)[:, :, :1]) < TOL
    finally:
        z.final()


@pytest.mark.parametrize("grid", GRIDS[:3])
def test_fluxdiv_grid_to_grid_vs_oracle(grid, plans):
    I, J, N = grid
    gpu, ora = plans(I, J, N, A)
    a, b, _ = _grids(4, J, I, seed=N + 5)
    cs = np.cos(gpu.y_Lat)[None, :, None]
    a, b = a * cs, b * cs
    ref = ora.xya_wa(ora.wa_alphaoptr_xya(a, b))
    assert relerr(gpu.xy_FluxDiv_xy(a, b), ref) < TOL
    out = gpu.xy_FluxDiv_xy(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    torch.cuda.synchronize()
    assert relerr(out.cpu().numpy(), ref) < TOL


def test_fluxdiv_pipelined_and_zonal(plans):
    gpu, ora = plans(128, 64, 42, A)
    a, b, _ = _grids(100, 64, 128, seed=31)  # host arrays: a pipeline of two chunks
    assert relerr(gpu.xy_FluxDiv_xy(a, b), ora.xya_wa(ora.wa_alphaoptr_xya(a, b))) < TOL
    z = pkg().SpmlUtil(1, 64, 1, -1, None, A)
    try:
        za, zb, _ = _grids(5, 64, 1, seed=32)
        io = _io(z.nm)
        full = O.OraclePlan(io, 64, z.nm, A)
        rep = lambda x: np.repeat(x, io, axis=2)
        ref = full.xya_wa(full.wa_alphaoptr_xya(rep(za), rep(zb)))[:, :, :1]
        assert relerr(z.xy_FluxDiv_xy(za, zb), ref) < TOL
    finally:
        z.final()
