"""The benchmark configurations' whole batches through the C-ABI, against the
CPU oracle (not against the FP64 GPU path):

  C1  T85,  60 levels x 8 fields = 480 field-levels, both precisions: the
      tracer-tendency pattern of HBEBaroc_hspm_vfvm_mod.f90:160-172 (U, V from
      vorticity and divergence, a tracer grid, the flux products analysed back
      by w_AlphaOptr_xy);
  C2  T170, 60 x 12 = 720 field-levels, split precision: synthesis, and the
      analysis of the synthesised grid;
  C4  T341, 60 x 16 = 960 field-levels, split precision: synthesis, analysis,
      both horizontal gradients, AlphaOptr of two grids, and the backward-Euler
      diffusion round trip (order 8, dt nu = 1e-3).

Each GPU call covers the whole batch; the oracle checks it in slices of field-
levels, which keeps host memory bounded at T341 (4 GB per grid array).
Tolerance: 1e-11 per-field normwise relative error (max|gpu - ref| / max|ref|
per field-level), the bound the transform is specified to.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11
RADIUS = 6.371e6


@pytest.fixture(scope="module", autouse=True)
def oracle_threads():
    O.set_threads(os.cpu_count() or 1)


def _sliced(got, ref_fn, *inputs, step=96):
    """Largest relerr of `got` against ref_fn(*inputs) computed slice by slice."""
    worst = 0.0
    for b0 in range(0, len(got), step):
        ref = ref_fn(*(x[b0:b0 + step] for x in inputs))
        worst = max(worst, relerr(got[b0:b0 + step], ref))
    return worst


@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_c1_full_batch_tendency(prec):
    P, W = pkg(), workloads()
    c = W.CONFIGS["C1"]
    I, J, N = W.GRIDS[c["grid"]]
    nb = c["levels"] * c["fields"]
    gpu = P.SpmlUtil(I, J, 1, N, None, RADIUS)
    ora = O.OraclePlan(I, J, N, RADIUS)
    try:
        gpu.set_precision(P.SHT_PREC_SPLIT if prec == "split" else P.SHT_PREC_FP64)
        vor = W.seeded_spectra(N, nb, 2.0, seed=W.SEED + 1) / RADIUS
        div = W.seeded_spectra(N, nb, 2.0, seed=W.SEED + 2) / RADIUS
        T = W.seeded_spectra(N, nb, 1.5, seed=W.SEED + 3)
        U, V = gpu.calc_VorDiv2UV(vor, div)
        Tg = gpu.xya_wa(T)
        cs = np.cos(gpu.y_Lat)[None, :, None]
        A, B = Tg * U * cs, Tg * V * cs
        out = gpu.wa_AlphaOptr_xya(A, B)
        gpu.synchronize()
        assert relerr(U, ora.vordiv2uv(vor, div)[0]) < TOL
        assert relerr(V, ora.vordiv2uv(vor, div)[1]) < TOL
        assert relerr(Tg, ora.xya_wa(T)) < TOL
        assert relerr(out, ora.wa_alphaoptr_xya(A, B)) < TOL
    finally:
        gpu.final()


def test_c2_full_batch_split():
    P, W = pkg(), workloads()
    c = W.CONFIGS["C2"]
    I, J, N = W.GRIDS[c["grid"]]
    nb = c["levels"] * c["fields"]
    gpu = P.SpmlUtil(I, J, 1, N, None, RADIUS)
    ora = O.OraclePlan(I, J, N, RADIUS)
    try:
        gpu.set_precision(P.SHT_PREC_SPLIT)
        w = W.seeded_spectra(N, nb, c["power"])
        g = gpu.xya_wa(w)
        back = gpu.wa_xya(g)
        gpu.synchronize()
        assert _sliced(g, ora.xya_wa, w) < TOL
        assert _sliced(back, ora.wa_xya, g) < TOL
    finally:
        gpu.final()


def test_c4_full_batch_split():
    P, W = pkg(), workloads()
    c = W.CONFIGS["C4"]
    I, J, N = W.GRIDS[c["grid"]]
    nb = c["levels"] * c["fields"]
    gpu = P.SpmlUtil(I, J, 1, N, None, RADIUS)
    ora = O.OraclePlan(I, J, N, RADIUS)
    try:
        gpu.set_precision(P.SHT_PREC_SPLIT)
        w = W.seeded_spectra(N, nb, c["power"])
        g = gpu.xya_wa(w)
        gpu.synchronize()
        assert _sliced(g, ora.xya_wa, w) < TOL, "synthesis"
        back = gpu.wa_xya(g)
        gpu.synchronize()
        assert _sliced(back, ora.wa_xya, g) < TOL, "analysis"
        del back
        glon = gpu.xya_GradLon_wa(w)
        gpu.synchronize()
        assert _sliced(glon, ora.xya_gradlon_wa, w) < TOL, "GradLon"
        del glon
        glat = gpu.xya_GradLat_wa(w)
        gpu.synchronize()
        assert _sliced(glat, ora.xya_gradlat_wa, w) < TOL, "GradLat"
        alpha = gpu.wa_AlphaOptr_xya(g, glat)
        gpu.synchronize()
        assert _sliced(alpha, ora.wa_alphaoptr_xya, g, glat) < TOL, "AlphaOptr"
        del alpha, glat
        # backward-Euler lateral diffusion between an analysis and a synthesis
        coef = W.diffusion_coef(N, 8, 1e-3)
        wd = gpu.diffuse(gpu.wa_xya(g), coef, 1.0)
        gd = gpu.xya_wa(wd)
        gpu.synchronize()

        def ref_diffused(x):
            s = ora.wa_xya(x)
            return ora.xya_wa(ora.diffuse(s, coef, 1.0))
        assert _sliced(gd, ref_diffused, g) < TOL, "diffusion round trip"
    finally:
        gpu.final()
