"""CPU oracle: pinned against the golden vectors and the known-answer tests.

The golden vectors are an independent scipy/numpy evaluation of the written
specification (tests/golden/make_golden.py).  The known-answer tests are the
identities the reference's documentation implies
(doc/description/ogcm/space_discretization.tex) and the in-tree pins on the
spectral layout (l_nm, rn, the 1/sqrt2 seeding of the experiments).
"""
import math

import numpy as np
import pytest
from scipy.special import roots_legendre

import oracle as O
from conftest import load_golden, relerr

TOL = 1e-12


@pytest.mark.parametrize("tag", ["T21", "T10", "T15_I48"])
def test_oracle_matches_golden(tag):
    g = load_golden(tag)
    p = O.OraclePlan(int(g["I"]), int(g["J"]), int(g["N"]), float(g["radius"]))
    cs = np.cos(np.arcsin(g["mu"]))[None, :, None]
    checks = {
        "xy_w": (p.xya_wa(g["w"]), g["xy_w"]),
        "w_xy_rand": (p.wa_xya(g["grid_rand"]), g["w_xy_rand"]),
        "gradlambda": (p.xya_gradlambda_wa(g["w"]), g["gradlambda"]),
        "gradmu": (p.xya_gradmu_wa(g["w"]), g["gradmu"]),
        "gradlon": (p.xya_gradlon_wa(g["w"]), g["gradlon"]),
        "gradlat": (p.xya_gradlat_wa(g["w"]), g["gradlat"]),
        "divlambda": (p.wa_divlambda_xya(g["divA"]), g["divlambda"]),
        "divmu": (p.wa_divmu_xya(g["divB"]), g["divmu"]),
        "w_alpha": (p.wa_alphaoptr_xya(g["divA"], g["divB"]), g["w_alpha"]),
        "xy_alpha": (p.xya_alphaoptr_wa(g["w"], g["w2"]), g["xy_alpha"]),
        "avr": (p.avrlonlat(g["xy_w"]), g["avr"]),
    }
    u, v = p.vordiv2uv(g["w"], g["w2"])
    checks["U"] = (u, g["U"])
    checks["V"] = (v, g["V"])
    vo, di = p.uvcoslat2vordiv(g["U"] * cs, g["V"] * cs)
    checks["vor"] = (vo, g["vor"])
    checks["div"] = (di, g["div"])
    bad = {k: relerr(a, b) for k, (a, b) in checks.items() if relerr(a, b) > (2e-12 if k not in ("vor", "div") else 2e-11)}
    assert not bad, bad


@pytest.mark.parametrize("J", [2, 16, 32, 128, 512])
def test_gauss_nodes_match_scipy(J):
    mu, w = O.gauss(J)
    x, wx = roots_legendre(J)
    assert np.abs(mu - x).max() < 1e-14
    assert np.abs(2 * w - wx).max() < 1e-13
    assert abs(w.sum() - 1.0) < 1e-14
    # exact for mu^{2k}, 2k <= 2J - 1
    for k in range(J):
        assert abs(np.sum(w * mu ** (2 * k)) - 1.0 / (2 * k + 1)) < 1e-13


def test_index_maps():
    # l_nm(n,m) = n(n+1)+m+1; l=1 is (0,0) (HBEBarot_hspm_vfvm_mod.f90:295-298)
    assert O.l_nm(0, 0) == 1
    for l in range(1, 500):
        n, m = O.nm_l(l)
        assert -n <= m <= n
        assert O.l_nm(n, m) == l


@pytest.mark.parametrize("grid", [(64, 32, 21), (128, 64, 42), (32, 16, 10)])
def test_round_trip_identity(grid):
    I, J, N = grid
    rng = np.random.default_rng(7)
    p = O.OraclePlan(I, J, N, 1.0)
    w = rng.standard_normal((3, p.lm))
    w[:, 0] = rng.standard_normal(3)
    for n in range(N + 1):  # keep the m=0 entries real by construction of the layout
        pass
    assert relerr(p.wa_xya(p.xya_wa(w)), w) < 1e-13


def test_single_mode_closed_form():
    """xy_w of a unit coefficient is sqrt2 Pbar_n^m cos(m lambda) (m > 0), Pbar_n^0 (m = 0)."""
    from scipy.special import lpmv
    I, J, N = 64, 32, 21
    p = O.OraclePlan(I, J, N, 1.0)
    xl, yl, _, _ = p.grid_info()
    mu = np.sin(yl)
    for (n, m) in [(0, 0), (5, 0), (4, 3), (21, 21), (13, 7)]:
        w = np.zeros(p.lm)
        w[O.l_nm(n, m) - 1] = 1.0
        g = p.xya_wa(w)[0]
        norm = math.sqrt((2 * n + 1) * math.factorial(n - m) / math.factorial(n + m))
        pb = ((-1) ** m) * norm * lpmv(m, n, mu)
        ref = pb[:, None] * np.cos(m * xl)[None, :] * (math.sqrt(2.0) if m else 1.0)
        assert np.abs(g - ref).max() < 1e-12
        if m:
            w[:] = 0
            w[O.l_nm(n, -m) - 1] = 1.0
            g = p.xya_wa(w)[0]
            ref = -pb[:, None] * np.sin(m * xl)[None, :] * math.sqrt(2.0)
            assert np.abs(g - ref).max() < 1e-12


def test_sqrt2_seeding_pin():
    """The 1/sqrt2 seeding of exp/BarotRossby (DOGCM_Exp_BarotRossby_mod.f90:121-123) gives an
    m != 0 mode the same mean square as a unit m = 0 mode."""
    p = O.OraclePlan(64, 32, 21, 1.0)
    w0 = np.zeros(p.lm); w0[O.l_nm(4, 0) - 1] = 1.0
    w1 = np.zeros(p.lm); w1[O.l_nm(4, 3) - 1] = 1.0 / math.sqrt(2.0)
    e0 = p.avrlonlat(p.xya_wa(w0) ** 2)[0]
    e1 = p.avrlonlat(p.xya_wa(w1) ** 2)[0]
    assert abs(e0 - 1.0) < 1e-13
    assert abs(e1 - 0.5) < 1e-13


def test_laplacian_and_gradlambda():
    p = O.OraclePlan(64, 32, 21, 1.0)
    rn = p.rn()
    for l in range(1, p.lm + 1):
        n, m = O.nm_l(l)
        assert rn[l - 1] == -n * (n + 1)
    rng = np.random.default_rng(3)
    w = rng.standard_normal((2, p.lm))
    lap = p.wa_lapla_wa(w)
    assert relerr(p.wa_laplainv_wa(lap)[:, 1:], w[:, 1:]) < 1e-14
    assert np.all(p.wa_laplainv_wa(w)[:, 0] == 0.0)
    # GradLambda == i m in spectral space: w'(n,m) = -m w(n,-m), w'(n,-m) = m w(n,m)
    gl = p.wa_xya(p.xya_gradlambda_wa(w))
    ref = np.zeros_like(w)
    for l in range(1, p.lm + 1):
        n, m = O.nm_l(l)
        ref[:, l - 1] = -m * w[:, O.l_nm(n, -m) - 1]
    assert relerr(gl, ref) < 1e-13


def test_vordiv_round_trip():
    """calc_UVCosLat2VorDiv(calc_VorDiv2UV(vor, div) cos) == (vor, div) for band-limited
    fields with the n = 0 modes removed."""
    a = 6.371e6
    p = O.OraclePlan(64, 32, 21, a)
    rng = np.random.default_rng(5)
    vor = rng.standard_normal((2, p.lm)) / a
    div = rng.standard_normal((2, p.lm)) / a
    vor[:, 0] = div[:, 0] = 0.0
    u, v = p.vordiv2uv(vor, div)
    cs = np.cos(p.grid_info()[1])[None, :, None]
    vo, di = p.uvcoslat2vordiv(u * cs, v * cs)
    # the truncation at N drops the degree N+1 part of U cos, V cos; compare up to N-1
    n_of_l = np.floor(np.sqrt(np.arange(p.lm)))
    keep = n_of_l < 21
    assert relerr(vo[:, keep], vor[:, keep]) < 1e-11
    assert relerr(di[:, keep], div[:, keep]) < 1e-11


def test_mean_of_y00():
    p = O.OraclePlan(64, 32, 21, 1.0)
    w = np.zeros(p.lm); w[0] = 1.0
    assert abs(p.avrlonlat(p.xya_wa(w))[0] - 1.0) < 1e-15
    assert abs(p.intlonlat(p.xya_wa(w))[0] - 4 * math.pi) < 1e-13


def test_recurrence_identity():
    """(1-mu^2) dPbar_n^m/dmu from the eps recurrence (space_discretization.tex:250-252)
    equals the classical (n+m) P_{n-1} - n mu P_n identity (via xy_GradMu_w of a unit mode)."""
    from scipy.special import lpmv
    p = O.OraclePlan(64, 32, 21, 1.0)
    xl, yl, _, _ = p.grid_info()
    mu = np.sin(yl)
    n, m = 9, 4
    w = np.zeros(p.lm); w[O.l_nm(n, m) - 1] = 1.0 / math.sqrt(2.0)
    g = p.xya_gradmu_wa(w)[0]
    norm = math.sqrt((2 * n + 1) * math.factorial(n - m) / math.factorial(n + m))
    h = ((-1) ** m) * norm * ((n + m) * lpmv(m, n - 1, mu) - n * mu * lpmv(m, n, mu))
    ref = h[:, None] * np.cos(m * xl)[None, :]
    assert np.abs(g - ref).max() < 1e-12
