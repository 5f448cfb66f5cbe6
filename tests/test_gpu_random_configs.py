"""Seeded random configurations against the oracle: Gauss grids (jm = im/2,
powers of two and the factor-3 counts), truncations from 4 to the default,
batches of 1 to 40 field-levels, every Legendre kernel choice (0-4) and every
precision mode, through eight operators (analysis, synthesis, GradMu, DivMu,
both AlphaOptr forms, U and V from vorticity and divergence).

The fixed parametrised cases elsewhere take the default truncations and the
bench batches; these cover the combinations in between.  Bound: 1e-11 per
field against the oracle.
"""
import numpy as np
import pytest

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _cases(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        I = int(rng.choice([16, 32, 64, 96, 128, 192, 256]))
        N = int(rng.integers(4, (I - 1) // 3 + 1))
        out.append((I, I // 2, N, int(rng.integers(1, 41)), int(rng.integers(0, 5)), int(rng.integers(0, 3)),
                    int(rng.integers(0, 2**31))))
    return out


@pytest.mark.parametrize("I,J,N,nb,kern,prec,seed", _cases(20261204, 40))
def test_random_configuration(I, J, N, nb, kern, prec, seed):
    P, W = pkg(), workloads()
    a = 6.371e6
    sp = P.SpmlUtil(I, J, 1, N, None, a)
    try:
        ora = O.OraclePlan(I, J, N, a)
        sp.set_option(P.SHT_OPT_LEGENDRE_KERNEL, kern)
        sp.set_precision([P.SHT_PREC_FP64, P.SHT_PREC_SPLIT, P.SHT_PREC_AUTO][prec])
        rng = np.random.default_rng(seed)
        w, w2 = W.seeded_spectra(N, nb, 1.5, rng=rng), W.seeded_spectra(N, nb, 2.0, rng=rng)
        x, y = rng.standard_normal((nb, J, I)), rng.standard_normal((nb, J, I))
        res = {
            "xy_w": relerr(sp.xya_wa(w), ora.xya_wa(w)),
            "w_xy": relerr(sp.wa_xya(x), ora.wa_xya(x)),
            "gradmu": relerr(sp.xya_GradMu_wa(w), ora.xya_gradmu_wa(w)),
            "divmu": relerr(sp.wa_DivMu_xya(x), ora.wa_divmu_xya(x)),
            "alpha_w": relerr(sp.wa_AlphaOptr_xya(x, y), ora.wa_alphaoptr_xya(x, y)),
            "alpha_x": relerr(sp.xya_AlphaOptr_wa(w, w2), ora.xya_alphaoptr_wa(w, w2)),
        }
        u, v = sp.calc_VorDiv2UV(w, w2)
        uo, vo = ora.vordiv2uv(w, w2)
        res["U"], res["V"] = relerr(u, uo), relerr(v, vo)
        bad = {k: e for k, e in res.items() if not e < TOL}
        assert not bad, bad
    finally:
        sp.final()
