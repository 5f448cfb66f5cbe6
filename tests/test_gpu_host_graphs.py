"""Small host-pointer calls replayed as CUDA graphs (SHT_OPT_HOST_GRAPHS).

dogcm calls the transform one level at a time with host arrays
(HBEBaroc_hspm_vfvm_mod.f90:160-172, 388-441).  Such calls are staged through
the plan's page-locked buffer, and from the second call of an operator and
size on, their copies and kernels replay as one CUDA graph.  These tests
check that the graph path gives bit-identical results to direct launches:

- for single- and two-input operators, two-output operators, operators that
  keep a spectral temporary in the workspace, spectral-only operators and
  reductions;
- for changing caller arrays (the graph names only plan buffers);
- across plan-buffer reallocations (larger calls in between), precision
  switches and the axisymmetric plan;
- with the same kernel count per call.
"""
import numpy as np
import pytest

from conftest import pkg

pytestmark = pytest.mark.gpu


def _plan(I, J, N, graphs, a=6.371e6):
    P = pkg()
    s = P.SpmlUtil(I, J, 1, N, None, a)
    s.set_option(P.SHT_OPT_HOST_GRAPHS, 1 if graphs else 0)
    return s


def _ops(s, rng):
    """(name, callable) pairs over fresh random inputs; each returns arrays."""
    J, I, L = s.jm, s.im, s.lm
    x = [rng.standard_normal((J, I)) for _ in range(3)]
    w = [rng.standard_normal(L) * 1e-6 for _ in range(2)]
    return [
        ("w_xy", lambda: [s.w_xy(x[0])]),
        ("xy_w", lambda: [s.xy_w(w[0])]),
        ("xy_GradLat_w", lambda: [s.xy_GradLat_w(w[1])]),
        ("w_AlphaOptr_xy", lambda: [s.w_AlphaOptr_xy(x[0], x[1])]),
        ("w_AlphaOptrProd_xy", lambda: [s.w_AlphaOptrProd_xy(x[0], x[1], x[2])]),
        ("calc_VorDiv2UV", lambda: list(s.calc_VorDiv2UV(w[0], w[1]))),
        ("calc_UVCosLat2VorDiv", lambda: list(s.calc_UVCosLat2VorDiv(x[1], x[2]))),
        ("xy_HGrad_xy", lambda: list(s.xy_HGrad_xy(x[2]))),
        ("xy_FluxDiv_xy", lambda: [s.xy_FluxDiv_xy(x[0], x[2])]),
        ("w_Lapla_w", lambda: [s.w_Lapla_w(w[0])]),
        ("AvrLonLat_xy", lambda: [np.atleast_1d(s.AvrLonLat_xy(x[1]))]),
    ]


@pytest.mark.parametrize("I,J,N", [(64, 32, 21), (256, 128, 85)])
def test_graph_replays_match_direct_launches(I, J, N):
    P = pkg()
    sg, sd = _plan(I, J, N, True), _plan(I, J, N, False)
    try:
        for rep in range(3):   # direct, captured, replayed
            rng_g, rng_d = np.random.default_rng(rep), np.random.default_rng(rep)
            for (name, fg), (_, fd) in zip(_ops(sg, rng_g), _ops(sd, rng_d)):
                n0 = P.launch_count()
                rg = fg()
                ng = P.launch_count() - n0
                n0 = P.launch_count()
                rd = fd()
                nd = P.launch_count() - n0
                for a, b in zip(rg, rd):
                    assert np.array_equal(a, b), (name, rep)
                assert ng == nd, (name, rep, ng, nd)
        assert sg.get_option(P.SHT_OPT_HOST_GRAPH_COUNT) >= 10
        assert sd.get_option(P.SHT_OPT_HOST_GRAPH_COUNT) == 0
    finally:
        sg.final()
        sd.final()


def test_graphs_follow_caller_arrays_and_buffer_growth():
    P = pkg()
    sg, sd = _plan(256, 128, 85, True), _plan(256, 128, 85, False)
    try:
        rng = np.random.default_rng(7)
        xs = [rng.standard_normal((128, 256)) for _ in range(4)]
        big = rng.standard_normal((120, 128, 256))      # chunked host path: new staging and workspace
        seq = [0, 1, 2, 3, 1, "big", 0, 2, "big", 3, 3]
        for k in seq:
            if k == "big":
                assert np.array_equal(sg.wa_xya(big), sd.wa_xya(big))
            else:
                wg, wd = sg.w_xy(xs[k]), sd.w_xy(xs[k])
                assert np.array_equal(wg, wd), k
                assert np.array_equal(sg.xy_w(wg), sd.xy_w(wd)), k
        assert sg.get_option(P.SHT_OPT_HOST_GRAPH_COUNT) >= 1
        # batches of a few levels are staged too, each size its own graph
        for nb in (2, 5, 2, 5, 2):
            x = rng.standard_normal((nb, 128, 256))
            assert np.array_equal(sg.wa_xya(x), sd.wa_xya(x)), nb
    finally:
        sg.final()
        sd.final()


def test_graphs_per_precision_and_kernel_choice():
    P = pkg()
    sg, sd = _plan(256, 128, 85, True), _plan(256, 128, 85, False)
    try:
        rng = np.random.default_rng(11)
        x = rng.standard_normal((128, 256))
        for prec in (P.SHT_PREC_SPLIT, P.SHT_PREC_FP64, P.SHT_PREC_SPLIT, P.SHT_PREC_FP64):
            sg.set_precision(prec)
            sd.set_precision(prec)
            for _ in range(3):
                assert np.array_equal(sg.w_xy(x), sd.w_xy(x)), prec
        for kern in (1, 2, 0):
            sg.set_option(P.SHT_OPT_LEGENDRE_KERNEL, kern)
            sd.set_option(P.SHT_OPT_LEGENDRE_KERNEL, kern)
            for _ in range(3):
                assert np.array_equal(sg.w_xy(x), sd.w_xy(x)), kern
        # the single-kernel small-grid transform replays as a graph as well
        tg, td = _plan(64, 32, 21, True), _plan(64, 32, 21, False)
        try:
            y = rng.standard_normal((32, 64))
            for s_ in (tg, td):
                s_.set_option(P.SHT_OPT_LEGENDRE_KERNEL, 4)
            for _ in range(3):
                assert np.array_equal(tg.w_xy(y), td.w_xy(y))
                assert np.array_equal(tg.xy_w(tg.w_xy(y)), td.xy_w(td.w_xy(y)))
            assert tg.get_option(P.SHT_OPT_HOST_GRAPH_COUNT) > 0
        finally:
            tg.final()
            td.final()
        # switching the option off keeps results and stops new captures
        sg.set_option(P.SHT_OPT_HOST_GRAPHS, 0)
        n = sg.get_option(P.SHT_OPT_HOST_GRAPH_COUNT)
        for _ in range(3):
            assert np.array_equal(sg.xy_GradLon_w(sg.w_xy(x)), sd.xy_GradLon_w(sd.w_xy(x)))
        assert sg.get_option(P.SHT_OPT_HOST_GRAPH_COUNT) == n
    finally:
        sg.final()
        sd.final()


def test_zonal_plan_graphs():
    sg, sd = _plan(1, 64, -1, True), _plan(1, 64, -1, False)
    try:
        rng = np.random.default_rng(3)
        for _ in range(4):
            x = rng.standard_normal((64, 1))
            assert np.array_equal(sg.w_xy(x), sd.w_xy(x))
            w = sg.w_xy(x)
            assert np.array_equal(sg.xy_GradLat_w(w), sd.xy_GradLat_w(w))
    finally:
        sg.final()
        sd.final()


def test_option_arguments():
    P = pkg()
    s = _plan(64, 32, 21, True)
    try:
        assert s.get_option(P.SHT_OPT_HOST_GRAPHS) == 1
        with pytest.raises(P.SpmlError):
            s.set_option(P.SHT_OPT_HOST_GRAPHS, 2)
        with pytest.raises(P.SpmlError):
            s.set_option(P.SHT_OPT_HOST_GRAPH_COUNT, 0)
    finally:
        s.final()


@pytest.mark.parametrize("nb", [97, 250, 385])
def test_pipelined_host_calls_match_device_calls(nb):
    """Host-pointer batches of 96 field-levels and more run as a pipeline of
    2 to 8 chunks of ramped sizes (upload, kernels and download on three
    streams): every field-level equals the device-pointer call's bit for bit,
    for an analysis, a synthesis and a two-output operator."""
    import torch

    s = _plan(128, 64, 42, True)
    try:
        rng = np.random.default_rng(nb)
        x = rng.standard_normal((nb, 64, 128))
        y = rng.standard_normal((nb, 64, 128))
        w = s.xya_wa(s.wa_xya(x))  # band-limited spectra
        xd, yd, wd = (torch.from_numpy(a).cuda() for a in (x, y, w))
        assert np.array_equal(s.wa_xya(x), s.wa_xya(xd).cpu().numpy())
        assert np.array_equal(s.xya_wa(w), s.xya_wa(wd).cpu().numpy())
        vh, dh = s.calc_UVCosLat2VorDiv(x, y)
        vd, dd = s.calc_UVCosLat2VorDiv(xd, yd)
        assert np.array_equal(vh, vd.cpu().numpy()) and np.array_equal(dh, dd.cpu().numpy())
    finally:
        s.final()
