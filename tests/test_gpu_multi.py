"""Multi-instance batches (sht_multi_* through MultiTransform): mixed truncations
in one step, per-plan tuning, CUDA-graph replay.

Every instance must give what a single batched call on its own plan gives, and
a few instances are checked against the CPU oracle.  Tolerances: 1e-12 against
the single-plan GPU path (the tuner may pick another FP64 kernel, which sums
in another order), 1e-11 against the oracle and for split precision.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import pkg, relerr, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plans():
    P, W = pkg(), workloads()
    out = {g: P.SpmlUtil(*W.GRIDS[g][:2], 1, W.GRIDS[g][2]) for g in ("T21", "T42", "T85", "T170")}
    yield out
    for p in out.values():
        p.final()


def _instances(plans, count, max_nb=None, seed=7):
    """C3-style instance list with its spectra (on the GPU) and grid buffers."""
    W = workloads()
    rng = np.random.default_rng(seed)
    out = []
    for d in W.mixed_instances(count, seed=seed):
        nb = d["levels"] * d["fields"]
        if max_nb:
            nb = min(nb, max_nb)
        p = plans[d["grid"]]
        w = W.seeded_spectra(p.nm, nb, 1.5, rng=rng)
        out.append(dict(grid=d["grid"], plan=p, w=w,
                        wa=torch.zeros((nb, p.lm), dtype=torch.float64, device="cuda"),
                        xya=torch.zeros((nb, p.jm, p.im), dtype=torch.float64, device="cuda")))
    return out


def _build(plans, insts, **kw):
    m = pkg().MultiTransform()
    for x in insts:
        m.add(x["plan"], x["wa"], x["xya"])
    m.build(**kw)
    for x in insts:  # build runs steps on the arrays: fill them afterwards
        x["wa"].copy_(torch.from_numpy(x["w"]))
    torch.cuda.synchronize()
    return m


def test_multi_matches_single_plan_and_oracle(plans):
    P = pkg()
    insts = _instances(plans, 16, max_nb=96)
    m = _build(plans, insts, autotune=True)
    try:
        groups = m.groups()
        assert len(groups) == 4 and sum(g["ncol"] for g in groups) == sum(x["w"].shape[0] for x in insts)
        assert all(g["tuned_ms"] > 0 for g in groups)
        m.run(P.SHT_MULTI_SYNTHESIS)
        m.synchronize()
        for x in insts:
            ref = x["plan"].xya_wa(x["w"])
            assert relerr(x["xya"].cpu().numpy(), ref) < 1e-12, x["grid"]
        m.run(P.SHT_MULTI_ANALYSIS)
        m.synchronize()
        for x in insts:
            assert relerr(x["wa"].cpu().numpy(), x["w"]) < 1e-11, x["grid"]
            assert relerr(x["wa"].cpu().numpy(), x["plan"].wa_xya(x["xya"].cpu().numpy())) < 1e-12
        # two instances against the CPU oracle
        for x in [i for i in insts if i["grid"] in ("T21", "T42")][:2]:
            ora = O.OraclePlan(x["plan"].im, x["plan"].jm, x["plan"].nm, 1.0)
            assert relerr(x["xya"].cpu().numpy(), ora.xya_wa(x["w"])) < 1e-11
    finally:
        m.close()


def test_multi_graph_replay_equals_stage_by_stage(plans):
    P = pkg()
    a = _instances(plans, 15, max_nb=40, seed=11)  # 15: every grid appears (8:4:2:1)
    b = _instances(plans, 15, max_nb=40, seed=11)
    ma = _build(plans, a, autotune=False, graph=True)
    mb = _build(plans, b, autotune=False, graph=False)
    try:
        for _ in range(3):
            ma.run(P.SHT_MULTI_ROUND_TRIP)
            mb.run(P.SHT_MULTI_ROUND_TRIP)
        ma.synchronize()
        mb.synchronize()
        for x, y in zip(a, b):
            assert torch.equal(x["wa"], y["wa"]) and torch.equal(x["xya"], y["xya"])
            assert relerr(x["wa"].cpu().numpy(), x["w"]) < 1e-11
        # the counted kernels are the ones a replay launches
        n = ma.kernels(P.SHT_MULTI_ROUND_TRIP)
        assert n >= 6 * len(ma.groups())
        before = P.launch_count()
        ma.run(P.SHT_MULTI_ROUND_TRIP)
        ma.synchronize()
        assert P.launch_count() - before == n
    finally:
        ma.close()
        mb.close()


def test_multi_split_precision(plans):
    """Split precision for the plans it covers (T21/T42/T85), FP64 for T170."""
    P = pkg()
    insts = _instances(plans, 15, max_nb=64, seed=13)
    for g in ("T21", "T42", "T85"):
        plans[g].set_precision(P.SHT_PREC_SPLIT)
    try:
        m = _build(plans, insts, autotune=False)
    finally:
        for g in ("T21", "T42", "T85"):
            plans[g].set_precision(P.SHT_PREC_FP64)
    try:
        precs = [g["precision"] for g in m.groups()]
        assert len(precs) == 4 and precs.count(P.SHT_PREC_SPLIT) == 3
        m.run(P.SHT_MULTI_SYNTHESIS)
        m.synchronize()
        for x in insts:
            assert relerr(x["xya"].cpu().numpy(), x["plan"].xya_wa(x["w"])) < 1e-11, x["grid"]
        m.run(P.SHT_MULTI_ANALYSIS)
        m.synchronize()
        for x in insts:
            assert relerr(x["wa"].cpu().numpy(), x["w"]) < 1e-11, x["grid"]
    finally:
        m.close()


def test_multi_tuner_may_pick_split(plans):
    P = pkg()
    insts = _instances(plans, 15, max_nb=32, seed=17)
    m = _build(plans, insts, autotune=True, allow_split=True)
    try:
        for g in m.groups():
            assert g["precision"] in (P.SHT_PREC_FP64, P.SHT_PREC_SPLIT, P.SHT_PREC_AUTO)
            assert g["legendre_tile"] in (0, 8, 16, 32)  # the tuner also picks a tile
            assert 0 <= g["sms"] <= 148  # and whether the groups share the SMs side by side
        m.run(P.SHT_MULTI_ROUND_TRIP)
        m.synchronize()
        for x in insts:
            assert relerr(x["wa"].cpu().numpy(), x["w"]) < 1e-11
    finally:
        m.close()


@pytest.mark.parametrize("autotune", [False, True])
def test_multi_side_by_side(plans, autotune):
    """Groups whose persistent kernels are sized for shares of the SMs (run
    side by side) give the same results as the single-plan calls and the
    oracle."""
    P = pkg()
    insts = _instances(plans, 9, max_nb=24, seed=29)
    m = _build(plans, insts, autotune=autotune, side_by_side=True)
    try:
        shares = [g["sms"] for g in m.groups()]
        assert all(s >= 4 for s in shares) and len(shares) > 1, shares
        m.run(P.SHT_MULTI_ROUND_TRIP)
        m.synchronize()
        for x in insts:
            assert relerr(x["wa"].cpu().numpy(), x["w"]) < 1e-11, x["grid"]
            ref = x["plan"].xya_wa(torch.from_numpy(x["w"]).cuda())
            torch.cuda.synchronize()
            assert relerr(x["xya"].cpu().numpy(), ref.cpu().numpy()) < 1e-12, x["grid"]
    finally:
        m.close()


def test_multi_argument_errors(plans):
    P = pkg()
    m = P.MultiTransform()
    try:
        with pytest.raises(P.SpmlError) as ei:
            m.build()
        assert ei.value.status == 1
        with pytest.raises(P.SpmlError) as ei:
            m.run()
        assert ei.value.status == 3
        p = plans["T21"]
        with pytest.raises(ValueError):
            m.add(p, torch.zeros((2, p.lm + 1), dtype=torch.float64, device="cuda"),
                  torch.zeros((2, p.jm, p.im), dtype=torch.float64, device="cuda"))
        with pytest.raises(TypeError):
            m.add(p, np.zeros((2, p.lm)), np.zeros((2, p.jm, p.im)))
    finally:
        m.close()


def test_multi_runs_on_a_torch_stream(plans):
    """Replays ordered on torch's stream: events around run() see the work."""
    P = pkg()
    insts = _instances(plans, 15, max_nb=48, seed=19)
    m = _build(plans, insts, autotune=False)
    try:
        s = torch.cuda.Stream()
        m.set_stream(s)
        with torch.cuda.stream(s):
            for x in insts:
                x["xya"].zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            m.run(P.SHT_MULTI_SYNTHESIS)
            e1.record(s)
        s.synchronize()
        assert e0.elapsed_time(e1) > 0.01  # a T170 synthesis alone takes longer than 10 us
        for x in insts:
            assert relerr(x["xya"].cpu().numpy(), x["plan"].xya_wa(x["w"])) < 1e-12
    finally:
        m.close()
