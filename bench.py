"""Benchmark: T85 L60 round-trip spherical-harmonic transforms per second.

Workload (config C1's grid and batch): T85 (256 lon x 128 Gauss lat), 60 levels
x 8 fields = 480 field-levels, seeded spectra ~ (n+1)^-2 (seed 20261203; no
dataset is involved).  One step = one round trip of the whole batch:
xya_wa (spectral -> grid) then wa_xya (grid -> spectral).  A round-trip
transform is one field-level through both.

  value  device throughput with the spectra resident in HBM: field-level round
         trips per second (CUDA events on the launching stream, L2 flushed with
         a 256 MiB write between steps, outside the timed events).
  e2e    the same metric through the host-pointer C-ABI (sht_xya_wa then
         sht_wa_xya on pinned host arrays): every step moves the spectra in,
         the grid out and back, and the spectra out over PCIe.  Its
         pcie_floor is the time plain pinned copies of the same bytes take
         (each call bound by its larger direction), against the measured time.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                        [--precision auto|fp64|split|per_direction] [--nb NB]
--precision auto times the three modes (FP64, split precision on the tensor
cores, and per_direction: split for the contractions of at least 128 terms,
FP64 for the others) and reports the fastest that meets 1e-11 as the value.
Under torchrun each rank runs the same batch on its own GPU (replicas: the
transform of independent field-levels needs no exchange), the timing is the
max over ranks and value is the total over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "T85L60 round-trip transforms/s: split-prec TC vs FP64 GPU, ≤1e-11 rel err"
UNIT = "round-trip transforms/s"
GRID = "T85"
LEVELS, FIELDS, POWER = 60, 8, 2.0
# the configurations' (levels, fields) per grid, for --grid runs at other
# resolutions (C0 T21 L20 x 3, C1 T85 L60 x 8, C2 T170 L60 x 12, C4 T341 L60 x 16)
GRID_BATCH = {"T21": (20, 3), "T42": (60, 8), "T85": (60, 8), "T170": (60, 12), "T341": (60, 16)}


def _workload(grid):
    lv, fd = GRID_BATCH[grid]
    metric = METRIC if grid == GRID else METRIC.replace("T85L60", f"{grid}L{lv}")
    return lv, fd, metric
RADIUS = 6.371e6


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def _traffic(kernel, mode, nb, grid=GRID):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    capture of this workload (the per-kernel dram__bytes_read.sum +
    dram__bytes_write.sum kept in profiles/t85_dram_traffic.json), FP64 path at
    the 480 field-level batch; None for any other configuration."""
    if mode != "fp64" or nb != LEVELS * FIELDS or grid != GRID:
        return None
    try:
        with open(os.path.join(ROOT, "profiles", "t85_dram_traffic.json")) as f:
            t = json.load(f)
    except Exception:
        return None
    keys = ("k_fft_fwd", "k_fft_inv") if kernel.startswith("k_fft") else ("k_leg_fwd_pair", "k_leg_inv_pair")
    return 1e6 * (t[keys[0]] + t[keys[1]]) / 2


def _rel(a, b):
    a = np.asarray(a).reshape(len(a), -1)
    b = np.asarray(b).reshape(len(b), -1)
    return float((np.abs(a - b).max(1) / np.abs(b).max(1)).max())


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples SM clock, max clock, power and clock-event reasons through NVML
    every millisecond in a background thread while the timed region runs (a
    few milliseconds at the default step count)."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, props):
        self.props = props
        self.samples = []
        self.reasons = set()
        self.err = None
        self._stop = None
        self._thr = None

    def _handle(self, nv):
        p = self.props
        bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        return nv.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception as ex:  # NVML missing: report it, do not guess
            self.err = f"nvml unavailable: {ex}"
            return
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, pw))
                    for name, const in self.REASONS:
                        if r & getattr(nv, const, 0):
                            self.reasons.add(name)
                except Exception as ex:
                    self.err = str(ex)
                self._stop.wait(0.001)

        self._thr = threading.Thread(target=run, daemon=True)
        self._thr.start()

    def stop(self):
        if self._thr is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "reasons": [self.err or "not sampled"]}
        self._stop.set()
        self._thr.join(timeout=2)
        sm = [s for s, _ in self.samples]
        pw = [p for _, p in self.samples]
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
               "samples": len(sm), "power_w_max": max(pw) if pw else None, "reasons": sorted(self.reasons)}
        if self.err:
            out["nvml_error"] = self.err
        return out


# ------------------------------------------------------------- reference
def run_reference(args):
    """The reference's CPU transform (the oracle's restatement of SPMODEL's
    w_xy/xy_w, OpenMP over field-levels as SpmlUtil does), all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W = importlib.import_module("dennou-ogcm_b200.workloads")
    I, J, N = W.GRIDS[args.grid]
    lv, fd, metric = _workload(args.grid)
    nb = args.nb or lv * fd
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    p = O.OraclePlan(I, J, N, RADIUS)
    w = W.seeded_spectra(N, nb, POWER)
    for _ in range(args.warmup):
        p.wa_xya(p.xya_wa(w))
    t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        out = p.wa_xya(p.xya_wa(w))
        t.append(time.perf_counter() - t0)
    tot = sum(t)
    value = nb * args.steps / tot
    rec = {"impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded spectra, seed 20261203)",
           "config": {"workload": f"{args.grid} L{lv} x {fd} fields round trip (xy_w then w_xy)",
                      "field_levels": nb, "im": I, "jm": J, "nm": N},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                            "sample": f"{args.steps} full steps of {nb} field-levels, OpenMP over field-levels"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "roundtrip_relerr": _rel(out, w)}
    print(json.dumps(rec))
    return 0


def _per_field(got, ref, levels):
    """Largest normwise relative error of each field (field f = levels
    [f L, (f+1) L) of the batch), over its levels."""
    got = np.asarray(got).reshape(len(got), -1)
    ref = np.asarray(ref).reshape(len(ref), -1)
    e = np.abs(got - ref).max(1) / np.where(np.abs(ref).max(1) == 0, 1.0, np.abs(ref).max(1))
    return [float(e[f * levels:(f + 1) * levels].max()) for f in range(len(e) // levels)]


def cpu_baseline(w_in, grid=GRID, seconds=10.0, checks=None, levels=LEVELS):
    """The oracle on all host cores, timed on the benchmark's own seeded
    spectra (a bounded sample of the same round trip), and the checker of the
    GPU results: `checks` maps a label to (inputs, GPU synthesis grid, GPU
    analysis of that grid[, grid name, levels]); each is compared with the
    oracle's synthesis of the inputs and the oracle's analysis of the GPU grid,
    field by field."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W = importlib.import_module("dennou-ogcm_b200.workloads")
    I, J, N = W.GRIDS[grid]
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    p = O.OraclePlan(I, J, N, RADIUS)
    nb = len(w_in)
    p.wa_xya(p.xya_wa(w_in))
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        p.wa_xya(p.xya_wa(w_in))
        done += nb
    el = time.perf_counter() - t0
    out = {"value": done / el, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"{done} field-level round trips ({done // nb} batches of {nb}) in {el:.1f} s"}
    if checks:
        rel = {}
        plans = {grid: p}
        for label, item in checks.items():
            w, g_gpu, w_gpu = item[:3]
            gname, lv = (item[3], item[4]) if len(item) > 3 else (grid, levels)
            if gname not in plans:
                plans[gname] = O.OraclePlan(*W.GRIDS[gname], RADIUS)
            q = plans[gname]
            syn = _per_field(g_gpu, q.xya_wa(w), lv)
            ana = _per_field(w_gpu, q.wa_xya(g_gpu), lv)
            rel[label] = {"grid": gname, "field_levels": len(w), "levels_per_field": lv,
                          "synthesis_max": max(syn), "analysis_max": max(ana),
                          "synthesis_per_field": syn, "analysis_per_field": ana}
        out["relerr_vs_oracle"] = rel
    return out


# ------------------------------------------------------------------ ours
def bench_multi(P, W, torch, dev, args, flush, max_over_ranks, world):
    """Config C3: 64 independent instances, truncations T21/T42/T85/T170 in
    ratio 8:4:2:1, levels U[10, 60] x 3-8 fields each, seeded spectra
    ~(n+1)^-1.5.  One step = one round trip of every instance = one replay of
    the batch's CUDA graph (sht_multi_run), timed with CUDA events on the
    launching stream, L2 flushed between steps outside the events."""
    grids = ("T21", "T42", "T85", "T170")
    plans = {g: P.SpmlUtil(*W.GRIDS[g][:2], 1, W.GRIDS[g][2], None, RADIUS) for g in grids}
    arrays = []
    for k, d in enumerate(W.mixed_instances(64)):
        p = plans[d["grid"]]
        nb = d["levels"] * d["fields"]
        w0 = W.seeded_spectra_torch(p.nm, nb, 1.5, dev, seed=W.SEED + k)
        arrays.append((p, torch.empty_like(w0), torch.empty((nb, p.jm, p.im), dtype=torch.float64, device=dev), w0))
    total = sum(a[3].shape[0] for a in arrays)
    stream = torch.cuda.current_stream(dev)
    out = {"workload": "C3: 64 instances T21/T42/T85/T170 (8:4:2:1), levels U[10,60] x fields 3-8",
           "field_levels_per_step": total,
           "instances_per_grid": {g: sum(1 for a in arrays if a[0] is plans[g]) for g in grids}}
    for mode, allow_split in (("fp64", False), ("split_allowed", True)):
        m = P.MultiTransform()
        for p, wa, xya, _ in arrays:
            m.add(p, wa, xya)
        t0 = time.perf_counter()
        m.build(autotune=True, allow_split=allow_split)
        build_s = time.perf_counter() - t0
        for _, wa, _, w0 in arrays:
            wa.copy_(w0)
        m.set_stream(stream)
        for _ in range(args.warmup):
            flush.zero_()
            m.run(P.SHT_MULTI_ROUND_TRIP)
        torch.cuda.synchronize()
        evs = []
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            m.run(P.SHT_MULTI_ROUND_TRIP)
            e1.record(stream)
            evs.append((e0, e1))
        m.synchronize()
        tot = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs))
        err = max(_rel(wa.cpu().numpy(), w0.cpu().numpy()) for _, wa, _, w0 in arrays)
        names = {0: "fp64", 1: "split", 2: "per-direction"}
        out[mode] = {"value": world * total * args.steps / (tot * 1e-3), "unit": UNIT,
                     "ms_per_step": tot / args.steps, "kernels_per_step": m.kernels(P.SHT_MULTI_ROUND_TRIP),
                     "graph_launches_per_step": 1, "build_s": build_s, "relerr": err,
                     "groups": [{"grid": g, "field_levels": x["ncol"], "precision": names[x["precision"]],
                                 "legendre_kernel": {0: "auto", 1: "per-band", 2: "paired persistent",
                                                     3: "latitude-chunked persistent",
                                                     4: "single-kernel small-grid transform"}
                                 [x["legendre_kernel"]], "legendre_tile": x["legendre_tile"], "sms": x["sms"],
                                 "tuned_round_trip_ms": x["tuned_ms"]}
                                for g, x in zip(sorted(grids, key=lambda g: plans[g]._h.value), m.groups())]}
        m.close()
    for p in plans.values():
        p.final()
    return out


def bench_operators(P, torch, dev, sht, args, flush, max_over_ranks, world):
    """The SpmlUtil composites on the headline plan and batch, FP64, each as
    one batched call, in transform-equivalents: the number of single-level
    SPML transforms the reference spends per level (w_AlphaOptr_xy is
    w_DivLambda_xy + w_DivMu_xy, two analyses; calc_UVCosLat2VorDiv two
    AlphaOptr, four analyses; calc_VorDiv2UV four syntheses;
    SpmlUtil_mod.f90:299-473).  CUDA events on the launching stream, L2
    flushed between steps outside the events."""
    nb = args.nb or 480
    g = torch.Generator(device=dev).manual_seed(20261204)
    shape = (nb, sht.jm, sht.im)
    xa, xb = (torch.randn(shape, generator=g, dtype=torch.float64, device=dev) for _ in range(2))
    wa = torch.randn((nb, sht.lm), generator=g, dtype=torch.float64, device=dev)
    wb = torch.randn((nb, sht.lm), generator=g, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sht.set_precision(P.SHT_PREC_FP64)
    ops = {  # name: (call, reference transforms per level)
        "w_xy": (lambda: sht.w_xy(xa), 1),
        "xy_w": (lambda: sht.xy_w(wa), 1),
        "w_DivMu_xy": (lambda: sht.w_DivMu_xy(xa), 1),
        "xy_GradLon_w": (lambda: sht.xy_GradLon_w(wa), 1),
        "xy_GradLat_w": (lambda: sht.xy_GradLat_w(wa), 1),
        "w_AlphaOptr_xy": (lambda: sht.w_AlphaOptr_xy(xa, xb), 2),
        "xy_AlphaOptr_w": (lambda: sht.xy_AlphaOptr_w(wa, wb), 2),
        "calc_UVCosLat2VorDiv": (lambda: sht.calc_UVCosLat2VorDiv(xa, xb), 4),
        "calc_VorDiv2UV": (lambda: sht.calc_VorDiv2UV(wa, wb), 4),
    }
    out = {"workload": f"{nb} field-levels on the headline grid, fp64",
           "unit": "transform-equivalents/s (reference single-level transforms per second)"}
    for name, (fn, count) in ops.items():
        for _ in range(max(args.warmup, 3)):
            flush.zero_()
            fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        ms = max_over_ranks(tot) / args.steps
        out[name] = {"ms": ms, "reference_transforms_per_level": count,
                     "transform_equivalents_per_s": world * nb * count / (ms * 1e-3)}
    return out


def bench_fused(P, torch, dev, sht, args, flush, max_over_ranks):
    """The fused clients against their unfused compositions on the headline
    plan and batch, FP64, CUDA events on the launching stream, L2 flushed
    between steps outside the events:
    - product epilogue: w_AlphaOptrProd_xy(A, B, Q) against A*Q, B*Q (torch)
      followed by w_AlphaOptr_xy (the tracer flux divergence of the thickness
      equation, Q = H cos(phi) T);
    - Redi/GM gradients: xy_HGrad_xy(T) against w_xy then xy_GradLon_w and
      xy_GradLat_w;
    - momentum products: calc_UVCosLat2VorDiv of cos(phi)(U Vor + Za) and
      cos(phi)(V Vor + Zb) formed in the load, against the two grids built by
      torch and then analysed;
    - batched callers: the transform parts of the tracer and momentum
      tendency loops over 60 levels in one call per operator, against the
      same operators called level by level."""
    nb = args.nb or 480
    g = torch.Generator(device=dev).manual_seed(20261203)
    shape = (nb, sht.jm, sht.im)
    A, B, T = (torch.randn(shape, generator=g, dtype=torch.float64, device=dev) for _ in range(3))
    Q = 1.0 + 0.5 * torch.randn(shape, generator=g, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sht.set_precision(P.SHT_PREC_FP64)

    def timeit(fn):
        for _ in range(max(args.warmup, 3)):
            flush.zero_()
            fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return max_over_ranks(tot) / args.steps

    def prod_unfused():
        return sht.w_AlphaOptr_xy(A * Q, B * Q)

    def hgrad_unfused():
        w = sht.w_xy(T)
        return sht.xy_GradLon_w(w), sht.xy_GradLat_w(w)

    Z = torch.randn(shape, generator=g, dtype=torch.float64, device=dev)
    cs = torch.cos(torch.as_tensor(sht.y_Lat, dtype=torch.float64, device=dev))[None, :, None]

    def mom_unfused():
        return sht.calc_UVCosLat2VorDiv(cs * (A * Q + T), cs * (B * Q + Z))

    fused_p, ref_p = sht.w_AlphaOptrProd_xy(A, B, Q), prod_unfused()
    (lon, lat), (rlon, rlat) = sht.xy_HGrad_xy(T), hgrad_unfused()
    (mv, md), (rmv, rmd) = sht.calc_UVCosLat2VorDiv_fma(A, B, Q, T, Z), mom_unfused()
    torch.cuda.synchronize()
    out = {"workload": f"{nb} field-levels on the headline grid, fp64"}
    for name, fused, unfused, err in (
            ("alphaoptr_prod", lambda: sht.w_AlphaOptrProd_xy(A, B, Q), prod_unfused,
             _rel(fused_p.cpu().numpy(), ref_p.cpu().numpy())),
            ("hgrad_xya", lambda: sht.xy_HGrad_xy(T), hgrad_unfused,
             max(_rel(lon.cpu().numpy(), rlon.cpu().numpy()), _rel(lat.cpu().numpy(), rlat.cpu().numpy()))),
            ("momentum_products", lambda: sht.calc_UVCosLat2VorDiv_fma(A, B, Q, T, Z), mom_unfused,
             max(_rel(mv.cpu().numpy(), rmv.cpu().numpy()), _rel(md.cpu().numpy(), rmd.cpu().numpy())))):
        tf, tu = timeit(fused), timeit(unfused)
        out[name] = {"fused_ms": tf, "unfused_ms": tu, "speedup": tu / tf, "relerr_vs_unfused": err}
    # the same analysis without the products: what the product epilogue adds
    out["alphaoptr_prod"]["alphaoptr_without_products_ms"] = timeit(lambda: sht.w_AlphaOptr_xy(A, B))

    # the per-level loops of HBEBaroc_HTRCRHS and HBEBaroc_MOMRHS_VorDivForm
    # (one field, 60 levels) as batched calls against the same calls issued
    # level by level from this host, as the reference's do-k loops do
    C = importlib.import_module("dennou-ogcm_b200.callers")
    K = 60
    lvl = (A[:K], B[:K], T[:K], Q[:K])
    filt = torch.ones(sht.lm, dtype=torch.float64, device=dev)
    hp = torch.zeros_like(A[:K])
    cases = {"htrc_rhs": (C.htrc_rhs, (*lvl, filt, hp)), "momrhs_vordiv": (C.momrhs_vordiv, lvl[:3])}
    calls = {}
    for name, (fn, xs) in cases.items():
        tb = timeit(lambda: fn(sht, *xs))
        tl = timeit(lambda: C.per_level(fn, sht, *xs))
        calls[name] = {"levels": K, "batched_ms": tb, "per_level_ms": tl, "speedup": tl / tb}
    out["batched_callers"] = calls
    return out


def c2_outputs(P, W, torch, dev):
    """Config C2 (T170, 60 levels x 12 fields, spectra ~(n+1)^-1.5) in both
    precisions: one synthesis of the seeded spectra and one analysis of the
    resulting grid each, for the per-field oracle check of the cpu_baseline leg."""
    c = W.CONFIGS["C2"]
    I, J, N = W.GRIDS[c["grid"]]
    nb = c["levels"] * c["fields"]
    sht = P.SpmlUtil(I, J, 1, N, None, RADIUS)
    w = W.seeded_spectra_torch(N, nb, c["power"], dev)
    out = {}
    try:
        for mode, prec in (("fp64", P.SHT_PREC_FP64), ("split", P.SHT_PREC_SPLIT)):
            sht.set_precision(prec)
            g = sht.xya_wa(w)
            back = sht.wa_xya(g)
            torch.cuda.synchronize()
            out[f"C2_{mode}"] = (w.cpu().numpy(), g.cpu().numpy(), back.cpu().numpy(), c["grid"], c["levels"])
    finally:
        sht.final()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "split", "per_direction"])
    ap.add_argument("--nb", type=int, default=0, help="field-levels (default: the grid's configuration, 480 at T85)")
    ap.add_argument("--grid", default=GRID, choices=sorted(GRID_BATCH),
                    help="resolution (default T85, the headline workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-c2", action="store_true", help="skip the C2 (T170 L60 x 12) per-field oracle check")
    ap.add_argument("--no-multi", action="store_true", help="skip the C3 multi-instance measurement")
    ap.add_argument("--no-fused", action="store_true", help="skip the fused-client measurements")
    ap.add_argument("--no-operators", action="store_true", help="skip the per-operator measurements")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    Rp = importlib.import_module("dennou-ogcm_b200.replicas")
    world, rank, local = Rp.world_info()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    rep = Rp.Replicas("nccl", device=dev)

    P = importlib.import_module("dennou-ogcm_b200")
    W = importlib.import_module("dennou-ogcm_b200.workloads")
    I, J, N = W.GRIDS[args.grid]
    lv, fd, metric = _workload(args.grid)
    nb = args.nb or lv * fd
    L = (N + 1) ** 2
    sht = P.SpmlUtil(I, J, lv, N, None, RADIUS)
    lib = P.load_library()
    stream = torch.cuda.current_stream(dev)

    w_in = W.seeded_spectra_torch(N, nb, POWER, dev)
    grid = torch.empty((nb, J, I), dtype=torch.float64, device=dev)
    w_out = torch.empty((nb, L), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    h = sht._h
    VP = ctypes.c_void_p
    lib.sht_set_stream(h, VP(stream.cuda_stream))

    def step():
        st = lib.sht_xya_wa_dev(h, VP(w_in.data_ptr()), nb, VP(grid.data_ptr()))
        st |= lib.sht_wa_xya_dev(h, VP(grid.data_ptr()), nb, VP(w_out.data_ptr()))
        if st:
            raise RuntimeError(lib.sht_last_error().decode())

    barrier = rep.barrier
    max_over_ranks = rep.max

    outputs = {}

    def timed(prec):
        sht.set_precision(prec)
        for _ in range(args.warmup):
            flush.zero_()
            step()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        n0 = P.launch_count()
        clk = ClockSampler(torch.cuda.get_device_properties(dev))
        clk.start()
        evs = []
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        barrier()
        torch.cuda.synchronize()
        clocks = clk.stop()
        launches = P.launch_count() - n0
        ms = [a.elapsed_time(b) for a, b in evs]
        tot = max_over_ranks(sum(ms))
        err = _rel(w_out.cpu().numpy(), w_in.cpu().numpy())
        outputs[prec] = (grid.cpu().numpy(), w_out.cpu().numpy())
        return {"value": world * nb * args.steps / (tot * 1e-3), "ms_per_step": tot / args.steps,
                "launches": launches, "clocks": clocks, "relerr": err, "wall_s": wall}

    # stage breakdown of one round trip for the roofline (separate pass, timing on)
    def stages(prec):
        sht.set_precision(prec)
        sht.set_timing(True)
        acc = {"syn": np.zeros(3), "ana": np.zeros(3)}
        reps = 5
        for _ in range(reps):
            flush.zero_()
            lib.sht_xya_wa_dev(h, VP(w_in.data_ptr()), nb, VP(grid.data_ptr()))
            t = sht.last_timing()
            acc["syn"] += [t["fft_ms"], t["legendre_ms"], t["spectral_ms"]]
            flush.zero_()
            lib.sht_wa_xya_dev(h, VP(grid.data_ptr()), nb, VP(w_out.data_ptr()))
            t = sht.last_timing()
            acc["ana"] += [t["fft_ms"], t["legendre_ms"], t["spectral_ms"]]
        sht.set_timing(False)
        return {k: (v / reps).tolist() for k, v in acc.items()}

    results = {}
    # per_direction: SHT_PREC_AUTO, split precision for the contractions of at
    # least 128 terms and FP64 for the others
    PREC = {"fp64": P.SHT_PREC_FP64, "split": P.SHT_PREC_SPLIT, "per_direction": P.SHT_PREC_AUTO}
    modes = ["fp64", "split"] if args.precision == "auto" else [args.precision]
    # per_direction differs from both only where one direction is long enough
    # for split precision and the other is not (T170 here)
    if args.precision == "auto" and (J // 2 >= 128) != ((N + 3) // 2 >= 128):
        modes.append("per_direction")
    for mode in modes:
        prec = PREC[mode]
        try:
            results[mode] = timed(prec)
            results[mode]["stages_ms"] = stages(prec)
        except (P.SpmlError, RuntimeError) as ex:
            results[mode] = {"error": str(ex)}
    ok = {m: r for m, r in results.items() if "value" in r and r["relerr"] <= 1e-11}
    # headline: the fastest precision mode that meets the 1e-11 bound
    head_mode = max(ok, key=lambda k: ok[k]["value"]) if ok else None
    if head_mode is None:
        raise SystemExit(f"no precision mode met 1e-11: {results}")
    head = results[head_mode]

    # roofline of the dominant kernel (largest share of the round trip)
    peaks, pk_kind = _peaks()
    fp64_dfma, fp64_dmma = ctypes.c_double(), ctypes.c_double()
    probe = ctypes.CDLL(os.path.join(ROOT, "dennou-ogcm_b200", "probe", "libfp64_peak.so"))
    probe.fp64_peak_tflops.argtypes = [ctypes.POINTER(ctypes.c_double)] * 2
    probe.fp64_peak_tflops(ctypes.byref(fp64_dfma), ctypes.byref(fp64_dmma))
    st = head["stages_ms"]
    fft_bytes = (8 * I * J + 16 * (N + 1) * J) * nb           # per launch, per direction
    leg_flops = 2 * J * (N + 1) * (N + 2) * nb                  # per launch, per direction (non-symmetric count)
    leg_exec_flops = J * (N + 1) * (N + 4) * nb                 # executed with the equatorial symmetry (N+2 degrees per band)
    cand = {
        "k_fft (forward+inverse)": (st["syn"][0] + st["ana"][0], "hbm", 2 * fft_bytes, "GB/s"),
        "k_leg (forward+inverse)": (st["syn"][1] + st["ana"][1], "tensor", 2 * leg_flops, "TFLOP/s"),
    }
    name = max(cand, key=lambda k: cand[k][0])
    ms_k, bound, work, unit = cand[name]
    if bound == "hbm":
        achieved = work / (ms_k * 1e-3) / 1e9
        peak = float(peaks.get("hbm_gbs", 6650.0))
        pk_note = f"HBM copy bandwidth ({pk_kind})"
    else:
        achieved = work / (ms_k * 1e-3) / 1e12
        if head_mode != "fp64":
            peak = float(peaks.get("bf16_tflops", 1590.0))
            pk_note = f"dense bf16 ({pk_kind}), the tensor-core peak the split contraction runs on"
        else:
            peak = float(fp64_dmma.value)
            pk_note = "FP64 mma.sync probe measured in this run"
    roofline = {"kernel": name, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                "frac": achieved / peak if peak else None, "traffic": _traffic(name, head_mode, nb, args.grid),
                "traffic_unit": "DRAM bytes per launch (mean of the forward and inverse kernel)",
                "algorithmic_per_launch": work / 2, "peak_source": pk_note,
                "stage_ms_per_step": {"synthesis[fft,legendre,spectral]": st["syn"],
                                      "analysis[fft,legendre,spectral]": st["ana"]},
                "fft_roofline_frac_of_hbm": (2 * fft_bytes / ((st["syn"][0] + st["ana"][0]) * 1e-3) / 1e9)
                / float(peaks.get("hbm_gbs", 6650.0)),
                # the Legendre contraction against the FP64 tensor path: in the
                # non-symmetric FLOP count 2 J (N+1)(N+2), and in the FLOPs the
                # symmetric kernels execute, 2 J (N+1)(N+4)/2 per field-level;
                # the denominator is the mma.sync f64 probe run by this bench
                # (the pool's measured peaks have no FP64 figure)
                "legendre_frac_of_fp64": (2 * leg_flops / ((st["syn"][1] + st["ana"][1]) * 1e-3) / 1e12)
                / max(fp64_dmma.value, 1e-9),
                "legendre_executed_frac_of_fp64": (2 * leg_exec_flops / ((st["syn"][1] + st["ana"][1]) * 1e-3) / 1e12)
                / max(fp64_dmma.value, 1e-9),
                "legendre_fp64_peak_source": "mma.sync.m8n8k4.f64 throughput probe run by this bench (not a pool-measured peak)"}
    # whole step against the fused round-trip floor: a round trip that read
    # and wrote each grid and each spectrum once, 2 (8 I J + 8 (N+1)^2) bytes
    # per field-level, at the measured HBM bandwidth
    floor_b = 2 * (8 * I * J + 8 * (N + 1) ** 2) * nb
    roofline["round_trip_floor"] = {
        "bytes_per_step": floor_b, "achieved_gbs": floor_b / (head["ms_per_step"] * 1e-3) / 1e9,
        "frac_of_hbm": floor_b / (head["ms_per_step"] * 1e-3) / 1e9 / float(peaks.get("hbm_gbs", 6650.0))}

    # e2e through the host-pointer C-ABI
    e2e = None
    if not args.no_e2e:
        import torch as _t
        wh = _t.empty((nb, L), dtype=_t.float64).pin_memory()
        wh.copy_(w_in.cpu())
        gh = _t.empty((nb, J, I), dtype=_t.float64).pin_memory()
        wo = _t.empty((nb, L), dtype=_t.float64).pin_memory()
        sht.set_precision(PREC[head_mode])
        for _ in range(2):
            lib.sht_xya_wa(h, VP(wh.data_ptr()), nb, VP(gh.data_ptr()))
            lib.sht_wa_xya(h, VP(gh.data_ptr()), nb, VP(wo.data_ptr()))
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            s1 = lib.sht_xya_wa(h, VP(wh.data_ptr()), nb, VP(gh.data_ptr()))
            s2 = lib.sht_wa_xya(h, VP(gh.data_ptr()), nb, VP(wo.data_ptr()))
            if s1 or s2:
                raise RuntimeError(lib.sht_last_error().decode())
        el = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": world * nb * args.steps / el, "unit": UNIT,
               "h2d_bytes_per_step": 8 * nb * (L + I * J), "d2h_bytes_per_step": 8 * nb * (I * J + L),
               "path": "sht_xya_wa + sht_wa_xya on pinned host arrays (synchronous C-ABI calls, host clock)",
               "relerr": _rel(wo.numpy(), wh.numpy())}
        # the copy floor: plain pinned copies of the grid batch in each
        # direction (CUDA events); each call is bound by its larger direction
        gd = _t.empty((nb, J, I), dtype=_t.float64, device=dev)
        cs = _t.cuda.Stream()
        bw = {}
        for name, dst, src in (("h2d", gd, gh), ("d2h", gh, gd)):
            with _t.cuda.stream(cs):
                for _ in range(2):
                    dst.copy_(src, non_blocking=True)
                e0, e1 = _t.cuda.Event(enable_timing=True), _t.cuda.Event(enable_timing=True)
                e0.record(cs)
                for _ in range(5):
                    dst.copy_(src, non_blocking=True)
                e1.record(cs)
            cs.synchronize()
            bw[name] = 5 * gd.numel() * 8 / (e0.elapsed_time(e1) * 1e-3) / 1e9
        del gd
        gb, lb = 8 * nb * I * J, 8 * nb * L
        floor_ms = 1e3 * (max(lb / bw["h2d"], gb / bw["d2h"]) + max(gb / bw["h2d"], lb / bw["d2h"])) / 1e9
        e2e["pcie_floor"] = {"copy_gbs": bw, "ms_per_step": floor_ms,
                             "measured_ms_per_step": 1e3 * el / args.steps,
                             "frac": floor_ms / (1e3 * el / args.steps)}

    multi = None if args.no_multi else bench_multi(P, W, torch, dev, args, flush, max_over_ranks, world)
    fused = None if args.no_fused else bench_fused(P, torch, dev, sht, args, flush, max_over_ranks)
    operators = None if args.no_operators else bench_operators(P, torch, dev, sht, args, flush, max_over_ranks, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        checks = {}
        for mode in modes:
            prec = PREC[mode]
            if prec in outputs:
                checks[f"{args.grid}_{mode}"] = (w_in.cpu().numpy(), *outputs[prec])
        if args.grid == GRID and not args.no_c2:
            checks.update(c2_outputs(P, W, torch, dev))
        cpu = cpu_baseline(w_in.cpu().numpy(), args.grid, checks=checks, levels=lv)

    if rank == 0:
        rec = {
            "metric": metric, "value": head["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded spectra (n+1)^-2, seed 20261203)",
            "config": {"workload": f"{args.grid} L{lv} x {fd} fields round trip (xya_wa then wa_xya)",
                       "field_levels_per_gpu": nb, "im": I, "jm": J, "nm": N,
                       "precision": head_mode, "l2": "flushed (256 MiB write) between steps, outside the timed events",
                       "parallelism": f"replicas x{world}"},
            "precision_modes": {m: {k: v for k, v in r.items() if k != "clocks"} for m, r in results.items()},
            "split_vs_fp64": (results["split"]["value"] / results["fp64"]["value"])
            if "value" in results.get("split", {}) and "value" in results.get("fp64", {}) else None,
            "relerr": head["relerr"],
            "relerr_vs_oracle": (cpu or {}).pop("relerr_vs_oracle", None),
            "roofline": roofline,
            "fp64_peak_tflops": {"dfma": fp64_dfma.value, "dmma": fp64_dmma.value},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": head["clocks"],
            "gpu_launches": head["launches"],
            "multi_instance": multi,
            "fused_clients": fused,
            "operators": operators,
        }
        print(json.dumps(rec))
    sht.final()
    rep.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
