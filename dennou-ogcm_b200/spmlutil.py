"""Host-side mirror of dogcm's SpmlUtil_mod (horizontal part) over libdogcm_sht.so.

Names, argument meaning and layouts follow
model/dogcm/src/util/math/SpmlUtil_mod.f90 (public list at :71-135).
Array shapes are the Fortran ones read in C order:

    xy(0:im-1, jm)        -> numpy (jm, im)
    xya(0:im-1, jm, km)   -> numpy (km, jm, im)
    w(lm)                 -> numpy (lm,)
    wa(lm, km)            -> numpy (km, lm)

numpy arrays go through the host-pointer entry points. CUDA torch tensors go
through the *_dev entry points on torch's current stream.  The reference
aborts through MessageNotify('E', ...) on misuse; here a nonzero status
raises SpmlError carrying sht_last_error().  There is no CPU fallback: the
shared library and a CUDA device are required for every transform.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import numpy as _numpy  # SpmlUtil_Init's argument `np` shadows the usual alias

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdogcm_sht.so")

SHT_OK = 0
SHT_PREC_FP64 = 0
SHT_PREC_SPLIT = 1
SHT_PREC_AUTO = 2
SHT_OPT_LEGENDRE_KERNEL = 1
SHT_OPT_HOST_GRAPHS = 2
SHT_OPT_HOST_GRAPH_COUNT = 3
SHT_OPT_LEGENDRE_TILE = 4
SHT_MULTI_SYNTHESIS, SHT_MULTI_ANALYSIS, SHT_MULTI_ROUND_TRIP = 1, 2, 3
SHT_MULTI_AUTOTUNE, SHT_MULTI_ALLOW_SPLIT, SHT_MULTI_NO_GRAPH, SHT_MULTI_SIDE_BY_SIDE = 1, 2, 4, 8

_D = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p
_lib = None

# (name, argtypes) for every entry point of include/dogcm_sht.h
_G2S = ["sht_wa_xya", "sht_xya_wa", "sht_wa_divlambda_xya", "sht_wa_divmu_xya",
        "sht_xya_gradlambda_wa", "sht_xya_gradmu_wa", "sht_xya_gradlon_wa",
        "sht_xya_gradlat_wa", "sht_wa_lapla_wa", "sht_wa_laplainv_wa",
        "sht_avrlonlat_xya", "sht_intlonlat_xya", "sht_ya_avrlon_xya", "sht_ya_intlon_xya"]
_TWO_IN = ["sht_wa_alphaoptr_xya", "sht_xya_alphaoptr_wa", "sht_xya_fluxdiv_xya"]
_TWO_IO = ["sht_uvcoslat2vordiv", "sht_vordiv2uv"]
_ONE_IN_TWO_OUT = ["sht_xya_hgrad_wa", "sht_xya_hgrad_xya"]


class SpmlError(RuntimeError):
    """A nonzero status from libdogcm_sht (the reference's MessageNotify('E'))."""

    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


def load_library(path: str | None = None):
    """Load libdogcm_sht.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with python dennou-ogcm_b200/build.py")
    lib = ctypes.CDLL(path)
    lib.sht_status_string.restype = ctypes.c_char_p
    lib.sht_status_string.argtypes = [ctypes.c_int]
    lib.sht_last_error.restype = ctypes.c_char_p
    lib.sht_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                             ctypes.POINTER(_VP)]
    lib.sht_final.argtypes = [_VP]
    lib.sht_is_initialized.argtypes = [_VP]
    lib.sht_dims.argtypes = [_VP] + [ctypes.POINTER(ctypes.c_int)] * 4
    lib.sht_grid_info.argtypes = [_VP, _D, _D, _D, _D]
    lib.sht_l_nm.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.sht_nm_l.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.sht_rn.argtypes = [_VP, _D]
    lib.sht_set_precision.argtypes = [_VP, ctypes.c_int]
    lib.sht_get_precision.argtypes = [_VP, ctypes.POINTER(ctypes.c_int)]
    lib.sht_set_stream.argtypes = [_VP, _VP]
    lib.sht_set_option.argtypes = [_VP, ctypes.c_int, ctypes.c_int]
    lib.sht_get_option.argtypes = [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.sht_synchronize.argtypes = [_VP]
    lib.sht_selftest_device_timeout.argtypes = [_VP, ctypes.c_int]
    lib.sht_set_timing.argtypes = [_VP, ctypes.c_int]
    lib.sht_last_timing.argtypes = [_VP] + [ctypes.POINTER(ctypes.c_float)] * 3
    lib.sht_launch_count.restype = ctypes.c_longlong
    for name in _G2S:
        for suf in ("", "_dev"):
            getattr(lib, name + suf).argtypes = [_VP, _VP, ctypes.c_int, _VP]
    for name in _TWO_IN:
        for suf in ("", "_dev"):
            getattr(lib, name + suf).argtypes = [_VP, _VP, _VP, ctypes.c_int, _VP]
    for name in _TWO_IO:
        for suf in ("", "_dev"):
            getattr(lib, name + suf).argtypes = [_VP, _VP, _VP, ctypes.c_int, _VP, _VP]
    for name in _ONE_IN_TWO_OUT:
        for suf in ("", "_dev"):
            getattr(lib, name + suf).argtypes = [_VP, _VP, ctypes.c_int, _VP, _VP]
    for suf in ("", "_dev"):
        getattr(lib, "sht_wa_alphaoptr_prod_xya" + suf).argtypes = [_VP, _VP, _VP, _VP, ctypes.c_int, _VP]
        getattr(lib, "sht_uvcoslat2vordiv_fma" + suf).argtypes = [_VP] * 6 + [ctypes.c_int, _VP, _VP]
    for suf in ("", "_dev"):
        getattr(lib, "sht_wa_diffuse" + suf).argtypes = [_VP, _VP, ctypes.c_int, _VP, ctypes.c_double, _VP]
    for suf in ("", "_dev"):
        getattr(lib, "sht_analysis" + suf).argtypes = [_VP, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP,
                                                       ctypes.c_int, ctypes.c_int]
        getattr(lib, "sht_synthesis" + suf).argtypes = [_VP, _VP, ctypes.c_int, ctypes.c_int, _VP, ctypes.c_int,
                                                        ctypes.c_int, ctypes.c_int]
    lib.sht_roundtrip_diffuse_dev.argtypes = [_VP, _VP, ctypes.c_int, _VP, ctypes.c_double, _VP]
    lib.sht_plan_l_nm.argtypes = [_VP, ctypes.c_int, ctypes.c_int]
    lib.sht_plan_nm_l.argtypes = [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.sht_multi_create.argtypes = [ctypes.POINTER(_VP)]
    lib.sht_multi_add.argtypes = [_VP, _VP, ctypes.c_int, _VP, _VP, ctypes.POINTER(ctypes.c_int)]
    lib.sht_multi_build.argtypes = [_VP, ctypes.c_int]
    lib.sht_multi_run.argtypes = [_VP, ctypes.c_int]
    lib.sht_multi_synchronize.argtypes = [_VP]
    lib.sht_multi_set_stream.argtypes = [_VP, _VP]
    lib.sht_multi_groups.argtypes = [_VP, ctypes.POINTER(ctypes.c_int)]
    lib.sht_multi_group_info.argtypes = [_VP, ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 3 + \
        [ctypes.POINTER(ctypes.c_float)]
    lib.sht_multi_group_tile.argtypes = [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.sht_multi_group_sms.argtypes = [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.sht_multi_kernels.argtypes = [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.sht_multi_destroy.argtypes = [_VP]
    _lib = lib
    return lib


def _check(status: int, where: str):
    if status != SHT_OK:
        lib = load_library()
        raise SpmlError(status, where, lib.sht_last_error().decode(errors="replace"))


def l_nm(n: int, m: int) -> int:
    """1-based spectral index of (n, m) (SPMODEL l_nm)."""
    return int(load_library().sht_l_nm(n, m))


def nm_l(l: int):
    """(n, m) of the 1-based spectral index l (SPMODEL nm_l)."""
    n, m = ctypes.c_int(), ctypes.c_int()
    _check(load_library().sht_nm_l(l, ctypes.byref(n), ctypes.byref(m)), "nm_l")
    return n.value, m.value


def launch_count() -> int:
    return int(load_library().sht_launch_count())


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


class SpmlUtil:
    """The module state of SpmlUtil_mod: one grid, truncation and planet radius.

    SpmlUtil(iMax, jMax, kMax, nMax, tMax, RPlanet) mirrors SpmlUtil_Init
    (SpmlUtil_mod.f90:192-241). tMax (vertical Chebyshev) is accepted and ignored.
    """

    def __init__(self, iMax: int, jMax: int, kMax: int = 1, nMax: int = -1, tMax: int | None = None,
                 RPlanet: float = 1.0, np: int | None = None):
        lib = load_library()
        h = _VP()
        _check(lib.sht_init(int(iMax), int(jMax), int(kMax), int(nMax), float(RPlanet), ctypes.byref(h)),
               "SpmlUtil_Init")
        self._h = h
        im, jm, nm, lm = (ctypes.c_int() for _ in range(4))
        _check(lib.sht_dims(h, ctypes.byref(im), ctypes.byref(jm), ctypes.byref(nm), ctypes.byref(lm)), "dims")
        self.im, self.jm, self.km, self.nm, self.lm = im.value, jm.value, int(kMax), nm.value, lm.value
        self.radius = float(RPlanet)
        info = self.get_SpmlGridInfo()
        self.x_Lon, self.y_Lat = info["x_Lon"], info["y_Lat"]
        self.x_Lon_Weight, self.y_Lat_Weight = info["x_Lon_Weight"], info["y_Lat_Weight"]
        self.xy_CosLat = _numpy.cos(info["xy_Lat"])

    # ---------------------------------------------------------------- admin
    def SpmlUtil_Final(self):
        if getattr(self, "_h", None):
            _check(load_library().sht_final(self._h), "SpmlUtil_Final")
            self._h = None

    final = SpmlUtil_Final

    def __del__(self):
        try:
            self.SpmlUtil_Final()
        except Exception:
            pass

    def isInitialzed(self) -> bool:
        return bool(getattr(self, "_h", None)) and bool(load_library().sht_is_initialized(self._h))

    def get_SpmlGridInfo(self):
        im, jm = self.im, self.jm
        xl, yl, xw, yw = np.zeros(im), np.zeros(jm), np.zeros(im), np.zeros(jm)
        _check(load_library().sht_grid_info(self._h, *(a.ctypes.data_as(_D) for a in (xl, yl, xw, yw))),
               "get_SpmlGridInfo")
        return {"x_Lon": xl, "y_Lat": yl, "x_Lon_Weight": xw, "y_Lat_Weight": yw,
                "xy_Lon": np.broadcast_to(xl[None, :], (jm, im)).copy(),
                "xy_Lat": np.broadcast_to(yl[:, None], (jm, im)).copy()}

    @property
    def zonal(self) -> bool:
        """True for an axisymmetric plan (iMax = 1: wa_zonal_module, lm = nm + 1)."""
        return self.im == 1

    def l_nm(self, n: int, m: int) -> int:
        """1-based spectral index of (n, m) in this plan's layout (0 if absent)."""
        return int(load_library().sht_plan_l_nm(self._h, int(n), int(m)))

    def nm_l(self, l: int):
        """(n, m) of the 1-based spectral index l in this plan's layout."""
        n, m = ctypes.c_int(), ctypes.c_int()
        _check(load_library().sht_plan_nm_l(self._h, int(l), ctypes.byref(n), ctypes.byref(m)), "nm_l")
        return n.value, m.value

    @property
    def rn(self):
        out = np.zeros(self.lm)
        _check(load_library().sht_rn(self._h, out.ctypes.data_as(_D)), "rn")
        return out

    def set_precision(self, mode: int):
        _check(load_library().sht_set_precision(self._h, int(mode)), "set_precision")

    def get_precision(self) -> int:
        m = ctypes.c_int()
        _check(load_library().sht_get_precision(self._h, ctypes.byref(m)), "get_precision")
        return m.value

    def set_option(self, option: int, value: int):
        _check(load_library().sht_set_option(self._h, int(option), int(value)), "set_option")

    def get_option(self, option: int) -> int:
        v = ctypes.c_int()
        _check(load_library().sht_get_option(self._h, int(option), ctypes.byref(v)), "get_option")
        return v.value

    def set_timing(self, on: bool):
        _check(load_library().sht_set_timing(self._h, int(bool(on))), "set_timing")

    def last_timing(self):
        a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        _check(load_library().sht_last_timing(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "last_timing")
        return {"fft_ms": a.value, "legendre_ms": b.value, "spectral_ms": c.value}

    def synchronize(self):
        _check(load_library().sht_synchronize(self._h), "synchronize")

    # -------------------------------------------------------------- plumbing
    def _grid_shape(self, x):
        s = tuple(x.shape)
        if s[-2:] != (self.jm, self.im):
            raise SpmlError(1, "shape", f"grid array must end in ({self.jm}, {self.im}), got {s}")
        return (s[0] if len(s) == 3 else 1), len(s) == 3

    def _spec_shape(self, w):
        s = tuple(w.shape)
        if s[-1] != self.lm:
            raise SpmlError(1, "shape", f"spectral array must end in {self.lm}, got {s}")
        return (s[0] if len(s) == 2 else 1), len(s) == 2

    def _set_torch_stream(self, x):
        import torch
        s = torch.cuda.current_stream(x.device)
        _check(load_library().sht_set_stream(self._h, _VP(s.cuda_stream)), "set_stream")

    def _run(self, name, ins, out_kind, nout=1):
        """ins: list of inputs (same kind); out_kind: 'grid' | 'spec' | 'avr' | 'ya'."""
        lib = load_library()
        x0 = ins[0]
        nb, batched = (self._grid_shape(x0) if x0.shape[-1] == self.im and x0.ndim >= 2 and x0.shape[-2] == self.jm
                       else self._spec_shape(x0))
        for x in ins[1:]:  # None: an optional input left out (a null pointer)
            if x is not None and tuple(x.shape) != tuple(x0.shape):
                raise SpmlError(1, name, "input shapes differ")
        if out_kind == "grid":
            oshape = (nb, self.jm, self.im)
        elif out_kind == "spec":
            oshape = (nb, self.lm)
        elif out_kind == "avr":
            oshape = (nb,)
        else:
            oshape = (nb, self.jm)
        if _is_torch_cuda(x0):
            import torch
            ins = [None if x is None else x.contiguous() for x in ins]
            if any(x is not None and x.dtype != torch.float64 for x in ins):
                raise SpmlError(1, name, "device arrays must be float64")
            outs = [torch.empty(oshape, dtype=torch.float64, device=x0.device) for _ in range(nout)]
            self._set_torch_stream(x0)
            st = getattr(lib, name + "_dev")(self._h, *(_VP(None if x is None else x.data_ptr()) for x in ins), nb,
                                             *(_VP(o.data_ptr()) for o in outs))
        else:
            ins = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in ins]
            outs = [np.empty(oshape) for _ in range(nout)]
            st = getattr(lib, name)(self._h, *(_VP(None if x is None else x.ctypes.data) for x in ins), nb,
                                    *(_VP(o.ctypes.data) for o in outs))
        _check(st, name)
        if not batched:
            outs = [o[0] if out_kind != "avr" else o[0] for o in outs]
        return outs[0] if nout == 1 else tuple(outs)

    # ------------------------------------------------- transforms (a2 - a12)
    def w_xy(self, xy):
        """Grid -> spectral (SPMODEL w_xy)."""
        return self._run("sht_wa_xya", [xy], "spec")

    def xy_w(self, w):
        """Spectral -> grid (SPMODEL xy_w)."""
        return self._run("sht_xya_wa", [w], "grid")

    wa_xya = w_xy
    xya_wa = xy_w
    wz_xyz = w_xy
    xyz_wz = xy_w

    def w_DivLambda_xy(self, xy):
        """Spectral of (1/(1-mu^2)) d/dlambda."""
        return self._run("sht_wa_divlambda_xya", [xy], "spec")

    def w_DivMu_xy(self, xy):
        """Spectral of d/dmu."""
        return self._run("sht_wa_divmu_xya", [xy], "spec")

    wa_DivLambda_xya = w_DivLambda_xy
    wa_DivMu_xya = w_DivMu_xy

    def xy_GradLambda_w(self, w):
        return self._run("sht_xya_gradlambda_wa", [w], "grid")

    def xy_GradMu_w(self, w):
        return self._run("sht_xya_gradmu_wa", [w], "grid")

    def xy_GradLon_w(self, w):
        return self._run("sht_xya_gradlon_wa", [w], "grid")

    def xy_GradLat_w(self, w):
        return self._run("sht_xya_gradlat_wa", [w], "grid")

    xya_GradLambda_wa = xy_GradLambda_w
    xya_GradMu_wa = xy_GradMu_w
    xya_GradLon_wa = xy_GradLon_w
    xya_GradLat_wa = xy_GradLat_w

    def w_AlphaOptr_xy(self, xy_A, xy_B):
        """(w_DivLambda_xy(A) + w_DivMu_xy(B)) / a (SpmlUtil_mod.f90:398-412)."""
        return self._run("sht_wa_alphaoptr_xya", [xy_A, xy_B], "spec")

    def xy_AlphaOptr_w(self, w_A, w_B):
        """(xy_GradLambda_w(A) + xy_GradMu_w(B)) / (a cos^2 phi) (SpmlUtil_mod.f90:414-428)."""
        return self._run("sht_xya_alphaoptr_wa", [w_A, w_B], "grid")

    wa_AlphaOptr_xya = w_AlphaOptr_xy
    xya_AlphaOptr_wa = xy_AlphaOptr_w

    def w_AlphaOptrProd_xy(self, xy_A, xy_B, xy_Q):
        """w_AlphaOptr_xy(A Q, B Q), the products formed inside the longitude
        transform (HBEBaroc_hspm_vfvm_mod.f90:160-165, Q = H cos(phi) T)."""
        return self._run("sht_wa_alphaoptr_prod_xya", [xy_A, xy_B, xy_Q], "spec")

    def xy_HGrad_w(self, w):
        """-> (xy_GradLon_w(w), xy_GradLat_w(w)) in one synthesis."""
        return self._run("sht_xya_hgrad_wa", [w], "grid", nout=2)

    def xy_HGrad_xy(self, xy):
        """-> (xy_GradLon_w(w_xy(T)), xy_GradLat_w(w_xy(T))), the Redi/GM tracer
        gradients before the 1/radius factor (LPhys_RediGM_hspm_vfvm_mod.f90:432-440)."""
        return self._run("sht_xya_hgrad_xya", [xy], "grid", nout=2)

    def xy_FluxDiv_xy(self, xy_A, xy_B):
        """xy_w(w_AlphaOptr_xy(A, B)), grid to grid (LPhys_RediGM_hspm_vfvm_mod.f90:350-355)."""
        return self._run("sht_xya_fluxdiv_xya", [xy_A, xy_B], "grid")

    wa_AlphaOptrProd_xya = w_AlphaOptrProd_xy
    xya_FluxDiv_xya = xy_FluxDiv_xy
    xya_HGrad_wa = xy_HGrad_w
    xya_HGrad_xya = xy_HGrad_xy

    def calc_UVCosLat2VorDiv(self, xy_UCosLat, xy_VCosLat):
        """-> (w_Vor, w_Div) (SpmlUtil_mod.f90:299-314, 342-368)."""
        return self._run("sht_uvcoslat2vordiv", [xy_UCosLat, xy_VCosLat], "spec", nout=2)

    def calc_UVCosLat2VorDiv_fma(self, xy_X1, xy_X2, xy_Q, xy_Z1=None, xy_Z2=None):
        """calc_UVCosLat2VorDiv(cos(phi) (X1 Q + Z1), cos(phi) (X2 Q + Z2))
        -> (w_Vor, w_Div), the momentum products formed inside the longitude
        transform (HBEBaroc_hspm_vfvm_mod.f90:394-418: Q the vorticity, X1, X2
        the velocities, Z1, Z2 the other terms; both Z or neither)."""
        if (xy_Z1 is None) != (xy_Z2 is None):
            raise SpmlError(1, "sht_uvcoslat2vordiv_fma", "Z1 and Z2 must be both given or both None")
        return self._run("sht_uvcoslat2vordiv_fma", [xy_X1, xy_X2, xy_Q, xy_Z1, xy_Z2], "spec", nout=2)

    def calc_VorDiv2UV(self, w_Vor, w_Div):
        """-> (xy_U, xy_V) (SpmlUtil_mod.f90:316-340, 370-396)."""
        return self._run("sht_vordiv2uv", [w_Vor, w_Div], "grid", nout=2)

    def w_Lapla_w(self, w):
        return self._run("sht_wa_lapla_wa", [w], "spec")

    def w_LaplaInv_w(self, w):
        return self._run("sht_wa_laplainv_wa", [w], "spec")

    wa_Lapla_wa = w_Lapla_w
    wa_LaplaInv_wa = w_LaplaInv_w

    def AvrLonLat_xy(self, xy):
        return self._run("sht_avrlonlat_xya", [xy], "avr")

    def IntLonLat_xy(self, xy):
        return self._run("sht_intlonlat_xya", [xy], "avr")

    def ya_AvrLon_xya(self, xya):
        return self._run("sht_ya_avrlon_xya", [xya], "ya")

    def ya_IntLon_xya(self, xya):
        return self._run("sht_ya_intlon_xya", [xya], "ya")

    def diffuse(self, wa, coef, dt: float, filt=None):
        """Backward-Euler lateral diffusion wa <- filt wa / (1 - dt coef), returns a new array
        (DOGCM_Phys_hspm_vfvm_mod.f90:638-641, 741-742)."""
        lib = load_library()
        nb, batched = self._spec_shape(wa)
        if _is_torch_cuda(wa):
            out = wa.contiguous().clone()
            self._set_torch_stream(out)
            st = lib.sht_wa_diffuse_dev(self._h, _VP(out.data_ptr()), nb, _VP(coef.data_ptr()), float(dt),
                                        _VP(filt.data_ptr()) if filt is not None else None)
        else:
            out = np.array(wa, dtype=np.float64, copy=True, order="C")
            c = np.ascontiguousarray(coef, dtype=np.float64)
            f = np.ascontiguousarray(filt, dtype=np.float64) if filt is not None else None
            st = lib.sht_wa_diffuse(self._h, _VP(out.ctypes.data), nb, _VP(c.ctypes.data), float(dt),
                                    _VP(f.ctypes.data) if f is not None else None)
        _check(st, "diffuse")
        return out

    # ------------------------------------ haloed arrays (leading dimensions)
    def _section(self, x, i0, j0, name):
        """(pointer to point (i0, j0) of level 0, ldi, ldj, nb, device?) of a
        C-contiguous (nb, JA, IA) or (JA, IA) array holding an im x jm section."""
        if x.ndim not in (2, 3):
            raise SpmlError(1, name, "grid array must be (JA, IA) or (nb, JA, IA)")
        ja, ia = int(x.shape[-2]), int(x.shape[-1])
        nb = int(x.shape[0]) if x.ndim == 3 else 1
        if i0 < 0 or j0 < 0 or i0 + self.im > ia or j0 + self.jm > ja:
            raise SpmlError(1, name, f"section ({i0}, {j0}) + ({self.im}, {self.jm}) exceeds ({ia}, {ja})")
        off = 8 * (j0 * ia + i0)
        if _is_torch_cuda(x):
            import torch
            if x.dtype != torch.float64 or not x.is_contiguous():
                raise SpmlError(1, name, "device grid array must be a contiguous float64 tensor")
            return x.data_ptr() + off, ia, ja, nb, True
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise SpmlError(1, name, "grid array must be a C-contiguous float64 array")
        return x.ctypes.data + off, ia, ja, nb, False

    def _spec_rows(self, w, nb, dev, name):
        """(pointer, ldw) of a C-contiguous (nb, LW) spectral array, LW >= lm."""
        if w.ndim != 2 or int(w.shape[0]) != nb or int(w.shape[1]) < self.lm:
            raise SpmlError(1, name, f"spectral array must be ({nb}, >= {self.lm}), got {tuple(w.shape)}")
        if dev != _is_torch_cuda(w):
            raise SpmlError(1, name, "grid and spectral arrays must both be host or both be device arrays")
        if dev:
            import torch
            if w.dtype != torch.float64 or not w.is_contiguous():
                raise SpmlError(1, name, "device spectral array must be a contiguous float64 tensor")
            return w.data_ptr(), int(w.shape[1])
        if w.dtype != np.float64 or not w.flags.c_contiguous:
            raise SpmlError(1, name, "spectral array must be a C-contiguous float64 array")
        return w.ctypes.data, int(w.shape[1])

    def analysis(self, xya, i0: int = 0, j0: int = 0, out=None, mode: int = -1):
        """w_xy of the im x jm section at (i0, j0) of each level of a haloed
        array (nb, JA, IA), e.g. i0 = j0 = 1 for the model's one-point halos;
        out: (nb, LW >= lm) array for the spectra (allocated if None); mode:
        precision for this call (-1: the plan's)."""
        lib = load_library()
        ptr, ldi, ldj, nb, dev = self._section(xya, i0, j0, "analysis")
        if out is None:
            if dev:
                import torch
                out = torch.empty((nb, self.lm), dtype=torch.float64, device=xya.device)
            else:
                out = np.empty((nb, self.lm))
        wp, ldw = self._spec_rows(out, nb, dev, "analysis")
        if dev:
            self._set_torch_stream(xya)
            st = lib.sht_analysis_dev(self._h, _VP(ptr), ldi, ldj, nb, _VP(wp), ldw, mode)
        else:
            st = lib.sht_analysis(self._h, _VP(ptr), ldi, ldj, nb, _VP(wp), ldw, mode)
        _check(st, "analysis")
        return out

    def synthesis(self, wa, out, i0: int = 0, j0: int = 0, mode: int = -1):
        """xy_w into the im x jm section at (i0, j0) of each level of the haloed
        array out (nb, JA, IA); its other points are left as they are.  wa:
        (nb, LW >= lm)."""
        lib = load_library()
        ptr, ldi, ldj, nb, dev = self._section(out, i0, j0, "synthesis")
        wp, ldw = self._spec_rows(wa, nb, dev, "synthesis")
        if dev:
            self._set_torch_stream(out)
            st = lib.sht_synthesis_dev(self._h, _VP(wp), ldw, nb, _VP(ptr), ldi, ldj, mode)
        else:
            st = lib.sht_synthesis(self._h, _VP(wp), ldw, nb, _VP(ptr), ldi, ldj, mode)
        _check(st, "synthesis")
        return out

    def roundtrip_diffuse_(self, xya, coef=None, dt: float = 0.0, filt=None):
        """In place on a CUDA tensor: xya <- xy_w(filt w_xy(xya) / (1 - dt coef))
        (DOGCM_Phys_hspm_vfvm_mod.f90:638-641)."""
        lib = load_library()
        nb, _ = self._grid_shape(xya)
        if not _is_torch_cuda(xya) or not xya.is_contiguous():
            raise SpmlError(1, "roundtrip_diffuse_", "needs a contiguous CUDA float64 tensor")
        self._set_torch_stream(xya)
        _check(lib.sht_roundtrip_diffuse_dev(self._h, _VP(xya.data_ptr()), nb,
                                             _VP(coef.data_ptr()) if coef is not None else None, float(dt),
                                             _VP(filt.data_ptr()) if filt is not None else None),
               "roundtrip_diffuse_")
        return xya


class MultiTransform:
    """Many independent transform instances run as one step (sht_multi_* C-ABI).

    Each instance is (plan, wa, xya): a SpmlUtil plan and CUDA torch tensors
    wa (nb, lm) and xya (nb, jm, im), FP64, contiguous.  build() groups the
    instances per plan, optionally tunes the Legendre variant of every plan and
    captures each step kind as a CUDA graph; run() replays one step on the
    batch's own stream.  build() runs steps on the registered arrays, so fill
    them afterwards.  The reference keeps a single grid per process; this is
    the batched step API of the transform path.
    """

    def __init__(self):
        self._lib = load_library()
        h = _VP()
        _check(self._lib.sht_multi_create(ctypes.byref(h)), "sht_multi_create")
        self._h = h
        self._keep = []  # the registered tensors must stay alive and in place

    def add(self, plan: "SpmlUtil", wa, xya) -> int:
        if not (_is_torch_cuda(wa) and _is_torch_cuda(xya)):
            raise TypeError("MultiTransform instances take CUDA torch tensors")
        import torch
        if wa.dtype != torch.float64 or xya.dtype != torch.float64 or not (wa.is_contiguous() and xya.is_contiguous()):
            raise TypeError("wa and xya must be contiguous float64 tensors")
        nb = wa.shape[0]
        if tuple(wa.shape) != (nb, plan.lm) or tuple(xya.shape) != (nb, plan.jm, plan.im):
            raise ValueError("wa must be (nb, lm) and xya (nb, jm, im) for the plan")
        idx = ctypes.c_int()
        _check(self._lib.sht_multi_add(self._h, plan._h, int(nb), wa.data_ptr(), xya.data_ptr(), ctypes.byref(idx)),
               "sht_multi_add")
        self._keep.append((plan, wa, xya))
        return idx.value

    def build(self, autotune: bool = True, allow_split: bool = False, graph: bool = True,
              side_by_side: bool = False):
        flags = (SHT_MULTI_AUTOTUNE if autotune else 0) | (SHT_MULTI_ALLOW_SPLIT if allow_split else 0) | \
            (0 if graph else SHT_MULTI_NO_GRAPH) | (SHT_MULTI_SIDE_BY_SIDE if side_by_side else 0)
        _check(self._lib.sht_multi_build(self._h, flags), "sht_multi_build")

    def run(self, what: int = SHT_MULTI_ROUND_TRIP):
        _check(self._lib.sht_multi_run(self._h, int(what)), "sht_multi_run")

    def synchronize(self):
        _check(self._lib.sht_multi_synchronize(self._h), "sht_multi_synchronize")

    def set_stream(self, stream):
        """Order runs on a torch CUDA stream (its handle; the default stream is 0)."""
        _check(self._lib.sht_multi_set_stream(self._h, stream.cuda_stream), "sht_multi_set_stream")

    def groups(self):
        """Per plan group: dict(ncol, precision, legendre_kernel, legendre_tile, sms, tuned_ms)."""
        n = ctypes.c_int()
        _check(self._lib.sht_multi_groups(self._h, ctypes.byref(n)), "sht_multi_groups")
        out = []
        for g in range(n.value):
            nc, pr, lk, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
            _check(self._lib.sht_multi_group_info(self._h, g, ctypes.byref(nc), ctypes.byref(pr), ctypes.byref(lk),
                                                  ctypes.byref(ms)), "sht_multi_group_info")
            tile, sms = ctypes.c_int(), ctypes.c_int()
            _check(self._lib.sht_multi_group_tile(self._h, g, ctypes.byref(tile)), "sht_multi_group_tile")
            _check(self._lib.sht_multi_group_sms(self._h, g, ctypes.byref(sms)), "sht_multi_group_sms")
            out.append(dict(ncol=nc.value, precision=pr.value, legendre_kernel=lk.value, legendre_tile=tile.value,
                            sms=sms.value, tuned_ms=ms.value))
        return out

    def kernels(self, what: int = SHT_MULTI_ROUND_TRIP) -> int:
        n = ctypes.c_int()
        _check(self._lib.sht_multi_kernels(self._h, int(what), ctypes.byref(n)), "sht_multi_kernels")
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            _check(self._lib.sht_multi_destroy(self._h), "sht_multi_destroy")
            self._h = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
