"""ctypes wrapper over the CPU oracle (libsht_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker.  The product path never
imports this module.

Parity status: unpinned against reference outputs (the SPMODEL/ISPACK
libraries that hold the reference arithmetic are not in the reference tree);
see sht_oracle.c for the specification lines it restates.

Arrays follow the Fortran layouts of model/dogcm/src/util/math/SpmlUtil_mod.f90:
grid  xya(0:I-1, 1:J, nb)  -> numpy shape (nb, J, I), C order
spec  wa(lm, nb)            -> numpy shape (nb, lm),   C order
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsht_oracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compile the oracle shared library in place (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "sht_oracle.c")):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    lib.or_init.restype = ctypes.c_void_p
    lib.or_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    lib.or_free.argtypes = [ctypes.c_void_p]
    lib.or_lm.restype = ctypes.c_long
    lib.or_lm.argtypes = [ctypes.c_void_p]
    lib.or_gauss.argtypes = [ctypes.c_int, _D, _D]
    lib.or_grid_info.argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
    lib.or_legendre_row.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D]
    for name in ("or_wa_xya", "or_xya_wa", "or_wa_divlambda_xya", "or_wa_divmu_xya",
                 "or_xya_gradlambda_wa", "or_xya_gradmu_wa", "or_xya_gradlon_wa",
                 "or_xya_gradlat_wa", "or_wa_lapla_wa", "or_wa_laplainv_wa"):
        getattr(lib, name).argtypes = [ctypes.c_void_p, _D, ctypes.c_int, _D]
    for name in ("or_wa_alphaoptr_xya", "or_xya_alphaoptr_wa"):
        getattr(lib, name).argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int, _D]
    for name in ("or_uvcoslat2vordiv", "or_vordiv2uv"):
        getattr(lib, name).argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int, _D, _D]
    lib.or_intlonlat.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, _D, ctypes.c_int]
    lib.or_intlon.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, _D, ctypes.c_int]
    lib.or_diffuse.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, _D, ctypes.c_double, _D]
    lib.or_diffcoef.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, _D, _D]
    lib.or_rn.argtypes = [ctypes.c_void_p, _D]
    lib.or_l_nm.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.or_nm_l.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.or_set_threads.argtypes = [ctypes.c_int]
    lib.or_get_threads.restype = ctypes.c_int
    _lib = lib
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    _load().or_set_threads(int(n))


def get_threads() -> int:
    return int(_load().or_get_threads())


def gauss(J: int):
    """Gauss nodes mu_j (ascending) and weights normalised to sum 1."""
    lib = _load()
    mu = np.zeros(J)
    w = np.zeros(J)
    lib.or_gauss(J, _p(mu), _p(w))
    return mu, w


def l_nm(n: int, m: int) -> int:
    return int(_load().or_l_nm(n, m))


def nm_l(l: int):
    n = ctypes.c_int()
    m = ctypes.c_int()
    _load().or_nm_l(l, ctypes.byref(n), ctypes.byref(m))
    return n.value, m.value


class OraclePlan:
    """FP64 CPU transform for one grid (I lon, J Gauss lat, truncation N, radius a)."""

    def __init__(self, im: int, jm: int, nm: int, radius: float = 1.0):
        lib = _load()
        self.im, self.jm, self.nm, self.radius = im, jm, nm, float(radius)
        self.lm = (nm + 1) ** 2
        self._h = lib.or_init(im, jm, nm, float(radius))
        if not self._h:
            raise ValueError(f"oracle: unsupported grid I={im} J={jm} N={nm}")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.or_free(h)
            self._h = None

    # -- layouts
    def _grid(self, x):
        x = _c(x)
        if x.ndim == 2:
            x = x[None]
        assert x.shape[1:] == (self.jm, self.im), x.shape
        return x

    def _spec(self, w):
        w = _c(w)
        if w.ndim == 1:
            w = w[None]
        assert w.shape[1] == self.lm, w.shape
        return w

    def grid_info(self):
        xl = np.zeros(self.im); yl = np.zeros(self.jm); xw = np.zeros(self.im); yw = np.zeros(self.jm)
        _load().or_grid_info(self._h, _p(xl), _p(yl), _p(xw), _p(yw))
        return xl, yl, xw, yw

    def legendre_row(self, n: int, m: int) -> np.ndarray:
        out = np.zeros(self.jm // 2)
        _load().or_legendre_row(self._h, n, m, _p(out))
        return out

    def _g2s(self, fn, x):
        x = self._grid(x)
        out = np.zeros((x.shape[0], self.lm))
        getattr(_load(), fn)(self._h, _p(x), x.shape[0], _p(out))
        return out

    def _s2g(self, fn, w):
        w = self._spec(w)
        out = np.zeros((w.shape[0], self.jm, self.im))
        getattr(_load(), fn)(self._h, _p(w), w.shape[0], _p(out))
        return out

    def _s2s(self, fn, w):
        w = self._spec(w)
        out = np.zeros_like(w)
        getattr(_load(), fn)(self._h, _p(w), w.shape[0], _p(out))
        return out

    def wa_xya(self, x):
        return self._g2s("or_wa_xya", x)

    def xya_wa(self, w):
        return self._s2g("or_xya_wa", w)

    def wa_divlambda_xya(self, x):
        return self._g2s("or_wa_divlambda_xya", x)

    def wa_divmu_xya(self, x):
        return self._g2s("or_wa_divmu_xya", x)

    def xya_gradlambda_wa(self, w):
        return self._s2g("or_xya_gradlambda_wa", w)

    def xya_gradmu_wa(self, w):
        return self._s2g("or_xya_gradmu_wa", w)

    def xya_gradlon_wa(self, w):
        return self._s2g("or_xya_gradlon_wa", w)

    def xya_gradlat_wa(self, w):
        return self._s2g("or_xya_gradlat_wa", w)

    def wa_lapla_wa(self, w):
        return self._s2s("or_wa_lapla_wa", w)

    def wa_laplainv_wa(self, w):
        return self._s2s("or_wa_laplainv_wa", w)

    def wa_alphaoptr_xya(self, a, b):
        a = self._grid(a); b = self._grid(b)
        out = np.zeros((a.shape[0], self.lm))
        _load().or_wa_alphaoptr_xya(self._h, _p(a), _p(b), a.shape[0], _p(out))
        return out

    def xya_alphaoptr_wa(self, wa, wb):
        wa = self._spec(wa); wb = self._spec(wb)
        out = np.zeros((wa.shape[0], self.jm, self.im))
        _load().or_xya_alphaoptr_wa(self._h, _p(wa), _p(wb), wa.shape[0], _p(out))
        return out

    def uvcoslat2vordiv(self, u, v):
        u = self._grid(u); v = self._grid(v)
        vor = np.zeros((u.shape[0], self.lm)); div = np.zeros_like(vor)
        _load().or_uvcoslat2vordiv(self._h, _p(u), _p(v), u.shape[0], _p(vor), _p(div))
        return vor, div

    def vordiv2uv(self, vor, div):
        vor = self._spec(vor); div = self._spec(div)
        u = np.zeros((vor.shape[0], self.jm, self.im)); v = np.zeros_like(u)
        _load().or_vordiv2uv(self._h, _p(vor), _p(div), vor.shape[0], _p(u), _p(v))
        return u, v

    def avrlonlat(self, x):
        x = self._grid(x)
        out = np.zeros(x.shape[0])
        _load().or_intlonlat(self._h, _p(x), x.shape[0], _p(out), 1)
        return out

    def intlonlat(self, x):
        x = self._grid(x)
        out = np.zeros(x.shape[0])
        _load().or_intlonlat(self._h, _p(x), x.shape[0], _p(out), 0)
        return out

    def ya_avrlon(self, x):
        x = self._grid(x)
        out = np.zeros((x.shape[0], self.jm))
        _load().or_intlon(self._h, _p(x), x.shape[0], _p(out), 1)
        return out

    def ya_intlon(self, x):
        x = self._grid(x)
        out = np.zeros((x.shape[0], self.jm))
        _load().or_intlon(self._h, _p(x), x.shape[0], _p(out), 0)
        return out

    def rn(self):
        out = np.zeros(self.lm)
        _load().or_rn(self._h, _p(out))
        return out

    def diffcoef(self, diff, visc, numdiff, order):
        ct = np.zeros(self.lm); cm = np.zeros(self.lm)
        _load().or_diffcoef(self._h, float(diff), float(visc), float(numdiff), int(order), _p(ct), _p(cm))
        return ct, cm

    def diffuse(self, w, coef, dt, filt=None):
        w = self._spec(w).copy()
        coef = _c(coef)
        f = _c(filt) if filt is not None else None
        _load().or_diffuse(self._h, _p(w), w.shape[0], _p(coef), float(dt), _p(f) if f is not None else None)
        return w
