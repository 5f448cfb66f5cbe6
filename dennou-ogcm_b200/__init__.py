"""B200 spherical-harmonic transform for dogcm (drop-in for SpmlUtil_mod's horizontal part).

The compute lives in libdogcm_sht.so (CUDA, sm_100a) behind the C-ABI of
include/dogcm_sht.h.  spmlutil.SpmlUtil mirrors the Fortran module's interface
for Python hosts and tests.
"""
from .spmlutil import (SHT_MULTI_ANALYSIS, SHT_MULTI_ROUND_TRIP, SHT_MULTI_SYNTHESIS, SHT_OPT_HOST_GRAPH_COUNT,
                       SHT_OPT_HOST_GRAPHS, SHT_OPT_LEGENDRE_KERNEL, SHT_OPT_LEGENDRE_TILE, SHT_PREC_AUTO, SHT_PREC_FP64, SHT_PREC_SPLIT, MultiTransform, SpmlError, SpmlUtil, l_nm, launch_count,
                       load_library, nm_l)

__all__ = ["SpmlUtil", "SpmlError", "MultiTransform", "load_library", "l_nm", "nm_l", "launch_count",
           "SHT_PREC_FP64", "SHT_PREC_SPLIT", "SHT_PREC_AUTO", "SHT_OPT_LEGENDRE_KERNEL", "SHT_OPT_LEGENDRE_TILE", "SHT_OPT_HOST_GRAPHS",
           "SHT_OPT_HOST_GRAPH_COUNT", "SHT_MULTI_SYNTHESIS",
           "SHT_MULTI_ANALYSIS", "SHT_MULTI_ROUND_TRIP"]
