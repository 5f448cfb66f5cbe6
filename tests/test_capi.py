"""C-ABI library: it loads, exports every symbol include/dogcm_sht.h declares, and
its host-side logic (argument checks, index maps, status text) behaves without
a GPU.  No compute call runs here."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, pkg

HEADER = os.path.join(ROOT, "include", "dogcm_sht.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^SHT_API [^;]*?\b(sht_[a-z0-9_]+)\s*\(", txt, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 50
    for s in ("sht_init", "sht_final", "sht_wa_xya", "sht_xya_wa", "sht_vordiv2uv", "sht_uvcoslat2vordiv"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = pkg().load_library()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_header_is_plain_c(tmp_path):
    """include/dogcm_sht.h is usable from C99 and C++ hosts (the Fortran shim
    binds the same declarations through ISO_C_BINDING)."""
    import shutil
    import subprocess

    src = tmp_path / "use_header.c"
    src.write_text('#include "dogcm_sht.h"\n'
                   "int main(void) { sht_plan *p = 0; return sht_wa_xya(p, 0, 0, 0) + SHT_OK; }\n")
    inc = os.path.dirname(HEADER)
    for cc, std in (("gcc", ["-std=c99", "-pedantic"]), ("g++", ["-std=c++11", "-x", "c++"])):
        if shutil.which(cc) is None:
            pytest.skip(f"{cc} not available")
        r = subprocess.run([cc, *std, "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I", inc, str(src)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_fortran_shim_binds_declared_symbols():
    """Every bind(C) interface of the Fortran front end names a declared entry
    point, with as many arguments as the C declaration (no Fortran compiler
    here, so this is the shim's link check)."""
    shim = open(os.path.join(ROOT, "dennou-ogcm_b200", "fortran", "wa_module_b200.f90")).read()
    binds = re.findall(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name='(\w+)'\)", shim)
    assert len(binds) >= 30
    hdr = open(HEADER).read()
    syms = set(declared_symbols())
    for fname, args, cname in binds:
        assert fname == cname and cname in syms, cname
        decl = re.search(r"^SHT_API [^;]*?\b" + cname + r"\s*\(([^)]*)\)", hdr, flags=re.M).group(1)
        n_c = 0 if decl.strip() in ("", "void") else decl.count(",") + 1
        n_f = 0 if not args.strip() else args.count(",") + 1
        assert n_c == n_f, (cname, n_c, n_f)


def test_index_maps_and_status_text():
    p = pkg()
    assert p.l_nm(0, 0) == 1
    for l in range(1, 2000):
        n, m = p.nm_l(l)
        assert p.l_nm(n, m) == l
    lib = p.load_library()
    assert lib.sht_status_string(0) == b"ok"
    assert lib.sht_status_string(2) == b"unsupported grid size"


@pytest.mark.parametrize("args", [(63, 32, 1, 21), (64, 31, 1, 21), (64, 32, 1, 40), (4096, 512, 1, 100),
                                  (64, 16, 1, 21), (2, 64, 1, 0), (1, 63, 1, 21), (1, 64, 1, 64)])
def test_init_rejects_unsupported_grids(args):
    """Sizes are validated on the host before any device work (status 2)."""
    lib = pkg().load_library()
    h = ctypes.c_void_p()
    st = lib.sht_init(*args, ctypes.c_double(1.0), ctypes.byref(h))
    assert st == 2
    assert not h.value


def test_calls_on_null_plan_fail_cleanly():
    lib = pkg().load_library()
    buf = (ctypes.c_double * 8)()
    assert lib.sht_wa_xya(None, buf, 1, buf) == 3
    assert lib.sht_final(None) == 3
    assert lib.sht_is_initialized(None) == 0
    assert b"not initialised" in lib.sht_last_error()


def test_fused_clients_check_arguments_on_the_host():
    """The product-epilogue and gradient entry points reject a null plan and
    null arrays before any device work."""
    lib = pkg().load_library()
    buf = (ctypes.c_double * 8)()
    assert lib.sht_wa_alphaoptr_prod_xya(None, buf, buf, buf, 1, buf) == 3
    assert lib.sht_wa_alphaoptr_prod_xya_dev(None, buf, buf, buf, 1, buf) == 3
    assert lib.sht_xya_hgrad_wa(None, buf, 1, buf, buf) == 3
    assert lib.sht_xya_hgrad_xya_dev(None, buf, 1, buf, buf) == 3
    assert lib.sht_xya_fluxdiv_xya(None, buf, buf, 1, buf) == 3


def test_strided_calls_check_arguments_on_the_host():
    """The leading-dimension entry points reject a null plan (whatever the
    other arguments) before any device work."""
    lib = pkg().load_library()
    buf = (ctypes.c_double * 8)()
    ptr = ctypes.cast(buf, ctypes.c_void_p)
    assert lib.sht_analysis(None, ptr, 66, 34, 1, ptr, 500, -1) == 3
    assert lib.sht_analysis_dev(None, ptr, 66, 34, 1, ptr, 500, 1) == 3
    assert lib.sht_synthesis(None, ptr, 500, 1, ptr, 66, 34, 0) == 3
    assert lib.sht_synthesis_dev(None, ptr, 500, 0, ptr, 66, 34, -1) == 3
    assert lib.sht_selftest_device_timeout(None, 10) == 3


def test_init_without_device_reports_no_device(cuda_available):
    if cuda_available:
        pytest.skip("a CUDA device is present")
    lib = pkg().load_library()
    h = ctypes.c_void_p()
    st = lib.sht_init(64, 32, 1, 21, ctypes.c_double(1.0), ctypes.byref(h))
    assert st == 5


def test_multi_without_device_reports_no_device(cuda_available):
    if cuda_available:
        pytest.skip("a CUDA device is present")
    lib = pkg().load_library()
    h = ctypes.c_void_p()
    assert lib.sht_multi_create(ctypes.byref(h)) == 5
    assert not h.value


def test_multi_calls_on_null_batch_fail_cleanly():
    lib = pkg().load_library()
    n = ctypes.c_int()
    assert lib.sht_multi_create(None) == 1
    assert lib.sht_multi_build(None, 0) == 1
    assert lib.sht_multi_run(None, 3) == 1
    assert lib.sht_multi_groups(None, ctypes.byref(n)) == 1
    assert lib.sht_multi_destroy(None) == 1
