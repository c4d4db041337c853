"""The C ABI library: it loads, exports every function include/lct.h declares, and rejects
bad arguments before touching the GPU."""
import ctypes as C
import subprocess

from listctrecons_b200 import capi


def test_library_loads_and_exports_every_declared_symbol():
    lib = capi.load()
    declared = capi.declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    # the binding declares a prototype for each of them
    assert sorted(capi.SIGNATURES) == declared
    out = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = sorted({l.split()[-1] for l in out.splitlines() if " T " in l})
    assert exported == declared  # nothing else leaks out of the library


def test_status_strings():
    lib = capi.load()
    assert lib.lct_status_string(0) == b"ok"
    assert b"range" in lib.lct_status_string(capi.LCT_ERR_RANGE)
    assert lib.lct_version() >= 100


def test_argument_checks_need_no_gpu():
    lib = capi.load()
    g = capi.Geom()
    assert lib.lct_rebin_fan2par(None, None, None, 0, 0, None) == capi.LCT_ERR_ARG
    assert lib.lct_rebin_fan2par(C.byref(g), None, None, 0, 0, None) == capi.LCT_ERR_ARG
    assert lib.lct_filter_rows(0, None, None, 1, 0, None) == capi.LCT_ERR_ARG
    assert lib.lct_filter_rows(16, None, None, 1, 7, None) == capi.LCT_ERR_ARG
    assert lib.lct_backproject_par(None, None, None, None, None, 0, 0, None) == capi.LCT_ERR_ARG
    assert lib.lct_sim_project(None, 1, 1, 1, 1.0, 1.0, 0, 0, 1.0, None, None, 0, 1, 0.0, 0,
                               None, None) == capi.LCT_ERR_ARG
    assert lib.lct_filter_taps(5, 0, 16, 1.0, None) == capi.LCT_ERR_ARG
