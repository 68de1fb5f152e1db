"""The C-ABI library loads without a GPU and exports every function that
include/cress_b200.h declares (no compute calls are made here)."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cress_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(?:int|void|long long|const char\*)\s+\*?\s*(cress_\w+)\s*\(", src)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("cress_create", "cress_destroy", "cress_set_base3d", "cress_small_steps",
              "cress_smalldrv", "cress_put_field", "cress_get_field"):
        assert n in names


def test_library_exports_every_declared_symbol(cress):
    lib = ctypes.CDLL(cress.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", cress.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\bT (cress_\w+)", out))
    assert set(declared_functions()) <= exported


def test_abi_version_and_error_string(cress):
    L = cress.lib()
    assert L.cress_abi_version() >= 1
    assert isinstance(L.cress_last_error(), bytes)


def test_bad_config_rejected_without_gpu(cress):
    # Argument checks run before any CUDA call.
    c = cress.Cfg()
    c.ni, c.nj, c.nk = 4, 4, 4
    h = ctypes.c_void_p()
    assert cress.lib().cress_create(ctypes.byref(c), 0, ctypes.byref(h)) == 1  # CRESS_E_ARG
    c.ni, c.nj, c.nk = 20, 20, 20
    c.impopt, c.dx, c.dy, c.dz = 2, 1.0, 1.0, 1.0   # pivoting Gauss elimination: not built
    assert cress.lib().cress_create(ctypes.byref(c), 0, ctypes.byref(h)) == 2  # unsupported


def test_open_boundary_configs_checked_without_gpu(cress):
    # Lateral boundaries: periodic everywhere, or open radiation x (4, 5, 7)
    # with periodic y; other combinations and open x with the Smagorinsky
    # closure or the explicit small step are rejected before any CUDA call.
    c = cress.Cfg()
    c.ni, c.nj, c.nk = 20, 20, 20
    c.dx, c.dy, c.dz = 1.0, 1.0, 1.0
    c.impopt, c.advopt, c.bbc, c.tbc = 1, 2, 2, 2
    c.sbc = c.nbc = -1
    h = ctypes.c_void_p()
    for wbc, ebc in ((6, 6), (4, 7), (2, 2), (-1, 4)):
        c.wbc, c.ebc = wbc, ebc
        assert cress.lib().cress_create(ctypes.byref(c), 0, ctypes.byref(h)) == 2, (wbc, ebc)
    c.wbc = c.ebc = 7
    c.sbc = c.nbc = 4
    assert cress.lib().cress_create(ctypes.byref(c), 0, ctypes.byref(h)) == 2
    c.sbc = c.nbc = -1
    c.tubopt = 1
    assert cress.lib().cress_create(ctypes.byref(c), 0, ctypes.byref(h)) == 2
    c.tubopt, c.impopt = 0, 0
    assert cress.lib().cress_create(ctypes.byref(c), 0, ctypes.byref(h)) == 2
