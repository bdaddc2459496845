"""The C-ABI library loads without a GPU and exports every symbol include/wavetoy_b200.h declares."""
import ctypes
import os
import re

import conftest

HEADER = os.path.join(conftest.ROOT, "include", "wavetoy_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wt_[A-Za-z0-9_]+)\s*\(", src)))


def test_header_declares_the_drop_in_surface():
    names = declared_symbols()
    for must in ("wt_ctx_create", "wt_mesh_create", "wt_background_set", "wt_workspace_create", "wt_rhs_curved",
                 "wt_rhs_sipg", "wt_rhs_strong", "wt_apply_D", "wt_step_rk4_curved", "wt_energy"):
        assert must in names


def test_library_exports_every_declared_symbol(wt):
    wt.build.build()
    lib = ctypes.CDLL(wt.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_bounds_check_library_exports_every_symbol_and_says_so(wt):
    """The debug variant (build.py --bounds-check) has the same ABI; wt_build_flags (host only)
    tells the two builds apart."""
    wt.build.build(bounds_check=True)
    for path, want in ((wt.LIB_PATH, wt.BUILD_NVTX), (wt.build.LIB_BC, wt.BUILD_NVTX | wt.BUILD_BOUNDS_CHECK)):
        lib = ctypes.CDLL(path)
        missing = [n for n in declared_symbols() if not hasattr(lib, n)]
        assert not missing, (path, missing)
        flags = ctypes.c_int()
        assert lib.wt_build_flags(ctypes.byref(flags)) == 0 and flags.value == want, path


def test_python_mirror_binds_every_symbol(wt):
    lib = wt.library()
    for n in declared_symbols():
        assert getattr(lib, n) is not None


def test_library_operators_equal_oracle_bitwise(wt, O):
    """The shipped GLL operators and the oracle's are computed independently in
    extended precision and rounded once, so they agree bit for bit."""
    import numpy as np
    for N in range(2, 9):
        x, H, G = wt.gll_operators(N)
        xo, Ho, Go = O.gll_ops(N)
        assert np.array_equal(x, xo) and np.array_equal(H, Ho) and np.array_equal(G, Go), N
