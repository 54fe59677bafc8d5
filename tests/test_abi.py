"""CPU checks of the C ABI: the library builds, loads without a GPU, and exports
every function include/mlegs_b200.h declares (no compute calls here)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(mlegs_[a-z0-9_]+)\s*\(", src, re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("mlegs_create", "mlegs_rtran", "mlegs_horfft", "mlegs_verfft", "mlegs_toff",
                 "mlegs_tofp", "mlegs_boussi_force", "mlegs_solver_init", "mlegs_step"):
        assert must in names


def test_library_exports_every_declared_symbol(lib_built):
    lib = ctypes.CDLL(lib_built)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(lib_built):
    from mlegs_b200 import _lib
    assert set(declared_functions()) <= set(_lib.SIGNATURES), \
        set(declared_functions()) - set(_lib.SIGNATURES)
    _lib.load(lib_built)


def test_create_rejects_bad_params_without_gpu(lib_built):
    """Argument validation happens before any device call."""
    from mlegs_b200 import _lib
    lib = _lib.load(lib_built)
    p = _lib.Params()
    p.nr, p.nth, p.nx = 64, 30, 32          # NTH not a power of two
    p.nrchop, p.ntchop, p.nxchop = 58, 16, 16
    p.ell, p.zlen, p.dt = 1.0, 6.283, 1e-3
    h = ctypes.c_void_p()
    assert lib.mlegs_create(ctypes.byref(p), ctypes.byref(h)) != 0
    assert not h.value
    assert lib.mlegs_destroy(None) != 0
    assert lib.mlegs_last_error(None) == b"null context"


def test_pad_and_space_codes_match_reference():
    """Space tags and ERR_FLAGS values are the reference's (mod_scalar3.f90:82-106)."""
    src = open(os.path.join(ROOT, "include", "mlegs_b200.h")).read()
    tags = dict(re.findall(r"#define (MLEGS_[A-Z0-9_]+)\s+(-?\d+)", src))
    assert (tags["MLEGS_PPP"], tags["MLEGS_FFF"], tags["MLEGS_PFP"], tags["MLEGS_PFF"]) == ("0", "1", "2", "3")
    assert tags["MLEGS_ERR_SCALAR3_ISNAN"] == "10" and tags["MLEGS_ERR_LOGTERM"] == "13"
    assert tags["MLEGS_ERR_TRANSFORM"] == "2" and tags["MLEGS_ERR_SOLVER"] == "5"


@pytest.mark.parametrize("mod", ["mlegs_b200", "mlegs_b200.inputs"])
def test_package_imports_without_oracle(mod):
    """The product package never imports the oracle."""
    import importlib
    import sys
    before = set(k for k in sys.modules if k.startswith("oracle"))
    importlib.import_module(mod)
    after = set(k for k in sys.modules if k.startswith("oracle"))
    assert after == before
    for fn in os.listdir(os.path.join(ROOT, "mlegs_b200")):
        if fn.endswith(".py"):
            assert "import oracle" not in open(os.path.join(ROOT, "mlegs_b200", fn)).read()
            assert "from oracle" not in open(os.path.join(ROOT, "mlegs_b200", fn)).read()
