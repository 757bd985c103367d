"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: these run without a GPU)."""
import glob
import os
import re

from cosenu_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(cosenu_\w+)\s*\(", src, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        from cosenu_b200.build import build
        build()
    lib = _lib.load()
    decl = declared_symbols()
    assert decl, "no declarations found"
    for name in sorted(decl):
        assert hasattr(lib, name), name
    assert decl == set(_lib.EXPORTS) | (decl - set(_lib.EXPORTS))
    assert set(_lib.EXPORTS) <= decl


def test_create_without_gpu_fails_loudly():
    """No CPU fallback: without a device the library returns an error."""
    import ctypes as C
    import torch
    if torch.cuda.is_available():
        return
    lib = _lib.load()
    p = _lib.default_params()
    h = C.c_void_p()
    rc = lib.cosenu_create(C.byref(p), C.byref(h))
    assert rc == _lib.ERR_CUDA
    assert b"device" in lib.cosenu_last_error(None)


def test_params_default_matches_presets():
    p = _lib.default_params()
    assert (p.scheme, p.bc, p.flags) == (_lib.FV, _lib.PERIODIC, _lib.VAC | _lib.COLL)
    assert (p.nz, p.nvz, p.gz, p.cfl) == (2400, 32, 4, 0.4)
