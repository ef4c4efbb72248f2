"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute: runs without a GPU)."""
import ctypes
import glob
import os
import re

from librint_b200 import _bindings as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        for m in re.finditer(r"^LRB_API\s+[^;(]*?\b([A-Za-z_][A-Za-z_0-9]*)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("int2e_sph", "int2e_cart", "int2e_optimizer", "CINTdel_optimizer", "int2e_c",
                 "free_c", "lrb_int2e_batch", "lrb_int2e_batch_device", "lrb_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(B.SO_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_load():
    L = B.lib()
    assert L.lrb_last_error() is not None
