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


_CTYPES = {"int": ctypes.c_int, "double": ctypes.c_double, "long long": ctypes.c_longlong,
           "size_t": ctypes.c_size_t}


def _header_struct(name):
    """(field, ctype) list of `typedef struct {...} name;` in include/librint_b200.h."""
    text = open(os.path.join(ROOT, "include", "librint_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = re.search(r"typedef struct \{([^}]*)\}\s*" + name + r"\s*;", text).group(1)
    fields = []
    for decl in body.split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        m = re.match(r"(long long|size_t|double|int) (.*)", decl)
        assert m, decl
        for f in m.group(2).split(","):
            fields.append((f.strip(), _CTYPES[m.group(1)]))
    return fields


def test_ctypes_structs_match_header():
    """The Python mirrors of the options / result structs carry the header's
    fields in the header's order and types (lrb_scf reads them by layout)."""
    for cname, py in (("LrbScfOptions", B.ScfOptions), ("LrbScfResult", B.ScfResult)):
        assert [(n, t) for n, t in py._fields_] == _header_struct(cname), cname


def test_ctypes_struct_layout_matches_c_compiler(tmp_path):
    """Offsets and sizes of the structs as gcc lays them out from the header
    equal the ctypes mirrors'."""
    import shutil
    import subprocess
    import pytest
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "librint_b200.h"',
             'int main(void) {']
    for cname, _ in (("LrbScfOptions", 0), ("LrbScfResult", 0)):
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _t in _header_struct(cname):
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in (("LrbScfOptions", B.ScfOptions), ("LrbScfResult", B.ScfResult)):
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _t in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def _batch(L, m, sh, coord=1):
    import numpy as np
    out = np.empty(8)
    atm, bas, env = m.atm, m.bas, m.env
    return L.lrb_int2e_batch(out.ctypes.data_as(B.P_d), coord, sh.ctypes.data_as(B.P_i),
                             sh.shape[0], atm.ctypes.data_as(B.P_i), atm.size // 6,
                             bas.ctypes.data_as(B.P_i), bas.size // 8,
                             env.ctypes.data_as(B.P_d), env.size)


def test_batch_host_checks_before_any_device_work():
    """lrb_int2e_batch checks every shell index and every bas entry on the
    host threads before it touches a device; a bad index or entry anywhere
    in a large batch (several threads' parts) is reported with the same code
    and message as in a small one."""
    import numpy as np
    from librint_b200 import synthetic
    L = B.lib()
    m, sh = synthetic.eri_sweep((1, 0, 1, 0), 300_000, seed=3)
    for pos in (0, 150_001, 299_999):
        bad = sh.copy()
        bad[pos, 2] = m.nbas
        assert _batch(L, m, bad) == -1
        assert b"shell index out of range" in L.lrb_last_error()
        bad[pos, 2] = -1
        assert _batch(L, m, bad) == -1
    for s in (3, m.nbas // 2 + 1, m.nbas - 1):
        bas = m.bas.copy().reshape(-1, 8)
        bas[s, 5] = m.env.size          # exponents beyond env
        mb = type(m)(m.atm, bas.ravel(), m.env)
        assert _batch(L, mb, sh) == -1
        assert b"bas entry out of range" in L.lrb_last_error()
    bad = np.ascontiguousarray(sh[:10])
    assert _batch(L, m, bad, coord=2) == -1
    assert b"coord" in L.lrb_last_error()


def test_batch_len_large_and_bad_indices():
    """lrb_int2e_batch_len (block lengths summed on the host threads) equals
    the sum of the blocks' products of shell dimensions, cartesian and
    spherical, and is -1 for an index out of range anywhere in the list."""
    import numpy as np
    from librint_b200 import synthetic
    L = B.lib()
    m, sh = synthetic.eri_sweep((2, 1, 1, 0), 300_000, seed=4)
    b = m.bas.reshape(-1, 8)
    l = b[sh, 1]
    for coord, dim in ((0, (l + 1) * (l + 2) // 2), (1, 2 * l + 1)):
        want = int(dim.astype(np.int64).prod(axis=1).sum())
        got = L.lrb_int2e_batch_len(coord, sh.ctypes.data_as(B.P_i), sh.shape[0],
                                    m.bas.ctypes.data_as(B.P_i), b.shape[0])
        assert got == want
    bad = sh.copy()
    bad[299_999, 3] = b.shape[0]
    assert L.lrb_int2e_batch_len(1, bad.ctypes.data_as(B.P_i), bad.shape[0],
                                 m.bas.ctypes.data_as(B.P_i), b.shape[0]) == -1
