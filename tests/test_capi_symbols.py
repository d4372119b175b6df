"""CPU: the C-ABI library loads and exports every function include/*.h declares."""
import ctypes
import glob
import os
import re

from crimsonflowsolver_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\*]+\s+\**\s*(crimson_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared()
    for n in ("crimson_elmgmr", "crimson_genadj", "crimson_memls_solve", "crimson_memls_lhs_create",
              "crimson_memls_ls_create", "crimson_memls_bc_create", "crimson_step"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(N.LIB_PATH)
    missing = [n for n in sorted(declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert declared() <= set(N.SIGNATURES), sorted(declared() - set(N.SIGNATURES))


def test_version_without_gpu():
    assert b"sm_100a" in N.lib().crimson_version()
