"""The C ABI library loads without a GPU and exports every declared entry point."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(hj_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_declared_symbols():
    import hegjoin_b200
    lib = ctypes.CDLL(hegjoin_b200.LIB_PATH)
    declared = _declared()
    assert "hj_join" in declared and "hj_index_create" in declared
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_without_gpu():
    import hegjoin_b200
    assert b"sm_100a" in hegjoin_b200.lib.hj_version()
    # argument validation happens before any CUDA call
    st = hegjoin_b200.lib.hj_index_create(None, 0, 0, 0, 0, 0.0, None, None, None, None)
    assert st == hegjoin_b200.HJ_ERR_INVALID
    assert "invalid" in hegjoin_b200.last_error() or "null" in hegjoin_b200.last_error()
