"""The C ABI library loads without a GPU and exports every declared entry point."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# header -> the library that must export every hj_* function it declares
LIBS = {"hegjoin_b200.h": "libhegjoin_b200.so", "hegjoin_datagen.h": "libhj_datagen.so"}


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    # function declarations: a name followed by "(", not a function-pointer typedef "(*"
    return {m.group(1) for m in re.finditer(r"\b(hj_\w+)\s*\((?!\s*\*)", src)}


def test_library_exports_declared_symbols():
    import hegjoin_b200  # noqa: F401  (the package loads its library)
    for header, libname in LIBS.items():
        lib = ctypes.CDLL(os.path.join(ROOT, "hegjoin_b200", libname))
        declared = _declared(header)
        assert declared, header
        missing = [n for n in sorted(declared) if not hasattr(lib, n)]
        assert not missing, (header, missing)
    assert {"hj_join", "hj_index_create"} <= _declared("hegjoin_b200.h")


def test_join_library_does_not_carry_the_generator():
    lib = ctypes.CDLL(os.path.join(ROOT, "hegjoin_b200", "libhegjoin_b200.so"))
    assert not hasattr(lib, "hj_generate_exp40")


def test_version_and_error_without_gpu():
    import hegjoin_b200
    assert b"sm_100a" in hegjoin_b200.lib.hj_version()
    # argument validation happens before any CUDA call
    st = hegjoin_b200.lib.hj_index_create(None, 0, 0, 0, 0, 0.0, None, None, None, None)
    assert st == hegjoin_b200.HJ_ERR_INVALID
    assert "invalid" in hegjoin_b200.last_error() or "null" in hegjoin_b200.last_error()


def test_join_opts_defaults_and_names():
    import hegjoin_b200 as hj
    o = hj.join_opts()
    assert o.refine == hj.HJ_REFINE_AUTO and o.shard_count == 0 and o.result_capacity == 0
    assert 0 < o.sample_rate <= 1 and 0 < o.mem_fraction <= 1
    for name, code in (("exact", hj.HJ_REFINE_EXACT), ("tc_f16", hj.HJ_REFINE_TC_F16),
                       ("tc_bf16", hj.HJ_REFINE_TC_BF16)):
        assert hj.join_opts(refine=name).refine == code
    o = hj.join_opts(refine="exact", sample_rate=0.5, shard_count=4, shard_index=3, keep_keys=True)
    assert (o.sample_rate, o.shard_count, o.shard_index, o.keep_keys) == (0.5, 4, 3, 1)
    import pytest
    with pytest.raises(KeyError):
        hj.join_opts(refine="no_such_refine")


def test_tensor_core_k_padding():
    import hegjoin_b200 as hj
    # d coordinates + 4 norm columns, rounded up to whole 32-element K blocks
    assert [hj.kpad_for(d) for d in (8, 18, 28, 29, 32, 90)] == [32, 32, 32, 64, 64, 96]
