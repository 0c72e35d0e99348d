"""C-ABI checks that need no GPU: the library builds for sm_100a, loads, and
exports every entry point that include/ygx.h declares."""

import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "ygx.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ygx_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = _declared()
    assert "ygx_encode_sort" in names and "ygx_traverse_walk" in names
    assert len(names) >= 20


def test_library_loads_and_exports_all_declared_symbols():
    from yggdrax_b200 import _lib, build_ext

    build_ext.build()
    lib = ctypes.CDLL(build_ext.LIB)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    bound = set(_lib.exported_symbols())
    assert set(_declared()) - {"ygx_traverse_status"} <= bound | {"ygx_traverse_status"}


def test_workspace_size_queries_run_without_gpu():
    from yggdrax_b200 import _lib

    lib = _lib.lib()
    for n in (0, 1, 1000, 1 << 20):
        assert lib.ygx_encode_sort_workspace_size(n) > 0
        assert lib.ygx_sort_pairs_workspace_size(n) > 0
    assert lib.ygx_topology_workspace_size(1024) > lib.ygx_topology_workspace_size(2)
    assert lib.ygx_traverse_workspace_size(2047, 1024, 1 << 16, 1 << 16) > (1 << 16) * 24


def test_packed_reorder_refuses_misaligned_records_before_launch():
    """The packed gather reads 16-byte records; a record array off that
    boundary is refused on the host (YGX_ERR_ARG) before any CUDA call, so
    the check runs here without a GPU on fake, never dereferenced pointers."""
    from yggdrax_b200 import _lib

    lib = _lib.lib()
    for addr in (0x10004, 0x10008, 0x1000C):
        assert lib.ygx_reorder_packed(addr, 0x20000, 100, 64, None, None, None, None,
                                      None) == 1
    assert lib.ygx_reorder_packed(0x10000, 0x20000, 100, 48, None, None, None, None,
                                  None) == 1  # index width
    assert lib.ygx_reorder_packed(0x10000, None, 100, 64, None, None, None, None, None) == 1


def test_sort_pairs_refuses_bad_arguments_before_launch():
    """ygx_sort_pairs checks its arguments on the host before any CUDA call
    (YGX_ERR_ARG = 1), under both digit widths; the pointers here are fake
    and never dereferenced."""
    from yggdrax_b200 import _lib

    lib = _lib.lib()
    n = 1000
    ws_bytes = lib.ygx_sort_pairs_workspace_size(n)
    keys, kout, vin, vout, ws = 0x100000, 0x200000, 0x300000, 0x400000, 0x500000
    old = ctypes.c_int(0)
    assert lib.ygx_tune_get(_lib.TUNE["sort_bits"], ctypes.byref(old)) == 0
    try:
        for bits in (8, 11):
            assert lib.ygx_tune_set(_lib.TUNE["sort_bits"], bits) == 0
            call = lib.ygx_sort_pairs
            assert call(keys, vin, -1, 0, 63, kout, vout, ws, ws_bytes, None) == 1
            assert call(keys, vin, n, 0, 63, kout, vout, ws, ws_bytes - 1, None) == 1
            assert call(keys, vin, n, 0, 63, kout, vout, None, ws_bytes, None) == 1
            assert call(keys, vin, n, 20, 20, kout, vout, ws, ws_bytes, None) == 1
            assert call(keys, vin, n, -1, 8, kout, vout, ws, ws_bytes, None) == 1
            assert call(keys, vin, n, 0, 65, kout, vout, ws, ws_bytes, None) == 1
            assert call(keys, vin, n, 0, 63, kout, vin, ws, ws_bytes, None) == 1  # values alias
            assert call(keys, vin, 0, 0, 63, kout, vout, ws, ws_bytes, None) == 0  # nothing to do
    finally:
        lib.ygx_tune_set(_lib.TUNE["sort_bits"], old.value)


def test_tune_knob_ids_match_the_header():
    """The binding's knob table (yggdrax_b200._lib.TUNE) and the header's
    YGX_TUNE_* numbers are kept by hand in two places; they must agree, and
    every knob the header declares must be readable."""
    from yggdrax_b200 import _lib

    src = open(os.path.join(ROOT, "include", "ygx.h")).read()
    header = {m.group(1).lower(): int(m.group(2))
              for m in re.finditer(r"#define YGX_TUNE_([A-Z_]+)\s+(\d+)", src)}
    assert header == _lib.TUNE
    lib = _lib.lib()
    v = ctypes.c_int(0)
    for knob in header.values():
        assert lib.ygx_tune_get(knob, ctypes.byref(v)) == 0


def test_product_does_not_import_oracle():
    pkg = os.path.join(ROOT, "yggdrax_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh")):
                text = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in text.replace("oracle is", ""), f
