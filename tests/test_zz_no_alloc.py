"""The allocation-free sort entry point (ygx_sort_pairs_noalloc).

It serves callers that cannot allocate device memory where they sort -- for
example an XLA custom-call handler registered without a scratch request,
whose framework already holds the GPU's memory pool.  Its scratch is a fixed
array inside libygx.so, so these tests check, through the C ABI, that two
calls in a row (sharing that array) each match the workspace-based
ygx_sort_pairs exactly, that the array's status word reads 0 after each
call (ygx_sort_pairs_noalloc_status), that the value-less and in-place forms
sort stably under the default and a non-default tile shape and with 11-bit
digits, and that sizes
above the array's limit are refused.  This file sorts last so a failure here
never hides another test's result.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 18
YGX_ERR_TOO_LARGE = 9


def _sort_with_workspace(lib, L, keys, vals, bits, dev):
    import torch

    n = keys.numel()
    ko = torch.empty_like(keys)
    vo = torch.empty(n, dtype=torch.int32, device=dev)
    ws = L.workspace(lib.ygx_sort_pairs_workspace_size(n), dev)
    L.check(lib.ygx_sort_pairs(L.ptr(keys), L.ptr(vals), n, 0, bits, L.ptr(ko), L.ptr(vo),
                               L.ptr(ws), ws.numel(), L.stream_handle(dev)), "ygx_sort_pairs")
    return ko, vo


def _sort_noalloc(lib, L, keys, vals, bits, dev):
    import torch

    n = keys.numel()
    ko = torch.empty_like(keys)
    vo = torch.empty(n, dtype=torch.int32, device=dev)
    rc = lib.ygx_sort_pairs_noalloc(L.ptr(keys), L.ptr(vals), n, 0, bits, L.ptr(ko), L.ptr(vo),
                                    L.stream_handle(dev))
    L.check(rc, "ygx_sort_pairs_noalloc")
    return ko, vo


def _noalloc_flags(lib, L, dev):
    flags = np.zeros(1, np.uint32)
    L.check(lib.ygx_sort_pairs_noalloc_status(flags.ctypes.data, L.stream_handle(dev)),
            "ygx_sort_pairs_noalloc_status")
    return int(flags[0])


def test_noalloc_sort_matches_workspace_sort_twice(cuda_device):
    import torch

    from yggdrax_b200 import _lib as L

    lib = L.lib()
    rng = np.random.default_rng(11)
    # Two calls in a row with different sizes and data: the second must not
    # see anything the first left in the shared scratch.
    for n, bits in [(MAX_KEYS, 63), (100_003, 40)]:
        keys_np = rng.integers(0, 1 << min(bits, 62), size=n, dtype=np.uint64)
        keys_np[: n // 4] = keys_np[n // 2]  # ties exercise stability
        vals_np = rng.permutation(n).astype(np.int32)
        keys = torch.from_numpy(keys_np).to(cuda_device)
        vals = torch.from_numpy(vals_np).to(cuda_device)
        k_ref, v_ref = _sort_with_workspace(lib, L, keys, vals, bits, cuda_device)
        k_na, v_na = _sort_noalloc(lib, L, keys, vals, bits, cuda_device)
        assert _noalloc_flags(lib, L, cuda_device) == 0
        torch.cuda.synchronize(cuda_device)
        assert torch.equal(k_na, k_ref)
        assert torch.equal(v_na, v_ref)
        order = np.argsort(keys_np, kind="stable")
        np.testing.assert_array_equal(v_na.cpu().numpy(), vals_np[order])


def test_noalloc_sort_rejects_sizes_above_its_limit(cuda_device):
    import torch

    from yggdrax_b200 import _lib as L

    lib = L.lib()
    n = MAX_KEYS + 1
    keys = torch.zeros(n, dtype=torch.int64, device=cuda_device).view(torch.uint64)
    ko = torch.empty_like(keys)
    vo = torch.empty(n, dtype=torch.int32, device=cuda_device)
    rc = lib.ygx_sort_pairs_noalloc(L.ptr(keys), None, n, 0, 8, L.ptr(ko), L.ptr(vo),
                                    L.stream_handle(cuda_device))
    assert rc == YGX_ERR_TOO_LARGE


@pytest.mark.parametrize("knob,value", [("sort_tile", 0), ("sort_tile", 2), ("sort_bits", 11)])
def test_noalloc_sort_without_values_and_in_place(cuda_device, knob, value):
    """values_in == NULL (each value is the input position) and keys_in ==
    keys_out (the input is staged inside the shared array first), at the
    array's key limit, under the default and one other tile shape, and with
    11-bit digits (a 20-bit key: two passes instead of three)."""
    import torch

    from yggdrax_b200 import _lib as L

    lib = L.lib()
    old = np.zeros(1, np.int32)
    L.check(lib.ygx_tune_get(L.TUNE[knob], old.ctypes.data), "ygx_tune_get")
    L.check(lib.ygx_tune_set(L.TUNE[knob], value), "ygx_tune_set")
    try:
        rng = np.random.default_rng(12 + value)
        n = MAX_KEYS
        keys_np = rng.integers(0, 1 << 20, size=n, dtype=np.uint64)  # many ties
        order = np.argsort(keys_np, kind="stable")
        st = L.stream_handle(cuda_device)
        # no values: positions travel with the keys
        keys = torch.from_numpy(keys_np).to(cuda_device)
        ko = torch.empty_like(keys)
        vo = torch.empty(n, dtype=torch.int32, device=cuda_device)
        L.check(lib.ygx_sort_pairs_noalloc(L.ptr(keys), None, n, 0, 20, L.ptr(ko), L.ptr(vo),
                                           st), "ygx_sort_pairs_noalloc")
        assert _noalloc_flags(lib, L, cuda_device) == 0
        np.testing.assert_array_equal(vo.cpu().numpy(), order.astype(np.int32))
        np.testing.assert_array_equal(ko.cpu().numpy(), keys_np[order])
        # in place: keys_in is keys_out
        vals_np = rng.permutation(n).astype(np.int32)
        kio = torch.from_numpy(keys_np.copy()).to(cuda_device)
        vals = torch.from_numpy(vals_np).to(cuda_device)
        vo2 = torch.empty(n, dtype=torch.int32, device=cuda_device)
        L.check(lib.ygx_sort_pairs_noalloc(L.ptr(kio), L.ptr(vals), n, 0, 20, L.ptr(kio),
                                           L.ptr(vo2), st), "ygx_sort_pairs_noalloc")
        assert _noalloc_flags(lib, L, cuda_device) == 0
        np.testing.assert_array_equal(kio.cpu().numpy(), keys_np[order])
        np.testing.assert_array_equal(vo2.cpu().numpy(), vals_np[order])
    finally:
        L.check(lib.ygx_tune_set(L.TUNE[knob], int(old[0])), "ygx_tune_set")
