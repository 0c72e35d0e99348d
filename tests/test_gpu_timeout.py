"""Bounded device waits: a look-back wait that runs out returns a status, not
a hang.

The onesweep sort's decoupled look-back waits for a predecessor tile's
published digit counts.  Every such wait has an iteration limit (knob
YGX_TUNE_SPIN_LIMIT); a waiter that reaches it sets YGX_FLAG_TIMEOUT in the
status word and the launch ends.  With the limit at 0 a tile gives up at
once whenever its predecessor has not published yet, which a multi-tile sort
meets many times over.  The call must return, report the flag, and the next
call at the default limit must sort correctly on the same context.  (The
reference's counterpart is its overflow-flag / RuntimeError ladder,
_interactions_impl.py:4306-4405: failures come back as flags the host
reads.)
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DEFAULT_SPIN_LIMIT = 1 << 22


def _sort(lib, L, keys, vals, ws, dev):
    import torch

    n = keys.numel()
    ko = torch.zeros_like(keys)
    vo = torch.zeros(n, dtype=torch.int32, device=dev)
    st = L.stream_handle(dev)
    L.check(lib.ygx_workspace_init(L.ptr(ws), ws.numel(), st), "ygx_workspace_init")
    rc = lib.ygx_sort_pairs(L.ptr(keys), L.ptr(vals), n, 0, 63, L.ptr(ko), L.ptr(vo), L.ptr(ws),
                            ws.numel(), st)
    return rc, L.read_status(ws), ko, vo


def test_spin_limit_knob_range(cuda_device):
    from yggdrax_b200 import _lib as L

    lib = L.lib()
    v = np.zeros(1, np.int32)
    L.check(lib.ygx_tune_get(L.TUNE["spin_limit"], v.ctypes.data), "ygx_tune_get")
    assert int(v[0]) == DEFAULT_SPIN_LIMIT
    assert lib.ygx_tune_set(L.TUNE["spin_limit"], -1) == 1  # YGX_ERR_ARG
    assert lib.ygx_tune_set(L.TUNE["spin_limit"], (1 << 24) + 1) == 1
    L.check(lib.ygx_tune_get(L.TUNE["spin_limit"], v.ctypes.data), "ygx_tune_get")
    assert int(v[0]) == DEFAULT_SPIN_LIMIT


@pytest.mark.parametrize("digit_bits", [8, 11])
def test_lookback_wait_that_runs_out_reports_timeout(cuda_device, digit_bits):
    import torch

    from yggdrax_b200 import _lib as L

    lib = L.lib()
    rng = np.random.default_rng(21)
    n = 1 << 24  # 4096 tiles per pass; 8 passes of 8-bit digits, 6 of 11-bit
    keys_np = rng.integers(0, 1 << 63, size=n, dtype=np.uint64)
    vals_np = np.arange(n, dtype=np.int32)
    keys = torch.from_numpy(keys_np).to(cuda_device)
    vals = torch.from_numpy(vals_np).to(cuda_device)
    ws = L.workspace(lib.ygx_sort_pairs_workspace_size(n), cuda_device)
    flags = []
    old_bits = np.zeros(1, np.int32)
    L.check(lib.ygx_tune_get(L.TUNE["sort_bits"], old_bits.ctypes.data), "ygx_tune_get")
    L.check(lib.ygx_tune_set(L.TUNE["sort_bits"], digit_bits), "ygx_tune_set")
    try:
        L.check(lib.ygx_tune_set(L.TUNE["spin_limit"], 0), "ygx_tune_set")
        try:
            for _ in range(4):  # the first call practically always meets a wait
                rc, f, _, _ = _sort(lib, L, keys, vals, ws, cuda_device)
                assert rc == 0  # the launch ended and the call returned
                flags.append(f)
                if f & L.FLAG_TIMEOUT:
                    break
        finally:
            L.check(lib.ygx_tune_set(L.TUNE["spin_limit"], DEFAULT_SPIN_LIMIT), "ygx_tune_set")
        assert any(f & L.FLAG_TIMEOUT for f in flags), flags
        # the context is still usable and the default limit sorts correctly
        rc, f, ko, vo = _sort(lib, L, keys, vals, ws, cuda_device)
    finally:
        L.check(lib.ygx_tune_set(L.TUNE["sort_bits"], int(old_bits[0])), "ygx_tune_set")
    assert rc == 0 and f == 0
    order = np.argsort(keys_np, kind="stable")
    np.testing.assert_array_equal(vo.cpu().numpy(), order.astype(np.int32))
    np.testing.assert_array_equal(ko.cpu().numpy(), keys_np[order])
