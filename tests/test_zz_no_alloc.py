"""vlm_exact_sum_noalloc (static device scratch, no allocation) against vlm_exact_sum.

Collected last on purpose: it must pass both in a fresh process, where its first call does the
per-device scratch set-up, and after every other test has used the device.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VLM_OK, VLM_ERR_BAD_ARG = 0, 1


def _noalloc_sum(lib, torch, values):
    """One call through the C ABI on torch's current stream; returns the device result."""
    dv = torch.as_tensor(values, dtype=torch.float64).cuda()
    out = torch.full((1,), -7.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.vlm_exact_sum_noalloc(C.c_void_p(dv.data_ptr()), dv.numel(), C.c_void_p(out.data_ptr()),
                                   C.c_void_p(stream))
    assert st == VLM_OK, lib.vlm_last_error(None)
    torch.cuda.synchronize()
    return float(out.item())


def test_noalloc_matches_exact_sum_twice():
    torch = pytest.importorskip("torch")
    import voluma_b200 as vb
    from voluma_b200._ffi import load
    lib = load()
    rng = np.random.default_rng(11)
    # wide dynamic range, heavy cancellation, more values than one pass of the fixed grid covers
    big = rng.standard_normal(3_000_017) * np.exp2(rng.integers(-60, 60, 3_000_017))
    small = rng.uniform(-1.0, 1.0, 1001)
    for v in (big, small):  # two calls in a row: the second must not see the first call's partials
        got = _noalloc_sum(lib, torch, v)
        assert got == vb.exact_sum(v)  # exact sums: the tolerance is zero
    assert _noalloc_sum(lib, torch, big[::-1].copy()) == vb.exact_sum(big)
    assert _noalloc_sum(lib, torch, np.zeros(0)) == 0.0
    assert _noalloc_sum(lib, torch, [1e20, 1.0, -1e20]) == 1.0


def test_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    from voluma_b200._ffi import load
    lib = load()
    dv = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # rejected on the host before any launch, so the short buffer is never read
    st = lib.vlm_exact_sum_noalloc(C.c_void_p(dv.data_ptr()), 2**31, C.c_void_p(out.data_ptr()), None)
    assert st == VLM_ERR_BAD_ARG
    assert b"exceeds the maximum" in lib.vlm_last_error(None)
    st = lib.vlm_exact_sum_noalloc(C.c_void_p(dv.data_ptr()), -1, C.c_void_p(out.data_ptr()), None)
    assert st == VLM_ERR_BAD_ARG
