"""The allocation-free point-statistics entry point, called through the C ABI.

flpr_point_stats_noalloc serves callers that may not allocate device memory
themselves (a host application or plugin runtime that owns every device
buffer through its own pool, or code that must not trigger the device
synchronisation an allocation implies).  It keeps its per-block partial
results in a static array inside the library instead of a caller workspace.
This test checks it against the workspace-based flpr_point_stats on two
calls in a row (so the second call runs on scratch that still holds the
first call's contents) and rejects an axis count beyond the scratch limit.

The file name makes pytest collect it last; it also passes alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stats_both(lib, _lib, torch, x):
    n, d = x.shape
    dev = torch.device("cuda", 0)
    dx = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    ref = torch.empty(4 * d, dtype=torch.float64, device=dev)
    ws = torch.empty(max(lib.flpr_point_stats_ws(d, n), 256), dtype=torch.uint8, device=dev)
    _lib.check(lib.flpr_point_stats(d, n, dx.data_ptr(), ref.data_ptr(), ws.data_ptr(),
                                    ws.numel(), stream), "flpr_point_stats")
    out = torch.full((4 * d,), float("nan"), dtype=torch.float64, device=dev)
    _lib.check(lib.flpr_point_stats_noalloc(d, n, dx.data_ptr(), out.data_ptr(), stream),
               "flpr_point_stats_noalloc")
    torch.cuda.synchronize()
    return ref.cpu().numpy().reshape(4, d), out.cpu().numpy().reshape(4, d)


def test_noalloc_point_stats_matches_workspace_version(cuda_ok):
    import torch
    from fastlpr_b200 import _lib
    lib = _lib.load()
    torch.cuda.set_device(0)
    rng = np.random.default_rng(99)
    # calls in a row with different shapes: each reuses the scratch; d = 8 is
    # the largest axis count the scratch holds, and 2e6 points fill every
    # block of the grid (4 per SM; the 1024-block clamp of the scratch is
    # above that on this part)
    for n, d in ((300_000, 2), (12_345, 3), (2_000_000, 8), (777, 8)):
        x = rng.standard_normal((n, d)) * np.arange(1, d + 1) + 5.0
        ref, got = _stats_both(lib, _lib, torch, x)
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)
        # and both agree with numpy (min, max, mean, sum of squared deviations)
        expect = np.stack([x.min(0), x.max(0), x.mean(0), ((x - x.mean(0)) ** 2).sum(0)])
        np.testing.assert_allclose(got, expect, rtol=1e-9)


def test_noalloc_rejects_too_many_axes(cuda_ok):
    from fastlpr_b200 import _lib
    lib = _lib.load()
    assert lib.flpr_point_stats_noalloc(9, 100, None, None, None) == -1
    assert b"static scratch" in lib.flpr_last_error()
