"""The allocation-free Dot2 entry point (hpb_dot2_f64_noalloc).

It serves callers that cannot allocate device memory and so cannot create an
hpb_context: code running under an external allocator that owns the whole
device-memory budget, or on a path where cudaMalloc/cudaFree (which can
synchronise the device) are not allowed.  Its scratch is a static device
array shared by all calls.

The test calls it through the C ABI twice in a row, on two different inputs
(the second call must not see the first call's scratch contents), and checks
each result against the context-based hpb_dot2_f64 on the same data with the
tolerance the other Dot2 tests use: both within the reference's compensated
bound B(n, cond)*|exact| of the exact dot (oracle), and within 2 ulp of each
other where cond <= 1e8.  It also checks the stated size limit.  This file
is collected last so that a run stopping at the first failure has run every
other test before it; it passes alone in a fresh process too.
"""
import numpy as np
import pytest

import oracle
from gpu_utils import dev, gendot, red, ulp
from high_precision_blas1_b200 import _lib

pytestmark = pytest.mark.gpu


def noalloc_dot2(torch, X, Y, n):
    out = torch.full((2,), np.nan, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = _lib.lib.hpb_dot2_f64_noalloc(n, X.data_ptr(), Y.data_ptr(), out.data_ptr(), stream)
    assert st == 0, _lib.STATUS.get(st, st)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_dot2_matches_context_dot2_on_two_calls(gpu):
    ctx, torch = gpu
    cases = [(21, 1 << 20, 1e20), (22, 100003, 1e6)]
    for seed, n, cond_target in cases:  # two calls in a row, different inputs
        x, y = gendot(seed, n, cond_target)
        X, Y = dev(torch, x), dev(torch, y)
        got = noalloc_dot2(torch, X, Y, n)
        want = red(ctx, "dot2", X, Y)[:2]
        exact, _ = oracle.exact_dot(x, y)
        cond = oracle.condition_dot(x, y)
        bound = oracle.bound_dot2(n, cond) * abs(exact)
        assert abs(got[0] - exact) <= bound, (seed, got[0], exact)
        assert abs(want[0] - exact) <= bound
        assert abs(got[0] - want[0]) <= 2 * bound
        if cond <= 1e8:
            assert abs(got[0] - want[0]) <= 2 * ulp(want[0])
        assert abs(got[1]) <= 0.5 * ulp(got[0])  # lo is the rounding error of hi


def test_noalloc_dot2_repeated_call_is_deterministic(gpu):
    ctx, torch = gpu
    x, y = gendot(23, 65537, 1e12)
    X, Y = dev(torch, x), dev(torch, y)
    a = noalloc_dot2(torch, X, Y, x.size)
    b = noalloc_dot2(torch, X, Y, x.size)
    assert np.array_equal(a, b)


def test_noalloc_dot2_rejects_sizes_beyond_maximum(gpu):
    ctx, torch = gpu
    X = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    st = _lib.lib.hpb_dot2_f64_noalloc(_lib.NOALLOC_MAX_N + 1, X.data_ptr(), X.data_ptr(), out.data_ptr(), None)
    assert st == -8 and _lib.STATUS[st] == "HPB_ERROR_SIZE_LIMIT"
    st = _lib.lib.hpb_dot2_f64_noalloc(-1, X.data_ptr(), X.data_ptr(), out.data_ptr(), None)
    assert st == -1
    # n = 0 writes a zero result
    st = _lib.lib.hpb_dot2_f64_noalloc(0, None, None, out.data_ptr(), None)
    torch.cuda.synchronize()
    assert st == 0 and out[0].item() == 0.0
