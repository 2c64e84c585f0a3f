"""iclblasSdotNoAlloc: the SDOT entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc -- code whose device memory
belongs to another allocator, or latency-critical paths where cudaMalloc and
cudaFree (which can synchronize the device) are not allowed.  Its scratch is a
fixed array inside the library shared by every call.  This test calls it
through the C ABI twice in a row (a large call, then a smaller one that reuses
fewer of the array's slots) and checks each result against the regular
iclblasSdot entry point, within the 1-ulp bar of the level-1 tests.  It lives
in a file of its own so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu


def test_sdot_no_alloc_matches_sdot_twice(cuda):
    import torch
    L = B.lib()
    h = C.c_void_p()
    assert L.iclblasCreate(C.byref(h)) == B.SUCCESS
    try:
        assert L.iclblasSetStream(h, C.c_void_p(torch.cuda.current_stream().cuda_stream or None)) == B.SUCCESS
        rng = np.random.default_rng(2024)
        for n, inc in ((3_000_001, 1), (40_000, 3)):
            xh = rng.uniform(-1, 1, n * inc).astype(np.float32)
            yh = rng.uniform(-1, 1, n * inc).astype(np.float32)
            x = torch.from_numpy(xh).to(cuda)
            y = torch.from_numpy(yh).to(cuda)
            r_noalloc = torch.full((1,), float("nan"), device=cuda)
            r_regular = torch.full((1,), float("nan"), device=cuda)
            assert L.iclblasSdotNoAlloc(h, n, C.c_void_p(x.data_ptr()), inc, C.c_void_p(y.data_ptr()), inc,
                                        C.c_void_p(r_noalloc.data_ptr())) == B.SUCCESS
            assert L.iclblasSdot(h, n, C.c_void_p(x.data_ptr()), inc, C.c_void_p(y.data_ptr()), inc,
                                 C.c_void_p(r_regular.data_ptr())) == B.SUCCESS
            torch.cuda.synchronize()
            got, want = np.float32(r_noalloc.item()), np.float32(r_regular.item())
            assert np.isfinite(got)
            assert O.ulp_diff(got, want).max() <= 1, (got, want)
    finally:
        assert L.iclblasDestroy(h) == B.SUCCESS


def test_sdot_no_alloc_rejects_host_operands(cuda):
    x = np.ones(16, np.float32)
    r = np.zeros(1, np.float32)
    with B.Handle() as h:
        assert B.iclblasSdotNoAlloc(h, 16, x, 1, x, 1, r) == B.INVALID_VALUE
