"""iclblasSdotNoAlloc: the SDOT entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc -- code whose device memory
belongs to another allocator (a framework's caching pool that has reserved
the free memory), or latency-critical paths where cudaMalloc and cudaFree
(which can synchronize the device) are not allowed.  Its scratch is a fixed
array inside the library shared by every call.

The test calls it through the C ABI on a fresh handle, before any other
routine could have grown that handle's workspace, twice in a row (a large
call, then a smaller strided one that reuses fewer of the array's slots).  It
checks that the device's free memory does not change across those calls, that
each result is bit-identical to the regular iclblasSdot (both launch the same
reduction kernel with the same grid) and within 1 ulp of the oracle.  It lives
in a file of its own so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

CASES = ((3_000_001, 1), (40_000, 3))


def test_sdot_no_alloc_allocates_nothing_and_matches_sdot_twice(cuda):
    import torch
    L = B.lib()
    rng = np.random.default_rng(2024)
    host = []
    dev = []
    for n, inc in CASES:
        xh = rng.uniform(-1, 1, n * inc).astype(np.float32)
        yh = rng.uniform(-1, 1, n * inc).astype(np.float32)
        host.append((xh, yh))
        dev.append((torch.from_numpy(xh).to(cuda), torch.from_numpy(yh).to(cuda),
                    torch.full((1,), float("nan"), device=cuda), torch.full((1,), float("nan"), device=cuda)))
    warm = torch.ones(4096, device=cuda)
    warm_r = torch.zeros(1, device=cuda)
    torch.cuda.synchronize()

    h = C.c_void_p()
    assert L.iclblasCreate(C.byref(h)) == B.SUCCESS
    try:
        stream = torch.cuda.current_stream()
        assert L.iclblasSetStream(h, C.c_void_p(stream.cuda_stream or None)) == B.SUCCESS
        P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        # first call on the fresh handle: loads the kernel's module (lazy
        # loading may allocate for the code) and looks up the array's address
        assert L.iclblasSdotNoAlloc(h, 4096, P(warm), 1, P(warm), 1, P(warm_r)) == B.SUCCESS
        torch.cuda.synchronize()
        assert warm_r.item() == 4096.0
        free_before = torch.cuda.mem_get_info()[0]
        for (n, inc), (x, y, r_noalloc, _) in zip(CASES, dev):
            assert L.iclblasSdotNoAlloc(h, n, P(x), inc, P(y), inc, P(r_noalloc)) == B.SUCCESS
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before, "iclblasSdotNoAlloc changed the device's free memory"
        # the regular entry point afterwards (it may grow the handle's workspace)
        for (n, inc), (x, y, _, r_regular) in zip(CASES, dev):
            assert L.iclblasSdot(h, n, P(x), inc, P(y), inc, P(r_regular)) == B.SUCCESS
        torch.cuda.synchronize()
        for (n, inc), (xh, yh), (_, _, r_noalloc, r_regular) in zip(CASES, host, dev):
            got, regular = np.float32(r_noalloc.item()), np.float32(r_regular.item())
            assert np.isfinite(got)
            assert got.tobytes() == regular.tobytes(), (n, inc, got, regular)
            want = np.float32(O.sdot(n, xh, inc, yh, inc))
            assert O.ulp_diff(got, want).max() <= 1, (n, inc, got, want)
    finally:
        assert L.iclblasDestroy(h) == B.SUCCESS


def test_sdot_no_alloc_rejects_host_operands(cuda):
    x = np.ones(16, np.float32)
    r = np.zeros(1, np.float32)
    with B.Handle() as h:
        assert B.iclblasSdotNoAlloc(h, 16, x, 1, x, 1, r) == B.INVALID_VALUE
