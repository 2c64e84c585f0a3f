"""The sharded (multi-GPU) calls' partitioning and combining logic, run as
world_size-2 gloo process groups on the CPU.

Each rank's local arithmetic is the oracle (the checker, on CPU ranks)
instead of the library: what is under test is which rank holds which
columns / elements / instances, and how the per-rank results are combined --
the dot product's rank-ordered FP64 sum, and iamax's first index across the
shard boundary with ties and NaN.  The results must equal the oracle's on
the whole problem."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, TESTS)

from clgpu_b200.sharded import column_blocks, combine_iamax, instance_ranges  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleLocal:
    """A rank's local arithmetic on CPU numpy arrays, through the oracle."""

    def __init__(self):
        import oracle_lib as O
        self.O = O

    def sdot(self, n, x, y):
        return float(np.float32(self.O.sdot(n, np.ascontiguousarray(x[:n]), 1, np.ascontiguousarray(y[:n]), 1)))

    def sasum(self, n, x):
        return float(np.float32(self.O.sasum(n, np.ascontiguousarray(x[:n]), 1)))

    def snrm2(self, n, x):
        return float(np.float32(self.O.snrm2(n, np.ascontiguousarray(x[:n]), 1)))

    def isamax(self, n, x):
        xs = np.ascontiguousarray(x[:n])
        i = int(self.O.isamax(n, xs, 1))
        return i, float(abs(xs[i]))

    def sgemm(self, ta, tb, m, n, k, alpha, A, lda, Bm, ldb, beta, Cm, ldc):
        self.O.sgemm(ta, tb, m, n, k, alpha, A, lda, Bm, ldb, beta, Cm, ldc)


def _vector(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    return x, rng.uniform(-1, 1, n).astype(np.float32)


def _rank(rank, world, port, out):
    import datetime

    from clgpu_b200.sharded import Sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sh = Sharded(local=OracleLocal())
        res = {}
        # ---- level 1: contiguous segments at 16-byte boundaries
        n = 100003
        x, y = _vector(n, 1)
        blocks = column_blocks(n, world, align=4)
        o, c = blocks[rank]
        res["sdot"] = sh.sdot(c, x[o:o + c], y[o:o + c])
        res["sasum"] = sh.sasum(c, x[o:o + c])
        res["snrm2"] = sh.snrm2(c, x[o:o + c])
        # iamax: the largest |x| twice, once in each segment (first index wins),
        # and a NaN at the start of the second segment (skipped)
        xi = x.copy()
        b0 = blocks[1][0]
        xi[b0 + 17] = -3.0
        xi[b0 - 5] = 3.0
        xi[b0] = np.nan
        res["isamax"] = sh.isamax(c, xi[o:o + c], o)
        # NaN as the very first element pins the answer to 0
        xn = x.copy()
        xn[0] = np.nan
        res["isamax_nan0"] = sh.isamax(c, xn[o:o + c], o)
        # ---- GEMM: A replicated by broadcast from rank 0, columns of B / C by rank
        m, k, nc = 37, 29, 150
        rng = np.random.default_rng(2)
        A = rng.uniform(-1, 1, m * k).astype(np.float32)
        if rank != 0:
            A[:] = 0.0                                    # only rank 0 holds A before the broadcast
        At = torch.from_numpy(A)
        sh.broadcast_(At, src=0)
        A = At.numpy()
        Bfull = rng.uniform(-1, 1, k * nc).astype(np.float32)
        Cfull = rng.uniform(-1, 1, m * nc).astype(np.float32)
        cb = column_blocks(nc, world, align=8)
        c0, cn = cb[rank]
        Bl = np.ascontiguousarray(Bfull[c0 * k:(c0 + cn) * k])
        Cl = np.ascontiguousarray(Cfull[c0 * m:(c0 + cn) * m])
        sh.sgemm(0, 0, m, cn, k, 1.5, A, m, Bl, k, 0.5, Cl, m)
        gathered = [None] * world
        dist.all_gather_object(gathered, (c0, Cl))
        res["sgemm_blocks"] = gathered
        res["A_sum"] = float(A.astype(np.float64).sum())
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_sharded_level1_and_gemm_world2():
    import oracle_lib as O
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    n = 100003
    x, y = _vector(n, 1)
    for r in (0, 1):
        assert res[r]["sdot"] == res[0]["sdot"]            # every rank the same value
        assert res[r]["isamax"] == res[0]["isamax"]
    # rank-ordered FP64 sum of the two FP32 partials: within 2 ulps of the whole-vector oracle
    want = np.float32(O.sdot(n, x, 1, y, 1))
    assert O.ulp_diff(np.float32(res[0]["sdot"]), want).max() <= 2
    assert O.ulp_diff(np.float32(res[0]["sasum"]), np.float32(O.sasum(n, x, 1))).max() <= 2
    assert O.ulp_diff(np.float32(res[0]["snrm2"]), np.float32(O.snrm2(n, x, 1))).max() <= 2
    b0 = column_blocks(n, 2, align=4)[1][0]
    assert res[0]["isamax"] == b0 - 5                      # first of the tie, across the boundary
    assert res[0]["isamax_nan0"] == 0
    # GEMM column blocks reassemble to the whole product, bit for bit
    m, k, nc = 37, 29, 150
    rng = np.random.default_rng(2)
    A = rng.uniform(-1, 1, m * k).astype(np.float32)
    Bfull = rng.uniform(-1, 1, k * nc).astype(np.float32)
    Cfull = rng.uniform(-1, 1, m * nc).astype(np.float32)
    assert res[1]["A_sum"] == float(A.astype(np.float64).sum())   # the broadcast replicated A
    O.sgemm(0, 0, m, nc, k, 1.5, A, m, Bfull, k, 0.5, Cfull, m)
    got = np.zeros(m * nc, np.float32)
    for c0, Cl in res[0]["sgemm_blocks"]:
        got[c0 * m:c0 * m + Cl.size] = Cl
    assert np.array_equal(got, Cfull)


def test_partitions_cover_everything_once():
    for n in (0, 1, 63, 64, 65, 4096, 100003):
        for parts in (1, 2, 3, 8):
            b = column_blocks(n, parts, align=64)
            assert len(b) == parts
            covered = [c for o, cnt in b for c in range(o, o + cnt)]
            assert covered == list(range(n))
            assert all(o % 64 == 0 for o, cnt in b if cnt)
    rng = np.random.default_rng(4)
    ns, rs = rng.integers(32, 1025, 512), rng.integers(1, 257, 512)
    cost = ns.astype(float) ** 2 * rs
    for parts in (1, 2, 4, 8):
        rg = instance_ranges(cost, parts)
        assert [i for o, c in rg for i in range(o, o + c)] == list(range(512))
        loads = [cost[o:o + c].sum() for o, c in rg]
        assert max(loads) <= cost.sum() / parts + cost.max()   # balanced to within one instance


def test_combine_iamax_rules():
    assert combine_iamax([(0.5, 3), (0.5, 1)]) == 1           # ties: smallest index
    assert combine_iamax([(-1.0, -1), (0.25, 9)]) == 9        # empty segment
    assert combine_iamax([(float("inf"), 0), (float("inf"), 5)]) == 0
    with pytest.raises(ValueError):
        column_blocks(10, 0)
