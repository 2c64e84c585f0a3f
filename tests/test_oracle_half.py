"""The oracle's half-precision GEMM (orc_hgemm, the checker of the library's
iclblasHgemm extension): its binary16 rounding agrees with numpy's IEEE
float -> float16 conversion (round to nearest even, subnormals, overflow to
infinity), and its products sum exactly as a float64 matrix product.

The reference ships FP16 GEMM only as stand-alone experimental OpenCL
kernels (experimental/kernels/hgemm_buf_*.cl: Intel image operands, not part
of its API), which do not build here; this routine's parity is pinned to
IEEE arithmetic instead."""
import numpy as np

import oracle_lib as O


def test_binary16_rounding_matches_numpy():
    rng = np.random.default_rng(1)
    vals = np.concatenate([rng.uniform(-7e4, 7e4, 4000), rng.uniform(-1e-4, 1e-4, 4000),
                           rng.uniform(-1e-7, 1e-7, 4000),
                           [2.98e-8, 2.9802322387695312e-08, 8.940696716308594e-08, 65504.0, 65519.99, 65520.0,
                            -65520.0, 0.0, -0.0, 6.103515625e-05, 6.1e-05]]).astype(np.float32)
    one = np.ones(1, np.float16)
    for v in vals:
        c = np.zeros(1, np.float16)
        O.hgemm(0, 0, 1, 1, 1, float(v), one, 1, one, 1, 0.0, c, 1)
        with np.errstate(over="ignore"):
            want = np.array([v]).astype(np.float16)
        assert c.view(np.uint16)[0] == want.view(np.uint16)[0], v


def test_hgemm_is_one_rounding_of_the_float64_product():
    rng = np.random.default_rng(2)
    for ta in (0, 1):
        for tb in (0, 1):
            m, n, k = 37, 29, 51
            A = rng.uniform(-1, 1, m * k).astype(np.float16)
            B = rng.uniform(-1, 1, k * n).astype(np.float16)
            Cm = rng.uniform(-1, 1, m * n).astype(np.float16)
            lda = k if ta else m
            ldb = n if tb else k
            Am = A.reshape(m, k) if ta else A.reshape(k, m).T      # op(A) row-major view
            Bm = B.reshape(k, n) if tb else B.reshape(n, k).T      # op(B)
            want = (1.5 * (Am.astype(np.float64) @ Bm.astype(np.float64))
                    + 0.5 * Cm.reshape(n, m).T.astype(np.float64)).astype(np.float16)
            C1 = Cm.copy()
            O.hgemm(ta, tb, m, n, k, 1.5, A, lda, B, ldb, 0.5, C1, m)
            assert np.array_equal(C1.reshape(n, m).T, want)
