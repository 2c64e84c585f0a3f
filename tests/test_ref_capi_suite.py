"""The reference's own C-API known-answer suite (tests/iclBLAS/test_<routine>.cpp
of the clGPU tree: the 21 hot-path routines, the 13 level-1 copy / swap /
rotation / iamin routines and Sger, Cgeru, Cgerc, Ssymv, Chemv, Ssyrk, Ssyr2k,
Ssymm; 221 tests), compiled unmodified
against the reference's iclBLAS.h by oracle/Makefile:

  - linked against the CPU oracle (oracle/_ref/ref_capi_tests_oracle): pins
    the oracle to the reference's golden vectors;
  - linked against libiclblas_b200.so (oracle/_ref/ref_capi_tests_b200): the
    same binary objects pass on the GPU library, i.e. the library is a
    source- and link-compatible drop-in for these calls.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


def _run(binary):
    r = subprocess.run([binary], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, timeout=600)
    out = r.stdout.decode(errors="replace")
    return r.returncode, out


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "ref_capi_tests_oracle")),
                    reason="reference suite not built (reference tree absent at build time)")
def test_reference_suite_against_oracle():
    rc, out = _run(os.path.join(REF, "ref_capi_tests_oracle"))
    assert rc == 0, out[-4000:]
    assert "[  PASSED  ] 221 tests." in out, out[-2000:]


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "ref_capi_tests_b200")),
                    reason="reference suite not built against the library (reference tree absent at build time); "
                           "tests/test_golden.py carries the reference's vectors instead")
def test_reference_suite_against_gpu_library(cuda):
    binary = os.path.join(REF, "ref_capi_tests_b200")
    rc, out = _run(binary)
    assert rc == 0, out[-4000:]
    assert "[  PASSED  ] 221 tests." in out, out[-2000:]
