"""GPU: the bounds-checked debug build (libqsv_debug.so).

compute-sanitizer is not available on the GPU pool, so the library carries its own checks:
built with DEBUG_BOUNDS=1, every instrumented global access of its kernels must fall inside a
device buffer the library holds, an access outside all of them is redirected to a sink and
counted, and the entry point that launched it fails with the address and source line.  The
cases (tests/debug_cases.py) run in a child process that loads the debug build through
QSV_LIBRARY: its self-test must flag a planted out-of-range read (inside a larger buffer, so
nothing can leave device memory) and pass an in-range one, and every executor, reduction,
sampler, adjoint sweep, batch launch and trajectory run must finish without a flagged access
and agree with the CPU oracle.
"""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

DEBUG_LIB = os.path.join(ROOT, "openqarp_b200", "libqsv_debug.so")


def test_debug_build_flags_nothing_on_the_suite_cases():
    if not os.path.exists(DEBUG_LIB):
        pytest.fail("libqsv_debug.so missing: build it with make -C openqarp_b200/csrc DEBUG_BOUNDS=1")
    env = dict(os.environ, QSV_LIBRARY=DEBUG_LIB)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "debug_cases.py")], env=env,
                       capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0 and "ALL OK" in r.stdout, r.stdout[-3000:] + r.stderr[-3000:]
