"""The bounds-checked build (-DDSB_CHECK): every index that comes from a
host-built table (ring slots and cells, gridding rows and baselines,
combine targets) is range-checked on the device; a violation is recorded as
DSB_E_BOUNDS in the status word and the access skipped, so a table error
shows as a failed status check instead of a stray write.  The streaming
pipeline's GPU tests run clean under it."""

import os
import subprocess
import sys

import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bounds_error_code_is_declared():
    with open(os.path.join(ROOT, "include", "dsb200.h")) as f:
        assert "#define DSB_E_BOUNDS 6" in f.read()


@pytest.mark.gpu
def test_pipeline_tests_clean_under_bounds_checked_build():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sys.path.insert(0, ROOT)
    import __graft_entry__ as g
    if not os.path.exists(g.SO_CHECK):
        g.build(check=True)
    env = dict(os.environ, DSB200_CHECK="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-x", "-q", "-m", "gpu",
                        "-p", "no:cacheprovider", "tests/test_pipeline_gpu.py",
                        "tests/test_batched.py"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout
