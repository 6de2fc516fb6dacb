"""The bounds-checked engine build (libkc_checked.so, compiled with -DKC_CHECKED).

compute-sanitizer is closed on this pool, so the counting kernels carry their
own checks in that build: every data-dependent scratch index (bitmap words,
membership map, row table, candidate lists, lane stacks) is tested before the
access, and a failure records DEV_ERR_BOUNDS, which the call returns as
KC_ERR_INTERNAL. The parity and local-count suites run against that build in a
child process (KC_LIBRARY selects it); they must pass unchanged.
"""
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def test_parity_suites_pass_on_the_checked_build():
    lib = ROOT / "kcgpu_b200" / "libkc_checked.so"
    assert lib.exists(), "build it with python -m kcgpu_b200.build --checked (build() does)"
    env = dict(os.environ, KC_LIBRARY="libkc_checked.so")
    name = subprocess.run([sys.executable, "-c", "import kcgpu_b200 as kc; print(kc.lib()._name)"], env=env,
                          cwd=ROOT, capture_output=True, text=True, check=True).stdout.strip()
    assert name.endswith("libkc_checked.so"), name
    r = subprocess.run([sys.executable, "-m", "pytest", "-m", "gpu", "-x", "-q", "-p", "no:cacheprovider",
                        "tests/test_gpu_parity.py", "tests/test_gpu_local.py"],
                       env=env, cwd=ROOT, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
