"""libsci's public API on a B200 through this backend (integration/), checked against libsci's CPU
path in the same program.

- integration/_build/device_test: sci::Array expressions, reductions, product, solve and
  decompose on Device(Target::cuda), each against the same call on the host (see
  integration/device_test.cpp for every check and its bar);
- integration/_build/reference_device_test: the reference's own tests/core/drivers/test_device.cpp,
  compiled unchanged; its Device(Target::graphics) is served by the CUDA GPU (no "running on the
  CPU" line), and its asserts pass.
"""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

BUILD = Path(__file__).resolve().parent.parent / "integration" / "_build"


def run(name):
    path = BUILD / name
    if not path.exists():
        pytest.fail(f"{path} is missing: build() compiles it where the reference sources are present")
    return subprocess.run([str(path)], capture_output=True, text=True, timeout=600)


def test_libsci_api_on_the_cuda_device():
    result = run("device_test")
    assert result.returncode == 0, result.stdout + result.stderr
    assert "PASSED: 0 failure(s)" in result.stdout
    assert "FAIL" not in result.stdout


def test_reference_device_test_on_the_gpu():
    result = run("reference_device_test")
    assert result.returncode == 0, result.stdout + result.stderr
    assert "running on the CPU" not in result.stderr, "the graphics target fell back to the CPU"
