"""libsci itself, built with this backend as its Device (integration/), on the host.

integration/Makefile compiles the reference's own headers and CPU sources, unchanged, with
integration/device.cpp standing where src/core/drivers/device.cpp stands. Without a GPU:
- the reference's own tests/core/drivers/test_device.cpp (compiled unchanged) asks for the graphics
  target, finds no GPU and runs on the CPU, as the reference does without Vulkan, and passes;
- our device_test asks for the CUDA target, which has no CPU fallback: it reports that no sm_100
  device exists and exits 77.
The same programs run on a B200 in tests/test_integration_gpu.py.
"""
import subprocess
from pathlib import Path

import pytest

BUILD = Path(__file__).resolve().parent.parent / "integration" / "_build"


def binary(name):
    path = BUILD / name
    if not path.exists():
        pytest.skip("integration/_build is not built (needs the reference sources)")
    return str(path)


def cuda_visible():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001 - no torch, no GPU
        return False


def test_reference_device_test_falls_back_to_the_cpu_without_a_gpu():
    if cuda_visible():
        pytest.skip("a GPU is visible: the GPU form of this test applies")
    run = subprocess.run([binary("reference_device_test")], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "running on the CPU" in run.stderr


def test_cuda_target_has_no_cpu_fallback():
    if cuda_visible():
        pytest.skip("a GPU is visible: the GPU form of this test applies")
    run = subprocess.run([binary("device_test")], capture_output=True, text=True, timeout=300)
    assert run.returncode == 77, run.stdout + run.stderr
    assert "no usable sm_100 CUDA device" in run.stdout
