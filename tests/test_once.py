"""The dynamic shared-memory limit of a step kernel is a per-device setting:
the library sets it once per (device, kernel) through csrc/hb_once.h, so a
process that steps batches on two GPUs sets it on each.  Compiled for the CPU
with a fake setter."""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "chans-hipims-flamegpu_b200", "csrc")


@pytest.fixture()
def lib(tmp_path):
    out = str(tmp_path / "libonce.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC,
                    os.path.join(HERE, "once_check.cpp"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    L.once_run.argtypes = [ctypes.c_int, ctypes.c_long]
    L.once_calls.argtypes = [ctypes.c_int, ctypes.c_long]
    return L


def test_setting_runs_once_per_device_and_kernel(lib):
    k1, k2 = 0x1000, 0x2000
    for _ in range(3):
        assert lib.once_run(0, k1) == 0
    assert lib.once_calls(0, k1) == 1
    # the same kernel on a second device is set again, once
    assert lib.once_run(1, k1) == 0 and lib.once_run(1, k1) == 0
    assert lib.once_calls(1, k1) == 1
    assert lib.once_run(0, k2) == 0
    assert lib.once_calls(0, k2) == 1
    assert lib.once_size() == 3


def test_failed_setting_is_retried(lib):
    lib.once_fail_next()
    assert lib.once_run(3, 0x10) == -2
    assert lib.once_run(3, 0x10) == 0  # not remembered after the failure
    assert lib.once_calls(3, 0x10) == 2
    assert lib.once_run(3, 0x10) == 0
    assert lib.once_calls(3, 0x10) == 2
