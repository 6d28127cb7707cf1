"""Runs the C++ mirror tests (tests/cpp/test_host.cpp): the registry rules on
the CPU, the CUDA strategy and the codec API on the GPU."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "cpp", "_build", "test_host")


def _run(group):
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "cpp")], check=True)
    p = subprocess.run([BIN, group], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr


def test_registry_rules():
    _run("registry")


@pytest.mark.gpu
def test_cuda_strategy_and_codec():
    _run("gpu")
