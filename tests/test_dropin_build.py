"""The integration patch leaves the reference intact (CPU only): the patched
reference tree of tests/dropin (StorageStrategyKind::Gpu added) still passes
the reference's own integration tests on its Dense backend, and without a GPU
the gpu strategy fails with the reference's runtime_error convention
(src/tmfqs/storage/factory/storage_strategy_registry.cpp:99-108)."""
import os
import subprocess

import pytest

from conftest import HAS_GPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "dropin", "_build", "bin")

needs_build = pytest.mark.skipif(not os.path.isdir(BIN), reason="tests/dropin not built (reference sources absent)")


@needs_build
@pytest.mark.parametrize("prog,banner", [("test_circuit", "Circuit integration tests passed."),
                                         ("test_register_validation", "Register validation tests passed."),
                                         ("test_storage_parity", "Storage parity tests passed.")])
def test_patched_reference_tests_pass_on_dense(prog, banner):
    p = subprocess.run([os.path.join(BIN, prog)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    assert banner in p.stdout


@needs_build
def test_gpu_strategy_without_a_device_is_a_runtime_error():
    if HAS_GPU:
        pytest.skip("a GPU is present")
    p = subprocess.run([os.path.join(BIN, "qftG"), "5", "--strategy", "gpu"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 2
    assert "qftG error:" in p.stdout and "Available strategies: dense, auto" in p.stdout
