"""The C++ host library and CLIs build and link (CPU only)."""
import os
import subprocess

import tmfqsfullstate_b200 as tq


def test_host_artifacts_exist():
    assert os.path.exists(tq.HOST_LIB_PATH)
    for b in ("grover", "groverLazy", "qftG", "test_host_api"):
        assert os.access(os.path.join(tq.BIN_DIR, b), os.X_OK), b


def test_cli_usage_without_arguments():
    for b, expect in (("grover", "Usage: ./grover"), ("groverLazy", "Usage: ./groverLazy"), ("qftG", "Usage: ./qftG")):
        p = subprocess.run([os.path.join(tq.BIN_DIR, b)], capture_output=True, text=True, timeout=60)
        assert p.returncode == 1 and expect in p.stdout


def test_cli_rejects_bad_arguments():
    p = subprocess.run([os.path.join(tq.BIN_DIR, "grover"), "0", "1"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "Number of qubits must be an integer >= 1" in p.stdout
    p = subprocess.run([os.path.join(tq.BIN_DIR, "qftG"), "5", "--bogus"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "Unknown option: --bogus" in p.stdout
