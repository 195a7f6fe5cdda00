"""The device backend behind the reference's own, unmodified code.

tests/dropin/ builds a copy of the reference tree with the integration patch
(apply_gpu_strategy.py: StorageStrategyKind::Gpu over libtmfqs_b200, the
binding of tests/dropin/gpu_state_backend.cpp) and links the reference's own
integration tests (tests/integration/*, as its tests/CMakeLists.txt:1-19
does), its CLIs and a QFT driver against it.  Here they run on the GPU:

* the four reference test programs with TMFQS_DENSE_BACKEND=gpu, which puts
  every register those programs create -- explicit Dense ones included -- on
  the device backend; each must pass and must have created device backends;
* the reference's qftG / grover / groverLazy CLIs with `--strategy gpu`;
* the QFT (random-phase input) and Grover-20 (configuration 1, both
  diffusion forms) through the reference's own Simulator and QuantumRegister
  (one backend call per operation) on both strategies: identical total
  probability and seeded measurement.
"""
import json
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "dropin", "_build", "bin")


def _run(args, env_extra=None, timeout=600):
    exe = os.path.join(BIN, args[0])
    assert os.path.exists(exe), f"{exe} missing: build it with `make -C tests/dropin` where the reference sources exist"
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = os.path.join(ROOT, "tmfqsfullstate_b200") + ":" + env.get("LD_LIBRARY_PATH", "")
    env.update(env_extra or {})
    return subprocess.run([exe] + list(args[1:]), capture_output=True, text=True, timeout=timeout, env=env)


@pytest.mark.parametrize("prog,banner", [("test_circuit", "Circuit integration tests passed."),
                                         ("test_register_validation", "Register validation tests passed."),
                                         ("test_storage_parity", "Storage parity tests passed."),
                                         ("test_storage_cache", "Storage cache/kernel tests passed.")])
def test_reference_test_programs_on_the_device_backend(prog, banner):
    p = _run([prog], {"TMFQS_DENSE_BACKEND": "gpu"})
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    assert banner in p.stdout
    m = re.search(r"\[tmfqs-gpu\] device backends created: (\d+)", p.stderr)
    assert m, p.stderr[-2000:]
    if prog != "test_storage_cache":  # that program only exercises the (absent) compressed backends
        assert int(m.group(1)) > 0


def test_reference_cli_strategy_gpu():
    p = _run(["qftG", "12", "--input-family", "random-phase", "--strategy", "gpu"])
    assert p.returncode == 0, p.stdout + p.stderr
    assert "Measured state (k):" in p.stdout
    p = _run(["qftG", "11", "--strategy", "gpu"])
    assert p.returncode == 0 and "Measured state (k):" in p.stdout, p.stdout + p.stderr
    for cli in ("grover", "groverLazy"):
        p = _run([cli, "10", "1000", "--strategy", "gpu"])
        assert p.returncode == 0, p.stdout + p.stderr
        assert "Resolved strategy: gpu" in p.stdout


@pytest.mark.parametrize("n", [14, 20])
def test_qft_through_the_reference_simulator_matches_dense(n):
    out = {}
    for strategy in ("dense", "gpu"):
        p = _run(["qft_through_simulator", str(n), strategy])
        assert p.returncode == 0, p.stdout + p.stderr
        out[strategy] = json.loads(p.stdout.strip().splitlines()[-1])
    assert out["gpu"]["operations"] == out["dense"]["operations"] == n + n * (n - 1) // 2 + n // 2
    assert out["gpu"]["total_probability"] == out["dense"]["total_probability"]
    assert out["gpu"]["measured"] == out["dense"]["measured"]


@pytest.mark.parametrize("materialized", [1, 0])
def test_grover20_through_the_reference_simulator_matches_dense(materialized):
    out = {}
    for strategy in ("dense", "gpu"):
        p = _run(["qft_through_simulator", "grover", "20", strategy, "524287", str(materialized)])
        assert p.returncode == 0, p.stdout + p.stderr
        out[strategy] = json.loads(p.stdout.strip().splitlines()[-1])
    assert out["gpu"]["operations"] == out["dense"]["operations"]
    assert out["gpu"]["total_probability"] == out["dense"]["total_probability"]
    assert out["gpu"]["measured"] == out["dense"]["measured"] == 524287
