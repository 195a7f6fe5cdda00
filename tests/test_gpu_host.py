"""The C++ host library (the tmfqs:: API with the gpu strategy) and its CLIs on the GPU.

* bin/test_host_api: the reference's integration-test cases restated for the
  gpu strategy, plus batched == per-operation equivalence, in C++.
* grover / groverLazy / qftG: output lines as the reference prints them, the
  golden Grover-20 index with --seed 123456, and the measured index of qftG
  equal to the oracle's on the same input and draw.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu
BIN = tq.BIN_DIR


def run(*args, timeout=600):
    p = subprocess.run([os.path.join(BIN, args[0]), *map(str, args[1:])], capture_output=True, text=True, timeout=timeout)
    return p.returncode, p.stdout


def test_host_api_checks():
    rc, out = run("test_host_api")
    assert rc == 0, out
    assert "host API checks passed" in out


@pytest.mark.parametrize("binary,mode", [("grover", "normal"), ("groverLazy", "lazy")])
def test_grover20_cli(binary, mode):
    rc, out = run(binary, 20, 524287, "--strategy", "gpu", "--seed", 123456, "--verbose")
    assert rc == 0, out
    lines = out.splitlines()
    assert lines[0] == f"Grover mode: {mode}"
    assert lines[1] == "Resolved strategy: gpu"
    assert lines[2] == "Grover search result: 524287"
    assert lines[3] == "Circuit operations: 1628"
    assert lines[4].startswith("Execution seconds: ")


def test_grover_multi_marked_fp32_and_fast():
    for extra in (["--precision", "fp32"], ["--fast"], ["--no-fusion"]):
        rc, out = run("grover", 12, "5,77,3000", "--seed", 1, *extra)
        assert rc == 0, out
        assert int(re.search(r"Grover search result: (\d+)", out).group(1)) in (5, 77, 3000)


@pytest.mark.parametrize("n,family", [(10, "pattern"), (16, "random-phase"), (20, "random-phase")])
def test_qftg_matches_oracle(n, family):
    rc, out = run("qftG", n, "--input-family", family, "--seed", 7, "--strategy", "gpu")
    assert rc == 0, out
    k = int(re.search(r"Measured state \(k\): (\d+)", out).group(1))
    if family == "random-phase":
        r = O.OracleRegister(n, amps=O.random_phase(n, 123456))
        assert "Random seed: 123456" in out
    else:
        states = [8 * x + (x % 2) for x in range(1 << n) if 8 * x + (x % 2) < (1 << n)]
        r = O.OracleRegister(n, uniform=states)
    r.run(O.qft_ops(n))
    assert k == r.measure(float(O.mt_unit(7, 1)[0]))
    if k:
        assert f"Calculated r (N/k): " in out


def test_cli_errors_and_unavailable_backends():
    rc, out = run("grover", 3, 8, "--strategy", "gpu")
    assert rc == 2 and "grover error: Grover marked state is out of range" in out
    rc, out = run("qftG", 4, "--strategy", "dense")
    assert rc == 2 and "Dense backend requested but unavailable in this build" in out
    assert "Available strategies: gpu, auto" in out
