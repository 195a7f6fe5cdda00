"""The QFT segment recogniser and planner on the host (CPU only), through
tests/qft_plan_check.cu: which passes run as QFT segments or as Walsh
segments (Hadamards only), their stage counts and their real scale
(1/sqrt(2))^P."""
import math
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("qft") / "qft_plan_check")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=compute_100a", "-std=c++17", "--expt-relaxed-constexpr",
                    "-DTMFQS_QFT_PLAN_ONLY",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tmfqsfullstate_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "qft_plan_check.cu")], check=True, timeout=600)
    out = subprocess.run([exe], capture_output=True, text=True, check=True, timeout=60).stdout
    res = {}
    for line in out.splitlines():
        f = line.split()
        res[f[1]] = {"segment": int(f[3]), "hb": int(f[5]), "r0": int(f[7]), "planned": int(f[9]),
                     "nstages": int(f[11]), "scale": float(f[13]), "walsh": int(f[15]), "marked": int(f[17]),
                     "tail": int(f[19]), "tma": int(f[21]), "dims": int(f[23]), "tok": int(f[25])}
    return res


@pytest.mark.parametrize("name,hadamards,stages,r0", [("qft28_first", 8, 2, 0), ("qft28_last", 12, 3, 0),
                                                     ("sub_register", 7, 2, 3)])
def test_ladder_passes_are_planned(cases, name, hadamards, stages, r0):
    c = cases[name]
    assert c["segment"] == 1 and c["planned"] == 1
    assert c["hb"] == hadamards and c["r0"] == r0 and c["nstages"] == stages
    assert math.isclose(c["scale"], 0.5 ** (hadamards / 2), rel_tol=1e-15)


def test_lone_hadamard_is_a_segment(cases):
    assert cases["lone_h"]["segment"] == 1 and cases["lone_h"]["planned"] == 1 and cases["lone_h"]["nstages"] == 1


@pytest.mark.parametrize("name", ["bare_run", "dropped_phase", "wrong_angle"])
def test_non_ladders_are_rejected(cases, name):
    """Hadamard runs without their phases, a chain missing a phase, and a
    wrong angle go to the general radix pass."""
    assert cases[name]["segment"] == 0


@pytest.mark.parametrize("name,hadamards,stages,tail", [("walsh_top", 8, 2, 0), ("walsh_low", 13, 3, 1),
                                                       ("walsh_scattered", 4, 1, 0), ("bare_run", 4, 1, 0)])
def test_walsh_passes_are_planned(cases, name, hadamards, stages, tail):
    """Hadamard-only passes are no QFT segment but plan as Walsh segments:
    every stage marked, no twiddles, the scale (1/sqrt(2))^P, the lowest
    bits' stage fused into the copy-out."""
    c = cases[name]
    assert c["segment"] == 0 and c["walsh"] == 1 and c["planned"] == 1
    assert c["hb"] == hadamards and c["nstages"] == stages and c["marked"] == stages and c["tail"] == tail
    assert math.isclose(c["scale"], 0.5 ** (hadamards / 2), rel_tol=1e-15)


def test_tensor_map_tiles(cases):
    """complex64 passes whose index bits 0-3 are local load each tile by one
    tensor-map copy when the copy's 128-byte swizzle costs the stages no more
    bank conflicts than the searched swizzle: the box walks the local index in
    order and that swizzle is the pass's shared-memory swizzle.  QFT-28's last
    pass (stages on bits 4-6) keeps the per-thread copies."""
    planned = [k for k, c in cases.items() if c["tma"]]
    assert "qft28_first" in planned and "walsh_top" in planned and "sub_register" in planned
    assert "qft28_last" not in planned and "walsh_low" not in planned
    for k in planned:
        assert cases[k]["tok"] == 1 and 2 <= cases[k]["dims"] <= 5, k
    assert cases["qft28_first"]["dims"] == 4
    # complex128: 8-amplitude rows
    assert cases["qft28_first_c128"]["planned"] == 1 and cases["qft28_last_c128"]["planned"] == 1


def test_walsh_with_diagonal_ops_is_no_segment(cases):
    """Hadamards with controlled phases (and flips) before or after them are
    no Walsh segment: the radix pass applies those phases as per-amplitude
    factors (a Walsh pass with a per-amplitude table factor measured no
    faster)."""
    for k in ("walsh_diag_after", "walsh_diag_before", "walsh_diag_both", "walsh_diag_after_top"):
        assert cases[k]["walsh"] == 0 and cases[k]["segment"] == 0, k
