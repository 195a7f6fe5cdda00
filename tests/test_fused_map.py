"""The exact fused pass's per-chain thread layouts on the host (CPU only),
through tests/fused_map_check.cu: for QFT passes and a pass with scattered
controls, every butterfly of a tile is covered once, each thread's phase mask
holds exactly the entries whose control bit is set in its |1> index, paired
butterflies share their mask, and each quarter-warp's shared accesses hit
distinct banks.  Also bounds the waste -- phase products a warp issues beyond
those its lanes need -- to 2.5 per butterfly (the lane bits that must be
controls on the first chains of a pass).

The same program checks the register-stage plans (plan_stages) of those
passes: register and thread bits partition the tile, the shared slots are a
bijection with conflict-free quarter-warps, every thread's walk applies exactly
the entries whose local control is set in each |1> output, no register-bit
control follows the op's split, and the lane waste stays within 2.5 products
per pair (none once a stage has bits that control nothing)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def run(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("fmap") / "fused_map_check")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=compute_100a", "-std=c++17", "--expt-relaxed-constexpr",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tmfqsfullstate_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "fused_map_check.cu")], check=True, timeout=600)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    return p.returncode, p.stdout


def test_chain_layouts_are_exact_and_conflict_free(run):
    rc, out = run
    assert rc == 0 and out.strip().endswith("result OK"), out[-2000:]
    assert "FAIL" not in out


def test_chain_layout_waste_is_bounded(run):
    _, out = run
    lines = [line.split() for line in out.splitlines() if line.startswith("case ")]
    assert len(lines) > 40
    for f in lines:
        issued, needed, pairs = (float(f[f.index(k) + 1]) for k in ("issued", "needed", "pairs"))
        assert issued - needed <= 2.5 * pairs, " ".join(f)


def test_stage_plans_are_exact(run):
    _, out = run
    lines = [line.split() for line in out.splitlines() if line.startswith("stage ")]
    assert len(lines) >= 40
    for f in lines:
        issued, needed, pairs = (float(f[f.index(k) + 1]) for k in ("issued", "needed", "pairs"))
        assert issued - needed <= 2.5 * pairs, " ".join(f)
    # QFT-28's later stages: lanes on bits that control nothing in them.
    p3 = [f for f in lines if f[1] == "qft28_p3" and f[5] != "0"]
    assert p3 and all(f[f.index("issued") + 1] == f[f.index("needed") + 1] for f in p3)
