"""The radix pass planner on the host (CPU only): stage programs of the
24-qubit layered circuit's passes, built by tests/radix_plan_check.cu.

Checks the compiled Walsh-Hadamard stage items, the constant-factor slot of
the last stage, and the per-stage geometry precomputed on the host (index
masks, swizzled register offsets, global bits of the direct stores).
"""
import math
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KRI_BFLY, KRI_DIAG, KRI_QFT, KRI_WALSH = 0, 2, 3, 4


@pytest.fixture(scope="module")
def plans(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("radix") / "radix_plan_check")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=compute_100a", "-std=c++17", "--expt-relaxed-constexpr",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tmfqsfullstate_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "radix_plan_check.cu")], check=True, timeout=600)
    out = subprocess.run([exe], capture_output=True, text=True, check=True, timeout=60).stdout
    passes, cur = {}, None
    for line in out.splitlines():
        f = line.split()
        if f[0] == "pass":
            cur = passes[f[1]] = {"ok": int(f[3]), "nstages": int(f[5]), "stages": [], "slots": []}
        elif f[0] == "stage":
            i = f.index("direct")
            st = {"items": [tuple(int(v) for v in t.split(":")) for t in f[3:i]], "direct": int(f[i + 1]),
                  "post": int(f[i + 3])}
            for key in ("rbit", "rsorted", "imask", "roff", "gbit"):
                j = f.index(key)
                st[key] = [int(v) for v in f[j + 1:j + 5]]
            cur["stages"].append(st)
        elif f[0] == "slot":
            cur["slots"].append({"scale": float(f[2]), "x": int(f[10])})
    return passes


def rswz8(j):
    return j ^ (((j >> 4) & 7) << 1)


def test_hadamard_passes_use_compiled_walsh_stages(plans):
    p = plans["h0_12"]
    assert p["ok"] and p["nstages"] == 4
    assert [s["items"] for s in p["stages"][:3]] == [[(KRI_WALSH, 4)]] * 3
    assert p["stages"][3]["items"] == [(KRI_QFT, 1)]
    q = plans["h23_16"]
    assert q["ok"] and [s["items"] for s in q["stages"]] == [[(KRI_WALSH, 4)]] * 2


def test_last_stage_takes_the_pass_scale_alone(plans):
    for name, nh in (("h0_12", 13), ("h23_16", 8)):
        p = plans[name]
        assert p["stages"][-1]["post"] == 1
        assert p["slots"][0]["x"] == 0
        assert math.isclose(p["slots"][0]["scale"], 0.5 ** (nh / 2), rel_tol=1e-15)


def test_stage_geometry_from_the_host(plans):
    lpos = {"h0_12": list(range(13)), "h23_16": list(range(5)) + list(range(16, 24)), "ring": list(range(13))}
    for name, p in plans.items():
        for st in p["stages"]:
            assert st["rsorted"] == sorted(st["rbit"])
            assert st["imask"] == [(1 << b) - 1 for b in st["rsorted"]]
            assert st["roff"] == [rswz8(1 << b) for b in st["rbit"]]
            assert st["gbit"] == [1 << lpos[name][b] for b in st["rbit"]]


def test_ring_pass_keeps_the_phases_after_the_last_hadamard(plans):
    p = plans["ring"]
    assert p["ok"] and p["nstages"] == 2
    assert p["stages"][0]["items"] == [(KRI_WALSH, 4)]
    kinds = [k for k, _ in p["stages"][1]["items"]]
    assert kinds[0] == KRI_WALSH and KRI_DIAG in kinds
