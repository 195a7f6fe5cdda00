#!/usr/bin/env python3
"""Benchmark of the dense state-vector path on B200.

Workload (one step): the reference's QFT circuit on n=28 qubits
(circuit::appendQft: 28 H + 378 controlled phases + 14 swaps = 420 circuit
ops) applied to the random-phase input of QuantumState::randomPhase(28,
123456) in complex128 -- the plain FP64 form, bit-identical to the reference
Dense backend.  Metric: amp-updates/s = circuit ops x 2^n per second of a
step.  The 4 GiB state is larger than L2 (126 MB), so no flush is needed
between steps.

  value   device-resident: the state stays in HBM; each step applies the QFT
          through tmfqs_gpu_apply_ops; timed with CUDA events on the handle's
          stream, max over ranks.
  e2e     the same metric through the C ABI with host buffers: each step
          loads the input from pinned host memory and runs the QFT
          (tmfqs_gpu_load_apply_ops: the copy goes in slabs, each overlapped
          with the first pass's tiles that need it), then reads back the exact
          total probability and a seeded measurement.
  forms   the same QFT in the two fast forms on the same GPU, device-resident:
          complex64 (QFT segment passes k_qft_pass, FP64 twiddles rounded
          once) and complex128 with TMFQS_OPT_EXACT=0; each with its
          amp-updates/s, the HBM fraction of its passes, and its accuracy
          against the plain result (relative L2 error, fidelity, measured
          index); and complex64 again on the general radix pass
          (TMFQS_OPT_QFT_PASS=0) for comparison.
  adjoint the differentiation form (24 qubits, 20 layers of H + ring
          controlled phases, 480 angles, E = sum_q <Z_q Z_{q+1}>): complex64
          forward and adjoint backward with a checkpoint every 48 ops; grad/s,
          backward/forward cost, and the error against the reference's
          parameter-shift gradients (tests/golden/adjoint_ps_n24.json) and
          FP64 central finite differences on the same 32 angles.
  qft32   configuration 3: QFT on 32 qubits, complex64 (32 GiB) beside the
          complex128 plain form (64 GiB) as its FP64 oracle, for the pattern
          input (uniform over k = 0 mod 2^10; analytic answer) and a random-phase
          input generated on the device (torch.Generator, seed 123456 -- the
          reference's host generator would take minutes and 64 GiB of host
          memory at this size).
  grover30 configuration 4: Grover search on 30 qubits, 4 marked states,
          12867 iterations, lazy and materialised diffusion, complex64 (8 GiB)
          and complex128 (16 GiB): per-iteration time and the marked-state
          probability error of complex64.
  block_gate a dense 5-qubit gate (random unitary, a fused 32 x 32 block) on a
          30-qubit complex64 state: the 3xTF32 tensor-core GEMM kernel beside
          the CUDA-core gate kernel, with its HBM fraction and its relative L2
          difference from the CUDA-core result.
  unmodified_simulator  QFT-28 through the reference's own, unmodified
          sim::Simulator and QuantumRegister (one backend call per operation)
          with the integration patch's gpu strategy (tests/dropin), beside the
          fused path above: the cost of per-operation calls without the
          batching hooks.
  --impl reference   the reference's own Dense CPU path (oracle/_ref, compiled
          from the reference sources) on this host, on a bounded sample of the
          same circuit: every 14th operation of QFT-28 (30 operations of all
          kinds: Hadamards, controlled phases on near and far qubits, swaps),
          timed by the reference's Simulator.

roofline: the plain form's dominant kernel k_fused_stages<double> (register
stages of an exact pass of Hadamards and H-chains) is bound by FP64
instruction issue, not HBM: every controlled phase is its own rounded complex
product in the reference's operation order (4 DMUL + 2 DADD, no FMA), and a
Hadamard butterfly is 4 FP64 operations per amplitude.  `achieved` is the
algorithmic FP64 operations of the passes (4 per amplitude per Hadamard, 1.5
per amplitude per controlled phase) over their CUDA-event time, against the
B200's nominal FP64 rate (148 SMs x 64 FP64 lanes x the sampled SM clock);
the HBM fraction of the same launches is reported beside it.

Multi-GPU: the path does not shard at this tier -- N ranks run N independent
replicas ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QFT/Grover amp-updates/s, %HBM peak: FP32-fused vs FP64-plain; adjoint grad/s"
UNIT = "amp-updates/s"
SEED = 123456
REF_SAMPLE_STRIDE = 14  # reference CPU sample: every 14th operation of the QFT circuit
FP64_LANES_PER_SM = 64  # B200 FP64 pipe: DMUL/DADD per SM per clock (nominal)
NUM_SMS = 148


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=25)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--qubits", type=int, default=28)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--form-steps", type=int, default=3)
    p.add_argument("--no-forms", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the QFT-32 and Grover-30 sections")
    p.add_argument("--no-dropin", action="store_true", help="skip the unmodified-Simulator timing")
    return p.parse_args()


def cpu_model():
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def qft_fp64_ops_per_amp(n):
    """Algorithmic FP64 operations per amplitude of the exact QFT-n: a Hadamard
    butterfly is 8 operations per pair (dense_state_backend.cpp:265-271), a
    controlled phase 6 per amplitude with both bits set (:300-301), a quarter
    of the state; the swaps move data only."""
    return 4.0 * n + 1.5 * (n * (n - 1) // 2)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return rank, local, world


def config(n):
    return {
        "workload": f"qft{n}_random_phase_c128_fp64_plain",
        "n_qubits": n,
        "circuit_ops": n + n * (n - 1) // 2 + n // 2,
        "amplitude": "complex128",
        "input": f"QuantumState::randomPhase({n}, {SEED}) (std::mt19937)",
        "state_bytes": 16 << n,
        "l2_policy": "inputs larger than L2 (state 4 GiB vs 126 MB L2); no flush needed",
        "form": "fused passes, bit-identical to the reference Dense backend",
    }


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(n):
    """DRAM bytes per fused-pass launch from the committed ncu summary, scaled to 2^n."""
    path = os.path.join(ROOT, "profiles", "fused_pass_qft_fp64.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["dram_bytes_per_launch"]) * (2.0 ** n) / (2.0 ** int(d["n_qubits"]))
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # Wait (up to 10 s) for the first sample so the timed region is covered.
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        load = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def pass_roofline(kt, name, peak):
    k = kt[name]
    if not k["launches"]:
        return None
    bytes_per = k["bytes"] / k["launches"]
    avg_ms = k["ms"] / k["launches"]
    achieved = bytes_per / (avg_ms / 1e3) / 1e9
    return {"launches": k["launches"], "bytes_per_launch": bytes_per, "avg_launch_ms": avg_ms,
            "achieved_gbs": achieved, "frac": achieved / peak}


def run_form(tq, torch, n, inp, ops, prec, exact, steps, peak, plain, rnd, device, qft_pass=True):
    """One fast form of the QFT on the same input: device-resident timing and accuracy."""
    import numpy as np

    g = tq.GpuState(prec, device)
    g.set_option(tq.OPT_EXACT, 1 if exact else 0)
    g.set_option(tq.OPT_QFT_PASS, 1 if qft_pass else 0)
    stream = torch.cuda.ExternalStream(g.stream())
    g.load(n, inp)
    g.apply_ops(ops)  # warm-up
    ms = []
    kts = []
    for _ in range(steps):
        g.load(n, inp)
        g.sync()
        g.reset_stats()
        g.set_option(tq.OPT_KERNEL_TIMING, 1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.apply_ops(ops)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        kts.append(g.kernel_times())
        qft_passes = g.stats()["qft_passes"]
        g.set_option(tq.OPT_KERNEL_TIMING, 0)
    best = min(range(steps), key=lambda i: ms[i])
    kt = kts[best]
    t = ms[best]
    got = g.export()
    measured = g.sample(rnd)
    g.close()
    ca = plain[0::2] + 1j * plain[1::2]
    cb = got[0::2] + 1j * got[1::2]
    fid = abs(np.vdot(ca, cb)) ** 2 / (np.vdot(ca, ca).real * np.vdot(cb, cb).real)
    rel = float(np.linalg.norm(plain - got) / np.linalg.norm(plain))
    sweep = 2 * (8 if prec == tq.FP32 else 16) * (1 << n)
    passes = kt["fused"]["launches"] + kt["permute"]["launches"]
    return {"ms_per_qft": t, "value": len(ops) * (1 << n) / (t / 1e3), "unit": UNIT,
            "hbm_frac_whole_qft": passes * sweep / (t / 1e3) / 1e9 / peak,
            "sweeps": passes, "fused_pass": pass_roofline(kt, "fused", peak),
            "permute_pass": pass_roofline(kt, "permute", peak), "qft_segment_passes": qft_passes,
            "rel_l2_vs_plain": rel, "fidelity_vs_plain": float(fid), "measured": measured}


def run_adjoint(tq, torch, device, reps=3):
    """Configuration 5: the adjoint gradient in complex64 and its checks."""
    import numpy as np

    n, layers, every = 24, 20, 48
    th = tq.random_angles(n * layers, SEED)
    ops = tq.layered_cphase_ops(n, th)
    masks, weights = tq.zz_ring_observable(n)
    g = tq.GpuState(tq.FP32, device)
    g.init_basis(n, 0)
    g.apply_ops(ops)  # warm-up
    g.adjoint_gradient(ops, masks, weights, every)
    fwd, tot = [], []
    for _ in range(reps):
        g.init_basis(n, 0)
        g.sync()
        t0 = time.perf_counter()
        g.apply_ops(ops)
        fwd.append(time.perf_counter() - t0)
        g.init_basis(n, 0)
        g.sync()
        t0 = time.perf_counter()
        e, grads = g.adjoint_gradient(ops, masks, weights, every)
        tot.append(time.perf_counter() - t0)
    g.close()
    f, t = min(fwd), min(tot)
    out = {"n_qubits": n, "layers": layers, "angles": len(grads), "form": "complex64", "checkpoint_every": every,
           "forward_ms": f * 1e3, "forward_backward_ms": t * 1e3, "backward_over_forward": (t - f) / f,
           "grad_per_s": len(grads) / t, "expectation": e}
    gold_path = os.path.join(ROOT, "tests", "golden", "adjoint_ps_n24.json")
    if os.path.exists(gold_path):
        with open(gold_path) as fh:
            gold = json.load(fh)
        idx = gold["indices"]
        out["max_abs_err_vs_reference_parameter_shift"] = float(np.max(np.abs(grads[idx] - np.array(gold["ps_grad"]))))
        out["expectation_err_vs_reference"] = abs(e - gold["expectation"])
        # FP64 central differences (h = 1e-6) on the same angles, complex128 fast form on the GPU.
        h = tq.GpuState(tq.FP64, device)
        h.set_option(tq.OPT_EXACT, 0)
        fd = []
        for i in idx:
            es = []
            for s in (+1e-6, -1e-6):
                tt = th.copy()
                tt[i] += s
                h.init_basis(n, 0)
                es.append(h.adjoint_gradient(tq.layered_cphase_ops(n, tt), masks, weights, 0)[0])
            fd.append((es[0] - es[1]) / 2e-6)
        h.close()
        out["max_abs_err_vs_fp64_fd"] = float(np.max(np.abs(grads[idx] - np.array(fd))))
        out["checked_angles"] = len(idx)
    return out


def _timed_ops(torch, g, ops):
    stream = torch.cuda.ExternalStream(g.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g.sync()
    e0.record(stream)
    g.apply_ops(ops)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _compare(torch, a, b, chunk=1 << 27):
    """Fidelity and relative L2 error of two interleaved device states (FP64 accumulation)."""
    dot_re = dot_im = na = nb = diff = 0.0
    for i in range(0, a.numel(), 2 * chunk):
        x = a[i:i + 2 * chunk].double().view(-1, 2)
        y = b[i:i + 2 * chunk].double().view(-1, 2)
        dot_re += float((x[:, 0] * y[:, 0] + x[:, 1] * y[:, 1]).sum())
        dot_im += float((x[:, 0] * y[:, 1] - x[:, 1] * y[:, 0]).sum())
        na += float((x * x).sum())
        nb += float((y * y).sum())
        diff += float(((x - y) ** 2).sum())
    return (dot_re ** 2 + dot_im ** 2) / (na * nb), (diff / na) ** 0.5


def _pattern_error(torch, t, n, m, chunk=1 << 27):
    """max |a_y - expected_y| for the QFT of the uniform state over k = 0 mod 2^m."""
    peak = 2.0 ** (-m / 2.0)
    step = 1 << (n - m)
    worst = 0.0
    for i in range(0, t.numel() // 2, chunk):
        x = t[2 * i:2 * (i + chunk)].double().view(-1, 2)
        idx = torch.arange(i, i + x.shape[0], device=x.device)
        exp_re = torch.where(idx % step == 0, torch.full_like(x[:, 0], peak), torch.zeros_like(x[:, 0]))
        worst = max(worst, float(torch.maximum((x[:, 0] - exp_re).abs(), x[:, 1].abs()).max()))
    return worst


def run_qft32(tq, torch, device, peak):
    import numpy as np

    n, m = 32, 10
    ops = tq.qft_ops(n)
    upd = len(ops) * (1 << n)
    out = {"n_qubits": n, "circuit_ops": len(ops)}
    g64 = tq.GpuState(tq.FP32, device)
    g128 = tq.GpuState(tq.FP64, device)
    try:
        for inp in ("pattern", "random_phase"):
            if inp == "pattern":
                states = np.arange(0, 1 << n, 1 << m, dtype=np.uint64)
                g64.init_uniform(n, states)
                g128.init_uniform(n, states)
            else:
                g64.init_zero(n)
                g128.init_zero(n)
                t64, t128 = g64.tensor(), g128.tensor()
                gen = torch.Generator(device=t128.device)
                gen.manual_seed(SEED)
                two_pi, norm = 2.0 * np.arccos(-1.0), 2.0 ** (-n / 2.0)
                chunk = 1 << 26
                for i in range(0, 1 << n, chunk):
                    th = torch.rand(chunk, dtype=torch.float64, device=t128.device, generator=gen) * two_pi
                    blk = torch.stack([torch.cos(th), torch.sin(th)], dim=1).reshape(-1) * norm
                    t128[2 * i:2 * (i + chunk)].copy_(blk)
                    t64[2 * i:2 * (i + chunk)].copy_(blk.float())
                del t64, t128
                torch.cuda.synchronize()
            res = {}
            for name, g, sweep in (("complex64_radix", g64, 16 << n), ("complex128_plain", g128, 32 << n)):
                g.reset_stats()
                g.set_option(tq.OPT_KERNEL_TIMING, 1)
                ms = _timed_ops(torch, g, ops)
                kt = g.kernel_times()
                g.set_option(tq.OPT_KERNEL_TIMING, 0)
                passes = kt["fused"]["launches"] + kt["permute"]["launches"]
                res[name] = {"ms_per_qft": ms, "value": upd / (ms / 1e3), "sweeps": passes,
                             "hbm_frac_whole_qft": passes * sweep / (ms / 1e3) / 1e9 / peak}
            fid, rel = _compare(torch, g128.tensor(), g64.tensor())
            res["fidelity_c64_vs_c128"] = fid
            res["rel_l2_c64_vs_c128"] = rel
            # experiment::compareStates on the device (reference semantics, exact sums).
            res["compare_states_c64_vs_c128"] = g128.compare(g64)
            res["speedup_c64_vs_c128_plain"] = res["complex128_plain"]["ms_per_qft"] / res["complex64_radix"]["ms_per_qft"]
            if inp == "pattern":
                res["max_abs_err_vs_analytic"] = {"complex64": _pattern_error(torch, g64.tensor(), n, m),
                                                  "complex128": _pattern_error(torch, g128.tensor(), n, m)}
            out[inp] = res
            torch.cuda.empty_cache()
    finally:
        g64.close()
        g128.close()
    return out


def run_grover30(tq, torch, device, peak, sweep_iters=64):
    """Configuration 4: Grover search on 30 qubits, 4 marked states, 12867 iterations.

    Forms: lazy (overlay; O(1) device work per iteration) and materialised,
    each in complex64 and complex128; the materialised complex128 run in the
    exact form (all iterations replayed per amplitude in one temporal pass,
    bit-identical) and in the fast form (the iterations' closed form as one
    affine sweep, like complex64).  Accuracy of complex64 against complex128:
    fidelity and relative L2 of the whole logical state, and the marked-state
    probability error.  The per-iteration sweep form (materialised diffusion
    as one update sweep per iteration, the cached sum maintained exactly as
    QuantumRegister does) is timed over `sweep_iters` iterations with its HBM
    fraction."""
    import math

    n, nm = 30, 4
    marked = [int(v) for v in tq.uniform_states(SEED, nm, 0, (1 << n) - 1)]
    iters = int(math.floor(math.pi / 4.0 * math.sqrt((1 << n) / nm)))
    out = {"n_qubits": n, "marked": marked, "iterations": iters}

    def prepared(prec, exact=True, fusion=True):
        g = tq.GpuState(prec, device)
        g.set_option(tq.OPT_EXACT, 1 if exact else 0)
        g.set_option(tq.OPT_GROVER_FUSION, 1 if fusion else 0)
        g.init_basis(n, 0)
        g.apply_ops([tq.h(q) for q in range(n)])
        return g, tq.RegisterView.fresh()

    def p_marked(g, view):
        p = 0.0
        for st in marked:
            re, im = g.amplitude(st)
            if view.overlay:
                re, im = ((view.scale_re * re - view.scale_im * im) + view.bias_re,
                          (view.scale_re * im + view.scale_im * re) + view.bias_im)
            p += re * re + im * im
        return p

    for form in ("lazy", "materialized"):
        mat = form == "materialized"
        runs = [("complex64", tq.FP32, True), ("complex128", tq.FP64, True)]
        if mat:
            runs.append(("complex128_fast", tq.FP64, False))
        held = {}
        for name, prec, exact in runs:
            g, view = prepared(prec, exact)
            g.sync()
            t0 = time.perf_counter()
            g.grover_run(view, marked, iters, mat)
            g.sync()
            secs = time.perf_counter() - t0
            d = {"seconds": secs, "us_per_iteration": secs / iters * 1e6, "p_marked": p_marked(g, view)}
            if mat:
                d["algorithm"] = ("one temporal pass: every iteration replayed per amplitude in registers, bit-identical"
                                  if exact and prec == tq.FP64 else
                                  "closed form: K iterations as one affine sweep (FP64 scalars, rounded once)")
            out[f"{name}_{form}"] = d
            if view.overlay:  # materialise the overlay so the stored state is the logical one
                g.affine((view.scale_re, view.scale_im), (view.bias_re, view.bias_im))
            if name == "complex128_fast":
                g.close()
            else:
                held[name] = g
        fid, rel = _compare(torch, held["complex128"].tensor(), held["complex64"].tensor())
        out[f"fidelity_c64_vs_c128_{form}"] = fid
        out[f"rel_l2_c64_vs_c128_{form}"] = rel
        out[f"p_marked_err_c64_{form}"] = abs(out[f"complex64_{form}"]["p_marked"] - out[f"complex128_{form}"]["p_marked"])
        for g in held.values():
            g.close()
        torch.cuda.empty_cache()
    m = out
    m["speedup_c64_vs_c128_exact_materialized"] = m["complex128_materialized"]["seconds"] / m["complex64_materialized"]["seconds"]
    m["speedup_c64_vs_c128_fast_materialized"] = (m["complex128_fast_materialized"]["seconds"] /
                                                  m["complex64_materialized"]["seconds"])
    m["speedup_c64_vs_c128_lazy"] = m["complex128_lazy"]["seconds"] / m["complex64_lazy"]["seconds"]

    # The per-iteration sweep form: one inversion sweep per iteration.
    for name, prec, b in (("complex64", tq.FP32, 8), ("complex128", tq.FP64, 16)):
        g, view = prepared(prec, True, fusion=False)
        g.grover_run(view, marked, 2, True)  # warm-up: the first sum pass and the first sweeps
        g.sync()
        g.reset_stats()
        g.set_option(tq.OPT_KERNEL_TIMING, 1)
        t0 = time.perf_counter()
        g.grover_run(view, marked, sweep_iters, True)
        g.sync()
        secs = time.perf_counter() - t0
        kt = g.kernel_times()
        g.set_option(tq.OPT_KERNEL_TIMING, 0)
        g.close()
        sweep = 2 * b * (1 << n)
        gate = kt["gate"]
        dev_ms = gate["ms"] / max(1, gate["launches"])
        out[f"{name}_per_iteration_sweep"] = {
            "iterations_timed": sweep_iters, "ms_per_iteration": secs / sweep_iters * 1e3,
            "sweep_ms": dev_ms, "sweeps": gate["launches"], "bytes_per_sweep": sweep,
            "hbm_frac": sweep / (dev_ms / 1e3) / 1e9 / peak if gate["launches"] else None,
            "projected_seconds_all_iterations": secs / sweep_iters * iters}
    return out


def run_block_gate(tq, torch, device, peak, reps=3):
    import numpy as np

    n, k = 30, 5
    rng = np.random.default_rng(SEED)
    q, r = np.linalg.qr(rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k)))
    u = q * (np.diag(r) / np.abs(np.diag(r)))
    qubits = np.array([0, 5, 11, 16, 22], dtype=np.uint32)  # index bits 29, 24, 18, 13, 7
    op = tq.gate(u, qubits)
    sweep = 2 * 8 * (1 << n)
    out = {"n_qubits": n, "k": k, "targets": qubits.tolist(), "bytes_per_gate": sweep}
    states = {}
    for name, tensor in (("tensor_cores_3xtf32", 1), ("cuda_cores", 0)):
        g = tq.GpuState(tq.FP32, device)
        g.set_option(tq.OPT_TENSOR, tensor)
        g.init_basis(n, 0)
        g.apply_ops([tq.h(qq) for qq in range(n)])
        g.apply_ops([op])  # warm-up
        ms = min(_timed_ops(torch, g, [op]) for _ in range(reps))
        out[name] = {"ms": ms, "gbs": sweep / (ms / 1e3) / 1e9, "frac": sweep / (ms / 1e3) / 1e9 / peak}
        states[name] = g
    out["rel_l2_tensor_vs_cuda_cores"] = states["cuda_cores"].compare(states["tensor_cores_3xtf32"])["rel_l2"]
    for g in states.values():
        g.close()
    return out


def run_unmodified_simulator(n, fused_ms):
    """QFT-n through the reference's own Simulator/QuantumRegister on the gpu
    strategy (tests/dropin, integration patch only): one backend call, and so
    one device pass, per operation."""
    exe = os.path.join(ROOT, "tests", "dropin", "_build", "bin", "qft_through_simulator")
    if not os.path.exists(exe):
        return {"unavailable": "tests/dropin not built"}
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = os.path.join(ROOT, "tmfqsfullstate_b200") + ":" + env.get("LD_LIBRARY_PATH", "")
    p = subprocess.run([exe, str(n), "gpu", str(SEED)], capture_output=True, text=True, timeout=900, env=env)
    if p.returncode != 0:
        return {"unavailable": (p.stdout + p.stderr)[-300:]}
    r = json.loads(p.stdout.strip().splitlines()[-1])
    r["execution_over_fused_step"] = r["execution_seconds"] * 1e3 / fused_ms
    r["note"] = ("Simulator executionSeconds: the circuit's operations one backend call each (no batching hooks); "
                 "run_wall_seconds adds the 4 GiB input load and the export of the result into a host QuantumState")
    # Configuration 1 (Grover-20, materialised) the same way, on both strategies of the patched reference.
    g = {}
    for strategy in ("gpu", "dense"):
        q = subprocess.run([exe, "grover", "20", strategy, "524287", "1", str(SEED)], capture_output=True, text=True,
                           timeout=600, env=env)
        if q.returncode == 0:
            g[strategy] = json.loads(q.stdout.strip().splitlines()[-1])
    if len(g) == 2:
        g["same_total_and_index"] = (g["gpu"]["total_probability"] == g["dense"]["total_probability"] and
                                     g["gpu"]["measured"] == g["dense"]["measured"])
    r["grover20"] = g
    return r


def _section(name, fn, *a, **k):
    """Runs one report section, logging its wall time to stderr."""
    t0 = time.perf_counter()
    out = fn(*a, **k)
    print(f"[bench] {name}: {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
    return out


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import tmfqsfullstate_b200 as tq

    rank, local, world = dist_env()
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    n = args.qubits
    N = 1 << n
    ops = tq.qft_ops(n)
    updates = len(ops) * N

    host = torch.empty(2 * N, dtype=torch.float64, pin_memory=True)
    inp = host.numpy()
    tq.random_phase(n, SEED, inp)
    rnd = float(tq.mt19937_unit(SEED, 1)[0])

    g = tq.GpuState(tq.FP64, local)
    g.load(n, inp)
    stream = torch.cuda.ExternalStream(g.stream())

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        g.apply_ops(ops)
    g.sync()
    g.reset_stats()
    g.set_option(tq.OPT_KERNEL_TIMING, 1)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        g.apply_ops(ops)
    e1.record(stream)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    stats = g.stats()
    kt = g.kernel_times()
    g.set_option(tq.OPT_KERNEL_TIMING, 0)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = world * updates * args.steps / (ms / 1e3)

    # End to end through the C ABI with host buffers.
    e2e_times = []
    measured = total = None
    for _ in range(max(1, args.e2e_steps)):
        barrier()
        t0 = time.perf_counter()
        g.load_apply_ops(n, inp, ops)  # the 4 GiB copy in slabs, overlapped with the first pass
        total = g.total_probability()
        measured = g.sample(rnd)
        t1 = time.perf_counter()
        e2e_times.append(t1 - t0)
    e2e_s = statistics.median(e2e_times)
    # The whole output state against the reference's own (tests/golden/qft28_ref.json: SHA-256 of the
    # reference Dense backend's 4 GiB result, its argmax): bit for bit, so relL2 = 0.
    whole_state = None
    gold_path = os.path.join(ROOT, "tests", "golden", f"qft{n}_ref.json")
    if rank == 0 and os.path.exists(gold_path):
        import hashlib

        with open(gold_path) as fh:
            gold = json.load(fh)
        out_state = g.export()
        digest = hashlib.sha256(memoryview(out_state).cast("B")).hexdigest()
        prob = out_state[0::2] * out_state[0::2] + out_state[1::2] * out_state[1::2]
        arg = int(np.argmax(prob))
        whole_state = {"sha256_equals_reference": digest == gold["sha256"], "argmax": arg,
                       "argmax_equals_reference": arg == gold["argmax"],
                       "rel_l2_vs_reference": 0.0 if digest == gold["sha256"] else None}
        del out_state, prob
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * updates / e2e_s

    fused = kt["fused"]
    peak, peak_kind = measured_peak_hbm()
    roofline = None
    if fused["launches"]:
        bytes_per = fused["bytes"] / fused["launches"]
        avg_ms = fused["ms"] / fused["launches"]
        hbm = bytes_per / (avg_ms / 1e3) / 1e9
        # FP64 operations of the fused passes per launch (each QFT step's fused passes hold all its H and CP).
        launches_per_step = fused["launches"] / args.steps
        fp64_per_launch = qft_fp64_ops_per_amp(n) * N / launches_per_step
        sm_mhz = clk.get("sm_mhz") or 1965.0
        fp64_peak = NUM_SMS * FP64_LANES_PER_SM * sm_mhz * 1e6 / 1e12
        achieved = fp64_per_launch / (avg_ms / 1e3) / 1e12
        roofline = {"bound": "fp64", "kernel": "k_fused_stages<double> (exact pass of Hadamards and H-chains)", "achieved": achieved,
                    "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                    "peak_source": f"nominal FP64 issue rate: {NUM_SMS} SMs x {FP64_LANES_PER_SM} lanes x {sm_mhz:.0f} MHz "
                                   f"(median SM clock sampled in the timed region)",
                    "fp64_ops_per_launch": fp64_per_launch, "fp64_ops_per_amplitude_qft": qft_fp64_ops_per_amp(n),
                    "traffic": profiled_traffic(n), "bytes_per_launch": bytes_per, "avg_launch_ms": avg_ms,
                    "hbm": {"achieved": hbm, "peak": peak, "unit": "GB/s", "frac": hbm / peak,
                            "peak_source": f"{peak_kind} hbm_gbs"},
                    "share_of_step": fused["ms"] / ms if ms else None}

    forms = None
    if rank == 0 and not args.no_forms:
        plain = g.export()
        forms = {}
        for name, prec, exact, qp in (("complex64_radix", tq.FP32, True, True), ("complex128_fast", tq.FP64, False, True),
                                      ("complex64_general_radix", tq.FP32, True, False)):
            forms[name] = run_form(tq, torch, n, inp, ops, prec, exact, max(1, args.form_steps), peak, plain, rnd,
                                   local, qp)
            forms[name]["speedup_vs_plain"] = (ms_per_step / forms[name]["ms_per_qft"])
        # complex64 against both complex128 forms: the exact one (bit-identical to the
        # reference) and the fast one (relL2 <= 1e-12), same GPU, same run.
        forms["speedup_complex64_vs_complex128_exact"] = forms["complex64_radix"]["speedup_vs_plain"]
        forms["speedup_complex64_vs_complex128_fast"] = (forms["complex128_fast"]["ms_per_qft"] /
                                                         forms["complex64_radix"]["ms_per_qft"])
        del plain

    adjoint = None
    if rank == 0 and not args.no_adjoint:
        adjoint = _section("adjoint", run_adjoint, tq, torch, local)
    configs = None
    if rank == 0 and not args.no_configs:
        configs = {"qft32": _section("qft32", run_qft32, tq, torch, local, peak),
                   "grover30": _section("grover30", run_grover30, tq, torch, local, peak),
                   "block_gate": run_block_gate(tq, torch, local, peak)}

    dropin = None
    if rank == 0 and not args.no_dropin:
        dropin = _section("unmodified_simulator", run_unmodified_simulator, n, ms_per_step)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = _section("cpu_baseline", cpu_baseline, n)

    g.close()
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference random-phase input, seed 123456)",
            "config": config(n), "parallelism": f"replicas x{world}",
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 16 * N, "d2h_bytes_per_step": 16,
                    "ms_per_step": e2e_s * 1e3},
            "gpu_launches": int(stats["kernel_launches"]),
            "clocks": clk, "roofline": roofline, "cpu_baseline": cpu, "forms": forms,
            "adjoint": adjoint, "configs": configs, "unmodified_simulator": dropin,
            "kernel_times_ms": {k: round(v["ms"], 3) for k, v in kt.items() if v["launches"]},
            "check": {"total_probability": total, "measured": measured, "whole_state": whole_state,
                      "reference_golden": {"total_probability": 0.99999999999986022, "measured": 138222191}},
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def reference_sample(n, stride, steps, warmup, per_step=None):
    """The reference Dense CPU path (oracle/_ref) on every `stride`-th op of QFT-n
    (all kinds of the circuit's operations, in circuit order).  With per_step,
    each step runs the next `per_step` ops of that sample (cycling), so that
    many steps stay within minutes.  Returns (kind, seconds per timed step,
    ops per timed step)."""
    import oracle as O

    src = "reference" if O.ref_available() else "port"
    sample = (O.ref_qft_ops(n) if src == "reference" else O.qft_ops(n))[::stride]
    k = per_step or len(sample)
    chunks = [[sample[(i * k + j) % len(sample)] for j in range(k)] for i in range(warmup + steps)]
    secs, nops = [], []
    if src == "reference":
        st = O.RefState(n, "random_phase", seed=SEED)
        for i, ops in enumerate(chunks):
            r = st.run(ops, want_amps=False)
            if i >= warmup:
                secs.append(r["seconds"])
                nops.append(len(ops))
    else:
        amps = O.random_phase(n, SEED)
        for i, ops in enumerate(chunks):
            reg = O.OracleRegister(n, amps=amps)
            t0 = time.perf_counter()
            reg.run(ops)
            if i >= warmup:
                secs.append(time.perf_counter() - t0)
                nops.append(len(ops))
    return src, secs, nops


def sample_text(n, nops):
    return (f"every {REF_SAMPLE_STRIDE}th operation of QFT-{n} ({nops} ops: Hadamards, controlled phases, swaps) "
            f"on the random-phase input, reference Simulator executionSeconds, single-threaded Dense backend")


def cpu_baseline(n):
    src, secs, nops = reference_sample(n, REF_SAMPLE_STRIDE, 1, 0)
    v = sum(nops) * (1 << n) / sum(secs)
    return {"value": v, "unit": UNIT, "cores": 1, "kind": src, "cpu_model": cpu_model(), "host_threads": os.cpu_count(),
            "sample": sample_text(n, sum(nops))}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    n = args.qubits
    per_step = 5
    try:
        src, secs, nops = reference_sample(n, REF_SAMPLE_STRIDE, args.steps, args.warmup, per_step)
    except Exception as e:  # the reference could not run here
        print(json.dumps({"impl": "reference", "unavailable": f"{type(e).__name__}: {e}"}))
        return
    s = sum(secs) / len(secs)
    value = sum(nops) * (1 << n) / sum(secs)
    cpu = {"value": value, "unit": UNIT, "cores": 1, "kind": src, "cpu_model": cpu_model(), "host_threads": os.cpu_count(),
           "sample": f"{per_step} consecutive ops per step of the sample: " + sample_text(n, per_step * len(secs)) +
                     " (the Dense backend is single-threaded, so one core)"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference random-phase input, seed 123456)",
        "config": config(n), "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
