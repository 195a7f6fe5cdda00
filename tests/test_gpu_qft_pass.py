"""The dedicated QFT pass of the fast forms against the FP64 oracle.

Passes that are a segment of the QFT ladder (Hadamards on consecutive
descending bits, each followed by the phases pi/2^(b-c) with every lower bit c
of the register), and passes of Hadamards only (Walsh segments), run as
k_qft_pass: register stages of up to 5 (complex64) or
4 (complex128) bits, per-thread and per-tile twiddle tables, a per-pass bank
swizzle.  These cases reach its layouts: whole-register QFTs from one tile up
(one pass, no outer bits) to several passes with outer bits between the local
ones; QFTs on a sub-register (phases stop at its lowest bit, bits below it are
outer or local non-phase bits); narrower passes (stages shorter than the
register width, filler bits); and two QFTs in a row.  Each case also checks
that the pass actually ran (tmfqs_stats.qft_passes) and agrees with the
general radix pass.

Tolerances: fast FP64 relative L2 <= 1e-12; complex64 relative L2 <= 1e-5.
"""
import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu

TOL = {tq.FP64: 1e-12, tq.FP32: 1e-5}


def sub_qft_ops(n, lo, hi):
    """circuit::appendQft restricted to qubits lo..hi-1 of an n-qubit register."""
    ops = []
    for t in range(lo, hi):
        ops.append(tq.h(t))
        for c in range(t + 1, hi):
            ops.append(tq.cphase(c, t, np.pi / float(1 << (c - t))))
    m = hi - lo
    for k in range(m // 2):
        ops.append(tq.swap(lo + k, hi - 1 - k))
    return ops


def run_gpu(n, amps, ops, prec, qft_pass=True, fused_qubits=0):
    with tq.GpuState(prec) as g:
        g.set_option(tq.OPT_EXACT, 0)
        g.set_option(tq.OPT_QFT_PASS, 1 if qft_pass else 0)
        if fused_qubits:
            g.set_option(tq.OPT_FUSED_QUBITS, fused_qubits)
        g.load(n, amps)
        g.apply_ops(ops)
        out = g.export()
        st = g.stats()
    return out, st


def oracle(n, amps, ops):
    r = O.OracleRegister(n, amps=amps)
    r.run([O.Op(kind=o.kind, q0=o.q0, q1=o.q1, theta=o.theta, state=o.state) for o in ops])
    return r.amplitudes()


def check(n, amps, ops, prec, expect_qft=True, **kw):
    want = oracle(n, amps, ops)
    got, st = run_gpu(n, amps, ops, prec, **kw)
    assert (st["qft_passes"] > 0) == expect_qft, st
    assert O.rel_l2(want, got) <= TOL[prec]
    ref, st0 = run_gpu(n, amps, ops, prec, qft_pass=False, **kw)
    assert st0["qft_passes"] == 0
    assert O.rel_l2(ref, got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("n", [10, 12, 13, 14, 17, 21])
def test_qft_pass_whole_register(prec, n):
    check(n, tq.random_phase(n, 300 + n), tq.qft_ops(n), prec)


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("lo,hi", [(0, 14), (3, 19), (6, 20), (2, 12)])
def test_qft_pass_sub_register(prec, lo, hi):
    n = 20
    rng = np.random.default_rng(lo * 31 + hi)
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    check(n, a, sub_qft_ops(n, lo, hi), prec)


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("fq", [6, 7, 8, 9])
def test_qft_pass_narrow_passes(prec, fq):
    n = 19
    check(n, tq.random_phase(n, 11 * fq), tq.qft_ops(n), prec, fused_qubits=fq)


def run_chunks(n, amps, ops, prec, chunk):
    with tq.GpuState(prec) as g:
        g.set_option(tq.OPT_EXACT, 0)
        g.load(n, amps)
        for i in range(0, len(ops), chunk):
            g.apply_ops(ops[i:i + chunk])
        return g.export(), g.stats()


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("chunk", [3, 7, 16])
def test_hadamard_runs_are_not_qft_segments(prec, chunk):
    # Runs of Hadamards on consecutive qubits without their phases (Hadamard
    # layers, cut into pieces) are not QFT segments: the compiled ladders would
    # add phases the circuit does not have.
    n = 12
    rng = np.random.default_rng(chunk)
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    th = tq.random_angles(3 * n, 9)
    ops = tq.layered_cphase_ops(n, th)
    got, _ = run_chunks(n, a, ops, prec, chunk)
    assert O.rel_l2(oracle(n, a, ops), got) <= TOL[prec]
    layer = [tq.h(q) for q in range(n)]
    got, st = run_chunks(n, a, layer, prec, chunk)
    # They run as Walsh segments instead (butterflies only, no twiddles).
    assert st["qft_passes"] > 0
    assert O.rel_l2(oracle(n, a, layer), got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("bits", ["top", "low", "scattered", "all"])
def test_walsh_pass(prec, bits):
    """Hadamard-only passes through k_qft_pass's Walsh stages: the top 8
    qubits, the 13 lowest index bits (last stage fused into the copy-out), and
    a whole-register layer; against the oracle and the general radix pass.
    Scattered qubits leave the tile's top local bits apart, which k_qft_pass's
    copies need contiguous: that pass stays on k_radix."""
    n = 22
    qs = {"top": list(range(8)), "low": list(range(n - 13, n)), "scattered": [1, 4, 9, 15, 18, 20],
          "all": list(range(n))}[bits]
    ops = [tq.h(q) for q in qs]
    rng = np.random.default_rng(len(qs))
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    check(n, a, ops, prec, expect_qft=bits != "scattered")


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
def test_truncated_ladder_is_not_a_segment(prec):
    # The approximate QFT (phases only between qubits at most 3 apart): its
    # chains stop short of a common lowest bit.
    n = 14
    ops = []
    for t in range(n):
        ops.append(tq.h(t))
        for c in range(t + 1, min(n, t + 4)):
            ops.append(tq.cphase(c, t, np.pi / float(1 << (c - t))))
    amps = tq.random_phase(n, 77)
    got, st = run_gpu(n, amps, ops, prec)
    assert O.rel_l2(oracle(n, amps, ops), got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
def test_qft_pass_twice(prec):
    n = 18
    check(n, tq.random_phase(n, 5), tq.qft_ops(n) + tq.qft_ops(n), prec)


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
def test_qft_pass_basis_inputs(prec):
    # |k> -> (1/sqrt(N)) sum_y exp(2 pi i k y / N) |y> (index bit 0 = last qubit).
    n = 16
    for k in (0, 1, 5, (1 << n) - 1, 12345):
        with tq.GpuState(prec) as g:
            g.set_option(tq.OPT_EXACT, 0)
            g.init_basis(n, k)
            g.apply_ops(tq.qft_ops(n))
            got = g.export()
            assert g.stats()["qft_passes"] > 0
        y = np.arange(1 << n, dtype=np.int64)
        # k*y reduced mod 2^n exactly, so the expected phases carry no argument error.
        want = np.exp(2j * np.pi * ((k * y) % (1 << n)) / (1 << n)) / np.sqrt(1 << n)
        got_c = got[0::2] + 1j * got[1::2]
        assert np.max(np.abs(got_c - want)) <= (1e-13 if prec == tq.FP64 else 2e-6)


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
def test_qft_pass_large_against_exact(prec):
    # 25 qubits: the exact complex128 GPU path (bit-identical to the reference)
    # is the check.
    n = 25
    amps = tq.random_phase(n, 2025)
    with tq.GpuState(tq.FP64) as g:
        g.load(n, amps)
        g.apply_ops(tq.qft_ops(n))
        want = g.export()
    got, st = run_gpu(n, amps, tq.qft_ops(n), prec)
    assert st["qft_passes"] >= 2
    assert O.rel_l2(want, got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("side", ["after", "before"])
def test_walsh_with_ring_phases_stays_radix(prec, side):
    """Hadamards on bits 7..0 of a 20-qubit state with a ring of controlled
    phases and a phase flip after or before them (the layered circuits' last
    pass of a layer and its inverse) are no Walsh segment: the radix pass runs
    them; against the oracle."""
    n = 20
    rng = np.random.default_rng(5 if side == "after" else 6)
    th = rng.uniform(0, 2 * np.pi, n)
    hs = [tq.h(q) for q in range(n - 8, n)]
    diag = [tq.cphase(q, (q + 1) % n, float(th[q])) for q in range(n)] + [tq.phase_flip(12345)]
    ops = hs + diag if side == "after" else diag + hs
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    check(n, a, ops, prec, expect_qft=False)
