"""Radix passes of the fast forms against the FP64 oracle.

The fast forms (complex64, and complex128 with TMFQS_OPT_EXACT=0) run
Hadamard / controlled-phase passes as radix-2^RB stages: unscaled butterflies,
in-stage phase tables, and cross-stage phases moved to the start or the end of
a stage.  These circuits reach each of those paths: the QFT (phases after
their Hadamard), the inverse QFT (phases before it), free controlled phases
between arbitrary qubits (constant factors, in-stage tables), repeated
Hadamards on one qubit (stage splits), and passes with X / CNOT that the radix
form leaves to the general fused pass.

Tolerances: fast FP64 relative L2 <= 1e-12; complex64 relative L2 <= 1e-5.
"""
import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu

TOL = {tq.FP64: 1e-12, tq.FP32: 1e-5}


def run_both(n, amps, ops, prec, radix=True):
    r = O.OracleRegister(n, amps=amps)
    r.run([O.Op(kind=o.kind, q0=o.q0, q1=o.q1, theta=o.theta) for o in ops])
    with tq.GpuState(prec) as g:
        g.set_option(tq.OPT_EXACT, 0)
        g.set_option(tq.OPT_RADIX, 1 if radix else 0)
        g.load(n, amps)
        g.apply_ops(ops)
        got = g.export()
    return r.amplitudes(), got


def inverse_qft_ops(n):
    out = []
    for o in reversed(tq.qft_ops(n)):
        if o.kind == tq.OP_CPHASE:
            out.append(tq.cphase(o.q0, o.q1, -o.theta))
        else:
            out.append(o)
    return out


def random_input(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(2 << n)
    return a / np.linalg.norm(a)


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("n", [14, 18, 22])
def test_radix_qft(prec, n):
    amps = tq.random_phase(n, 99 + n)
    want, got = run_both(n, amps, tq.qft_ops(n), prec)
    assert O.rel_l2(want, got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("n", [15, 21])
def test_radix_inverse_qft(prec, n):
    amps = random_input(n, n)
    want, got = run_both(n, amps, inverse_qft_ops(n), prec)
    assert O.rel_l2(want, got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("seed", range(4))
def test_radix_random_h_cphase(prec, seed):
    n = 17
    rng = np.random.default_rng(1000 + seed)
    ops = []
    for _ in range(120):
        q = [int(v) for v in rng.permutation(n)[:2]]
        if rng.random() < 0.35:
            ops.append(tq.h(q[0]))
        else:
            ops.append(tq.cphase(q[0], q[1], float(rng.uniform(-np.pi, np.pi))))
    amps = random_input(n, seed)
    want, got = run_both(n, amps, ops, prec)
    assert O.rel_l2(want, got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
def test_radix_repeated_hadamards(prec):
    n = 16
    ops = []
    for q in (0, 3, 3, 0, 15, 15, 7, 0):
        ops.append(tq.h(q))
        ops.append(tq.cphase(q, (q + 5) % n, 0.3 + q))
    amps = random_input(n, 5)
    want, got = run_both(n, amps, ops, prec)
    assert O.rel_l2(want, got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
def test_radix_mixed_with_other_gates(prec):
    n = 16
    ops = tq.qft_ops(n)[:40] + [tq.x(3), tq.cnot(2, 9)] + tq.qft_ops(n)[40:80]
    amps = random_input(n, 6)
    want, got = run_both(n, amps, ops, prec)
    assert O.rel_l2(want, got) <= TOL[prec]


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
def test_radix_matches_general_pass(prec):
    n = 20
    amps = tq.random_phase(n, 7)
    ops = tq.qft_ops(n)
    _, a = run_both(n, amps, ops, prec, radix=True)
    _, b = run_both(n, amps, ops, prec, radix=False)
    assert O.rel_l2(a, b) <= TOL[prec]
