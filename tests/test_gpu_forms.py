"""The two non-bit-exact forms against the FP64 oracle.

* fast FP64 (TMFQS_OPT_EXACT=0): each H-chain of controlled phases applied as
  one twiddle per amplitude from FP64 tables.  Tolerance: relative L2 <= 1e-12
  (the plain-form bound), identical argmax and seeded measurement.
* complex64 (TMFQS_FP32): FP32 amplitudes, FP64 twiddles rounded once, FP64
  exact reductions.  Tolerance: fidelity >= 1 - 1e-6, relative L2 <= 1e-5.
"""
import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu


def oracle_qft(n, amps):
    r = O.OracleRegister(n, amps=amps)
    r.run(O.qft_ops(n))
    return r


def fidelity(a, b):
    ca = a[0::2] + 1j * a[1::2]
    cb = b[0::2] + 1j * b[1::2]
    return abs(np.vdot(ca, cb)) ** 2 / (np.vdot(ca, ca).real * np.vdot(cb, cb).real)


@pytest.mark.parametrize("n", [2, 5, 9, 13, 16, 20])
def test_fast_fp64_qft(n):
    amps = tq.random_phase(n, 123456)
    ref = oracle_qft(n, amps)
    want = ref.amplitudes()
    with tq.GpuState(tq.FP64) as g:
        g.set_option(tq.OPT_EXACT, 0)
        g.load(n, amps)
        g.apply_ops(tq.qft_ops(n))
        got = g.export()
        rl2 = O.rel_l2(want, got)
        assert rl2 <= 1e-12, rl2
        p = got[0::2] ** 2 + got[1::2] ** 2
        q = want[0::2] ** 2 + want[1::2] ** 2
        assert int(np.argmax(p)) == int(np.argmax(q))
        for rnd in tq.mt19937_unit(123456, 8):
            assert g.sample(float(rnd)) == ref.measure(float(rnd))


@pytest.mark.parametrize("n", [3, 8, 12, 17, 21])
def test_c64_qft_fidelity(n):
    amps = tq.random_phase(n, 123456)
    want = oracle_qft(n, amps).amplitudes()
    with tq.GpuState(tq.FP32) as g:
        g.load(n, amps)
        g.apply_ops(tq.qft_ops(n))
        got = g.export()
        assert 1.0 - fidelity(want, got) <= 1e-6
        assert O.rel_l2(want, got) <= 1e-5
        assert abs(g.total_probability() - 1.0) <= 1e-5


def test_c64_pattern_known_answer():
    """Uniform input over k = 0 mod 2^m: QFT output is 2^-((n-m)/2)... at multiples of 2^(n-m)."""
    n, m = 16, 10
    states = np.arange(0, 1 << n, 1 << m, dtype=np.uint64)
    with tq.GpuState(tq.FP32) as g:
        g.init_uniform(n, states)
        g.apply_ops(tq.qft_ops(n))
        got = g.export()
    c = got[0::2] + 1j * got[1::2]
    peaks = np.arange(0, 1 << n, 1 << (n - m))
    expect = np.zeros(1 << n, dtype=complex)
    expect[peaks] = 2.0 ** (-m / 2.0)
    assert np.max(np.abs(c - expect)) < 1e-6


@pytest.mark.parametrize("n", [6, 11])
def test_c64_single_ops(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    ops = []
    for _ in range(40):
        q = [int(v) for v in rng.permutation(n)[:2]]
        k = int(rng.integers(0, 5))
        ops.append([tq.h(q[0]), tq.x(q[0]), tq.cnot(*q), tq.cphase(q[0], q[1], float(rng.uniform(-3, 3))),
                    tq.swap(*q)][k])
    r = O.OracleRegister(n, amps=a)
    r.run([O.Op(kind=o.kind, q0=o.q0, q1=o.q1, theta=o.theta) for o in ops])
    with tq.GpuState(tq.FP32) as g:
        g.load(n, a)
        g.apply_ops(ops)
        assert O.rel_l2(r.amplitudes(), g.export()) < 1e-5
        g.load(n, a)
        g.set_option(tq.OPT_FUSION, 0)
        g.apply_ops(ops)
        assert O.rel_l2(r.amplitudes(), g.export()) < 1e-5


@pytest.mark.parametrize("materialized", [True, False])
def test_c64_grover(materialized):
    n, marked = 12, [100, 2000]
    with tq.GpuState(tq.FP32) as g:
        g.init_basis(n, 0)
        g.apply_ops([tq.h(q) for q in range(n)])
        v = tq.RegisterView.fresh()
        iters = O.lib().or_grover_iterations(1 << n, 2)
        g.grover_run(v, marked, iters, materialized)
        r = O.OracleRegister(n)
        r.run(O.grover_ops(n, marked, materialized))
        for s in marked:
            re, im = g.amplitude(s)
            if v.overlay:
                re, im = (v.scale_re * re - v.scale_im * im) + v.bias_re, (v.scale_re * im + v.scale_im * re) + v.bias_im
            pr = r.amplitude(s)
            assert abs(re * re + im * im - (pr[0] ** 2 + pr[1] ** 2)) < 1e-5


@pytest.mark.parametrize("materialized", [True, False])
def test_fast_fp64_grover(materialized):
    """The fast FP64 form's Grover run (closed-form materialised pass) against the oracle."""
    n, marked = 12, [100, 2000, 3001]
    with tq.GpuState(tq.FP64) as g:
        g.set_option(tq.OPT_EXACT, 0)
        g.init_basis(n, 0)
        g.apply_ops([tq.h(q) for q in range(n)])
        v = tq.RegisterView.fresh()
        iters = O.lib().or_grover_iterations(1 << n, 3)
        g.grover_run(v, marked, iters, materialized)
        r = O.OracleRegister(n)
        r.run(O.grover_ops(n, marked, materialized))
        for s in list(marked) + [0, 77, 4095]:
            re, im = g.amplitude(s)
            if v.overlay:
                re, im = (v.scale_re * re - v.scale_im * im) + v.bias_re, (v.scale_re * im + v.scale_im * re) + v.bias_im
            pr = r.amplitude(s)
            assert abs(re - pr[0]) < 1e-12 and abs(im - pr[1]) < 1e-12
