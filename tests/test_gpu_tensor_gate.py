"""Dense 4- and 5-qubit gates on complex64 states through the tensor cores.

tcgen05 3xTF32 GEMMs (tc_gate.cu) against the FP64 oracle's applyGate
(gate_block_apply.h:64-213 semantics: targets in block order, first = most
significant block bit) and against the CUDA-core complex64 gate kernel.
Tolerance: relative L2 1e-5 (the complex64 form's bound), on two calls in a
row and for target sets that include the lowest bits (uncoalesced groups).
"""
import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu


def unitary(d, seed):
    rng = np.random.default_rng(seed)
    q, r = np.linalg.qr(rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))
    return q * (np.diag(r) / np.abs(np.diag(r)))


@pytest.mark.parametrize("k", [4, 5])
@pytest.mark.parametrize("targets", ["high", "low", "mixed"])
def test_tensor_gate_matches_oracle(k, targets):
    n = 14
    rng = np.random.default_rng(k * 10 + len(targets))
    qubits = {"high": list(range(k)), "low": list(range(n - 1, n - 1 - k, -1)),
              "mixed": [int(v) for v in rng.permutation(n)[:k]]}[targets]
    u1, u2 = unitary(1 << k, 1), unitary(1 << k, 2)
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    r = O.OracleRegister(n, amps=a)
    r.run([O.gate(u1, qubits), O.gate(u2, qubits[::-1])])
    want = r.amplitudes()
    outs = []
    for tensor in (1, 0):
        with tq.GpuState(tq.FP32) as g:
            g.set_option(tq.OPT_TENSOR, tensor)
            g.load(n, a)
            g.apply_ops([tq.gate(u1, np.array(qubits, dtype=np.uint32))])
            g.apply_ops([tq.gate(u2, np.array(qubits[::-1], dtype=np.uint32))])
            outs.append(g.export())
    assert O.rel_l2(want, outs[0]) < 1e-5
    assert O.rel_l2(outs[1], outs[0]) < 1e-5


def test_tensor_gate_large_state():
    n, k = 24, 5
    qubits = [3, 9, 12, 17, 20]
    u = unitary(1 << k, 7)
    a = tq.random_phase(n, 5)
    with tq.GpuState(tq.FP32) as g, tq.GpuState(tq.FP32) as h:
        g.load(n, a)
        h.load(n, a)
        h.set_option(tq.OPT_TENSOR, 0)
        op = tq.gate(u, np.array(qubits, dtype=np.uint32))
        g.apply_ops([op])
        h.apply_ops([op])
        assert g.compare(h)["rel_l2"] < 1e-6


def brickwork(n, window, layers, seed):
    """Dense 2-qubit unitaries on neighbouring pairs of `window`, with H / X /
    CNOT / controlled phases / swaps between them (both libraries' ops)."""
    rng = np.random.default_rng(seed)
    ours, theirs = [], []
    for layer in range(layers):
        for a in range(layer % 2, len(window) - 1, 2):
            q = [window[a], window[a + 1]]
            u = unitary(4, int(rng.integers(1 << 30)))
            ours.append(tq.gate(u, np.array(q, dtype=np.uint32)))
            theirs.append(O.gate(u, q))
            kind = int(rng.integers(0, 5))
            c, t = (q[0], q[1]) if rng.random() < 0.5 else (q[1], q[0])
            th = float(rng.uniform(-3, 3))
            ours.append([tq.h(c), tq.x(t), tq.cnot(c, t), tq.cphase(c, t, th), tq.swap(c, t)][kind])
            theirs.append([O.h(c), O.x(t), O.cnot(c, t), O.cphase(c, t, th), O.swap(c, t)][kind])
    return ours, theirs


@pytest.mark.parametrize("window", [[3, 4, 5, 6, 7], [9, 10, 11, 12, 13, 14, 15], [0, 2, 4]])
def test_dense_block_fusion(window):
    n = 16
    ours, theirs = brickwork(n, window, 6, len(window))
    rng = np.random.default_rng(3)
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    r = O.OracleRegister(n, amps=a)
    r.run(theirs)
    want = r.amplitudes()
    outs, passes = [], []
    # complex64 on the tensor cores, complex64 on the CUDA-core block kernel,
    # the fast complex128 form (CUDA-core blocks), the exact complex128 form
    # (no blocks: gate by gate, bit-identical).
    for prec, tensor, exact in ((tq.FP32, 1, 1), (tq.FP32, 0, 1), (tq.FP64, 1, 0), (tq.FP64, 1, 1)):
        with tq.GpuState(prec) as g:
            g.set_option(tq.OPT_TENSOR, tensor)
            g.set_option(tq.OPT_EXACT, exact)
            g.load(n, a)
            g.reset_stats()
            g.apply_ops(ours)
            st = g.stats()
            passes.append(st["gate_passes"] + st["fused_passes"])
            outs.append(g.export())
    assert O.rel_l2(want, outs[0]) < 1e-5
    assert O.rel_l2(outs[1], outs[0]) < 1e-5
    assert O.rel_l2(want, outs[2]) < 1e-12
    assert np.array_equal(want, outs[3])
    if len(window) <= 5:
        assert passes[0] == passes[2] == 1  # the whole circuit is one block
    assert passes[0] == passes[1] == passes[2] < passes[3]


@pytest.mark.parametrize("prec,exact,tol", [(tq.FP32, 1, 1e-5), (tq.FP64, 0, 1e-12)])
def test_block_that_starts_with_gates_before_the_dense_gate(prec, exact, tol):
    """H, a controlled phase and a CNOT that lead into a dense gate, and the
    gates after it, within five qubits, make one block: one sweep for the run
    (fast forms)."""
    n = 18
    u = unitary(4, 11)
    ours = [tq.h(2), tq.cphase(2, 5, 0.7), tq.cnot(5, 9), tq.gate(u, np.array([5, 9], dtype=np.uint32)), tq.x(9),
            tq.h(0), tq.h(1)]
    theirs = [O.h(2), O.cphase(2, 5, 0.7), O.cnot(5, 9), O.gate(u, [5, 9]), O.x(9), O.h(0), O.h(1)]
    rng = np.random.default_rng(5)
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    r = O.OracleRegister(n, amps=a)
    r.run(theirs)
    with tq.GpuState(prec) as g:
        g.set_option(tq.OPT_EXACT, exact)
        g.load(n, a)
        g.reset_stats()
        g.apply_ops(ours)
        st = g.stats()
        got = g.export()
    assert O.rel_l2(r.amplitudes(), got) < tol
    # All seven ops act within qubits {2, 5, 9, 0, 1}: one block sweep, no other pass.
    assert st["gate_passes"] == 1 and st["fused_passes"] == 0
