"""The adjoint benchmark's inputs on the CPU: the angle stream against the
reference-generated golden fixture (tests/golden/adjoint_ps_n24.json), the
layered circuit's structure and the ring observable."""
import json
import os

import numpy as np

import tmfqsfullstate_b200 as tq

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "adjoint_ps_n24.json")


def test_angles_match_the_reference_stream():
    with open(GOLDEN) as fh:
        gold = json.load(fh)
    th = tq.random_angles(gold["n"] * gold["layers"], gold["seed"])
    assert th.shape == (480,)
    assert np.array_equal(th[gold["indices"]], np.array(gold["thetas"]))
    assert np.all((th >= 0) & (th < 2 * np.pi))


def test_layered_circuit_structure():
    n, layers = 24, 20
    th = tq.random_angles(n * layers, 123456)
    ops = tq.layered_cphase_ops(n, th)
    assert len(ops) == layers * 2 * n + n  # 984 gates
    cp = [o for o in ops if o.kind == tq.OP_CPHASE]
    assert len(cp) == n * layers
    assert [o.theta for o in cp] == list(th)
    for l in range(layers):
        block = ops[l * 2 * n:(l + 1) * 2 * n]
        assert [(o.kind, o.q0) for o in block[:n]] == [(tq.OP_H, q) for q in range(n)]
        assert [(o.q0, o.q1) for o in block[n:]] == [(q, (q + 1) % n) for q in range(n)]
    assert [(o.kind, o.q0) for o in ops[-n:]] == [(tq.OP_H, q) for q in range(n)]


def test_ring_observable():
    n = 24
    masks, weights = tq.zz_ring_observable(n)
    assert weights == [1.0] * n
    for q, m in enumerate(masks):
        assert m == (1 << (n - 1 - q)) | (1 << (n - 1 - (q + 1) % n))
        assert bin(m).count("1") == 2
