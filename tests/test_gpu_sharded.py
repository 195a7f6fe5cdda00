"""The sharded plan on the GPU, with the ranks emulated in one process.

Four shards of a 20-qubit state are four device states of 18 qubits on the
one GPU; local steps run through the library's fused passes
(sharded.device_applier), exchanges are the same half-shard copies as the
multi-rank path (sharded.exchange_half_in_process; no rank waits on another).
The gathered result must equal the single-device exact result bit for bit
(inputs without zero amplitudes): controlled phases on global qubits become
per-shard phase gates or scalars whose products round exactly as the
controlled phase's own.
"""
import numpy as np
import pytest

import tmfqsfullstate_b200 as tq
from tmfqsfullstate_b200 import sharded as S

pytestmark = pytest.mark.gpu


def _sharded_run(n, world, ops, amps):
    layout = S.ShardLayout(n, world)
    L0 = layout.local_n
    steps = S.ShardPlan(layout).plan(ops)
    states = []
    try:
        for r in range(world):
            g = tq.GpuState(tq.FP64)
            g.load(L0, np.ascontiguousarray(amps[(2 * r) << L0:(2 * (r + 1)) << L0]))
            states.append(g)
        tensors = [g.tensor() for g in states]
        for st in steps:
            if st[0] == "swap":
                S.exchange_half_in_process(tensors, st[1], st[2])
                continue
            for r, g in enumerate(states):
                if not S.rank_selected(r, st[2], L0):
                    continue
                apply_local, scale = S.device_applier(g)
                if st[0] == "local":
                    apply_local(tensors[r], st[1])
                else:
                    scale(tensors[r], st[1])
        got = np.empty(2 << n)
        for r, g in enumerate(states):
            part = g.export().reshape(-1, 2)
            got.reshape(-1, 2)[S.global_indices(layout, r).astype(np.int64)] = part
        return got, sum(1 for s in steps if s[0] == "swap")
    finally:
        for g in states:
            g.close()


def _single(n, ops, amps):
    with tq.GpuState(tq.FP64) as g:
        g.load(n, amps)
        g.apply_ops(S.to_device_ops(ops))
        return g.export()


def test_sharded_qft20_on_four_emulated_ranks():
    n = 20
    amps = tq.random_phase(n, 123456)
    ops = [S.SOp(S.OP_H, t) if c == t else S.SOp(S.OP_CPHASE, c, t, theta=np.pi / float(1 << (c - t)))
           for t in range(n) for c in range(t, n)]
    ops += [S.SOp(S.OP_SWAP, l, n - 1 - l) for l in range(n // 2)]
    got, swaps = _sharded_run(n, 4, ops, amps)
    want = _single(n, ops, amps)
    assert np.array_equal(got, want), float(np.linalg.norm(got - want) / np.linalg.norm(want))
    assert swaps == 3


def test_sharded_random_circuit_is_bit_identical():
    n, world = 18, 4
    rng = np.random.default_rng(9)
    amps = rng.standard_normal(2 << n)
    amps /= np.linalg.norm(amps)
    ops = []
    for _ in range(80):
        k = int(rng.integers(0, 4))
        a, b = (int(v) for v in rng.permutation(n)[:2])
        if k == 0:
            ops.append(S.SOp(S.OP_H, a))
        elif k == 1:
            ops.append(S.SOp(S.OP_CNOT, a, b))
        elif k == 2:
            ops.append(S.SOp(S.OP_CPHASE, a, b, theta=float(rng.uniform(-3, 3))))
        else:
            ops.append(S.SOp(S.OP_SWAP, a, b))
    got, swaps = _sharded_run(n, world, ops, amps)
    assert swaps > 0
    assert np.array_equal(got, _single(n, ops, amps))
