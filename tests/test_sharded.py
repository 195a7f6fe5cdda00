"""The sharded state's plan and exchange on CPU ranks (gloo), no GPU.

tmfqsfullstate_b200.sharded splits a state over 2^g ranks by the top index
bits, brings global qubits local by pairwise half-shard exchanges, turns
controlled phases on global qubits into per-rank phase gates or scalars, and
relabels swaps.  Here world_size 2 and 4 gloo processes run random circuits
(H, X, CNOT, controlled phases, swaps, 1- and 2-qubit dense gates, phase
flips) with the oracle applying each rank's local steps to its shard; the
gathered state must equal the oracle's whole-state run bit for bit on inputs
without zero amplitudes.  (A controlled phase with a global control becomes
a phase gate diag(1, e^{i theta}) on the ranks where the control is set: the
dense-gate product adds exact zeros to the same rounded complex product, so
only the sign of a zero amplitude could differ.)
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from tmfqsfullstate_b200 import sharded as S


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _to_oracle(op: S.SOp):
    if op.kind == S.OP_H:
        return O.h(op.q0)
    if op.kind == S.OP_X:
        return O.x(op.q0)
    if op.kind == S.OP_CNOT:
        return O.cnot(op.q0, op.q1)
    if op.kind == S.OP_CPHASE:
        return O.cphase(op.q0, op.q1, op.theta)
    if op.kind == S.OP_SWAP:
        return O.swap(op.q0, op.q1)
    if op.kind == S.OP_PHASE_FLIP:
        return O.phase_flip(op.state)
    d = int(round(len(op.matrix) ** 0.5))
    return O.gate(np.array(op.matrix, dtype=complex).reshape(d, d), list(op.qubits))


def random_circuit(n, count, seed, global_phases=True):
    rng = np.random.default_rng(seed)
    ops = []
    for _ in range(count):
        k = int(rng.integers(0, 7))
        a, b = (int(v) for v in rng.permutation(n)[:2])
        if k == 0:
            ops.append(S.SOp(S.OP_H, a))
        elif k == 1:
            ops.append(S.SOp(S.OP_X, a))
        elif k == 2:
            ops.append(S.SOp(S.OP_CNOT, a, b))
        elif k == 3:
            if not global_phases:
                a, b = (int(v) for v in rng.permutation(np.arange(2, n))[:2])
            ops.append(S.SOp(S.OP_CPHASE, a, b, theta=float(rng.uniform(-3, 3))))
        elif k == 4:
            ops.append(S.SOp(S.OP_SWAP, a, b))
        elif k == 5:
            m = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0]
            ops.append(S.SOp(S.OP_GATE, matrix=tuple(m.reshape(-1)), qubits=(a, b)))
        else:
            ops.append(S.SOp(S.OP_PHASE_FLIP, state=int(rng.integers(0, 1 << n))))
    return ops


def qft(n):
    ops = []
    for t in range(n):
        ops.append(S.SOp(S.OP_H, t))
        for c in range(t + 1, n):
            ops.append(S.SOp(S.OP_CPHASE, c, t, theta=np.pi / float(1 << (c - t))))
    for l in range(n // 2):
        ops.append(S.SOp(S.OP_SWAP, l, n - 1 - l))
    return ops


def _worker(rank, world, port, n, case, seed, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(seed)
        full = rng.standard_normal(2 << n)
        full /= np.linalg.norm(full)
        layout = S.ShardLayout(n, world)
        L0 = layout.local_n
        shard = torch.from_numpy(full[(2 * rank) << L0:(2 * (rank + 1)) << L0].copy())
        ops = qft(n) if case == "qft" else random_circuit(n, 60, seed, global_phases=(case != "no_global_phase"))
        steps = S.ShardPlan(layout).plan(ops)

        def apply_local(sh, local_ops):
            reg = O.OracleRegister(L0, amps=sh.numpy())
            reg.run([_to_oracle(o) for o in local_ops])
            sh.copy_(torch.from_numpy(reg.amplitudes()))

        def scale(sh, ph):
            z = sh.view(-1, 2)
            re = z[:, 0] * ph.real - z[:, 1] * ph.imag
            im = z[:, 0] * ph.imag + z[:, 1] * ph.real
            z[:, 0], z[:, 1] = re.clone(), im.clone()

        S.run_sharded(steps, shard, rank, L0, apply_local, scale)
        parts = [torch.empty_like(shard) for _ in range(world)]
        dist.all_gather(parts, shard)
        if rank == 0:
            got = np.empty(2 << n)
            for r in range(world):
                p = parts[r].numpy()
                for loc in range(1 << L0):
                    x = layout.global_index(r, loc)
                    got[2 * x:2 * x + 2] = p[2 * loc:2 * loc + 2]
            reg = O.OracleRegister(n, amps=full)
            reg.run([_to_oracle(o) for o in ops])
            want = reg.amplitudes()
            out.put((bool(np.array_equal(got, want)), O.rel_l2(want, got), sum(1 for s in steps if s[0] == "swap")))
    finally:
        dist.destroy_process_group()


def _run(world, n, case, seed):
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(world, _free_port(), n, case, seed, q), nprocs=world, start_method="spawn", join=True)
    return q.get()


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_random_circuits_without_global_phases_are_exact(world):
    equal, rel, swaps = _run(world, 9, "no_global_phase", 11 + world)
    assert equal, rel
    assert swaps > 0


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_random_circuits(world):
    equal, rel, swaps = _run(world, 9, "random", 21 + world)
    assert equal, rel
    assert swaps > 0


def test_sharded_qft_world4():
    equal, rel, swaps = _run(4, 10, "qft", 5)
    assert equal, rel
    # Each global qubit comes local for its Hadamard; the qubit given up first is
    # one whose Hadamard is still ahead, so one more exchange brings it back.
    # The final swaps are relabellings.
    assert swaps == 3


def test_layout_and_plan_bookkeeping():
    L = S.ShardLayout(6, 4)
    assert (L.g, L.local_n) == (2, 4)
    assert [L.is_global(q) for q in range(6)] == [True, True, False, False, False, False]
    plan = S.ShardPlan(L)
    steps = plan.plan([S.SOp(S.OP_H, 0), S.SOp(S.OP_SWAP, 1, 5), S.SOp(S.OP_CPHASE, 5, 2, theta=0.3),
                       S.SOp(S.OP_PHASE_FLIP, state=0b100001)])
    kinds = [s[0] for s in steps]
    # H(0) brings qubit 0 local for qubit 2 (the only local qubit above the
    # shard's rows); the swap relabels qubits 1 and 5, so the controlled phase
    # joins two global qubits: a scalar on the ranks where both bits are set.
    assert kinds == ["swap", "local", "scale", "local"]
    assert steps[0][1:] == (1, 3)  # qubit 0 is physical bit 5 = rank bit 1
    assert steps[2][2] == {"bits": {L.pos[5] - L.local_n: 1, L.pos[2] - L.local_n: 1}}
    owner, local = plan._locate(0b100001)
    assert steps[3][2] == {"rank": owner} and steps[3][1][0].state == local
    with pytest.raises(ValueError):
        S.ShardLayout(4, 3)
