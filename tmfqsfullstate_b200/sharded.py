"""A state vector sharded over ranks: the host-side plan and its exchange step.

The state of n qubits is split over G = 2^g ranks (one process per GPU) by the
top g bits of the physical index: rank r holds the 2^(n-g) amplitudes whose
physical index is (r << (n-g)) | local.  Qubit q of a circuit starts at
physical bit n-1-q (the reference's qubit 0 = most significant bit,
include/tmfqs/core/types.h:12-13); the layout tracks where each qubit sits as
exchanges move qubits between global (rank) and local bits.

Planning (ShardPlan.plan) turns an op list into steps:

* ``("local", ops, rank_filter)`` -- operations on local qubits only, run on
  every rank's shard as a state of n-g qubits (qubit indices remapped) through
  the device library's own entry points; ``rank_filter`` restricts a step to
  the ranks whose global bits match (controlled phases whose control is a
  global qubit become phase gates on the target there).
* ``("swap", global_bit, local_bit)`` -- before a non-diagonal operation on a
  global qubit, that qubit trades places with a local qubit that the next
  operations do not need: every rank exchanges half of its shard (the half
  whose local bit differs from its own global bit) with the partner rank
  that differs in that global bit.  One send and one receive of 2^(n-g-1)
  amplitudes per rank; no other data moves.
* ``("scale", phase, rank_filter)`` -- a controlled phase on two global qubits
  is a scalar phase on the ranks where both bits are set.

Both rewrites of a controlled phase round exactly as the controlled phase
itself (dense_state_backend.cpp:289-304): the phase gate's product adds exact
zeros to the same rounded complex product, and the scalar is an affine map
with zero bias.  Swaps are relabellings.  So a sharded run gives the same
amplitudes as one device, bit for bit, except possibly the sign of a zero
amplitude.

Reductions (total probability, sums) are per-rank partials combined by an
all-reduce; the CDF of a measurement is an all-gather of the per-rank totals,
then the rank that holds the draw finishes it on its shard.

The exchange goes through torch.distributed: NCCL for device tensors (over
NVLink), gloo for host tensors -- the multi-process tests run it on CPU ranks.
Nothing here computes amplitudes itself: local steps call an applier (the
device library on a GPU).
"""
from __future__ import annotations

import cmath
import dataclasses
from typing import Callable, Sequence

OP_H, OP_X, OP_CNOT, OP_CPHASE, OP_SWAP, OP_GATE, OP_PHASE_FLIP = range(7)


@dataclasses.dataclass
class SOp:
    """One circuit operation (the fields of tmfqs_op that the plan needs)."""

    kind: int
    q0: int = 0
    q1: int = 0
    theta: float = 0.0
    state: int = 0
    matrix: tuple | None = None  # OP_GATE: row-major complex entries
    qubits: tuple | None = None  # OP_GATE: targets, first = most significant


class ShardLayout:
    """Where each logical qubit sits: physical bit position, n-1-q at the start.

    Physical bits >= local_n are global (bit local_n + j is bit j of the rank)."""

    def __init__(self, n: int, world: int):
        g = world.bit_length() - 1
        if world < 1 or (1 << g) != world:
            raise ValueError("the number of ranks must be a power of two")
        if g >= n:
            raise ValueError("more ranks than the state can be split over")
        self.n, self.g, self.world = n, g, world
        self.local_n = n - g
        self.pos = [n - 1 - q for q in range(n)]  # qubit -> physical bit

    def is_global(self, q: int) -> bool:
        return self.pos[q] >= self.local_n

    def local_qubit(self, q: int) -> int:
        """The qubit index of q inside a shard (a state of local_n qubits)."""
        p = self.pos[q]
        assert p < self.local_n
        return self.local_n - 1 - p

    def swap_positions(self, qa: int, qb: int):
        self.pos[qa], self.pos[qb] = self.pos[qb], self.pos[qa]

    def qubit_at(self, p: int) -> int:
        return self.pos.index(p)

    def global_index(self, rank: int, local: int) -> int:
        """The logical basis index of amplitude `local` of rank's shard."""
        phys = (rank << self.local_n) | local
        x = 0
        for q in range(self.n):
            if (phys >> self.pos[q]) & 1:
                x |= 1 << (self.n - 1 - q)
        return x


def global_indices(layout: ShardLayout, rank: int):
    """layout.global_index for every amplitude of rank's shard (numpy, uint64)."""
    import numpy as np

    phys = (np.uint64(rank) << np.uint64(layout.local_n)) | np.arange(1 << layout.local_n, dtype=np.uint64)
    x = np.zeros_like(phys)
    for q in range(layout.n):
        x |= ((phys >> np.uint64(layout.pos[q])) & np.uint64(1)) << np.uint64(layout.n - 1 - q)
    return x


def to_device_ops(ops):
    """Planned local ops as operations of the device library (tmfqs_op)."""
    import numpy as np

    import tmfqsfullstate_b200 as tq

    out = []
    for op in ops:
        if op.kind == OP_H:
            out.append(tq.h(op.q0))
        elif op.kind == OP_X:
            out.append(tq.x(op.q0))
        elif op.kind == OP_CNOT:
            out.append(tq.cnot(op.q0, op.q1))
        elif op.kind == OP_CPHASE:
            out.append(tq.cphase(op.q0, op.q1, op.theta))
        elif op.kind == OP_SWAP:
            out.append(tq.swap(op.q0, op.q1))
        elif op.kind == OP_PHASE_FLIP:
            out.append(tq.phase_flip(op.state))
        else:
            d = int(round(len(op.matrix) ** 0.5))
            out.append(tq.gate(np.array(op.matrix, dtype=complex).reshape(d, d), np.array(op.qubits, dtype=np.uint32)))
    return out


def device_applier(state):
    """apply_local / scale_shard for a rank whose shard is the device state of
    `state` (a GpuState of local_n qubits): the library's fused passes do the
    work; a scalar phase is an affine map with zero bias."""

    def apply_local(shard, ops):
        state.apply_ops(to_device_ops(ops))
        state.sync()

    def scale(shard, ph):
        state.affine((ph.real, ph.imag), (0.0, 0.0))
        state.sync()

    return apply_local, scale


def _op_qubits(op: SOp):
    if op.kind in (OP_H, OP_X):
        return [op.q0]
    if op.kind in (OP_CNOT, OP_CPHASE, OP_SWAP):
        return [op.q0, op.q1]
    if op.kind == OP_GATE:
        return list(op.qubits)
    return []


class ShardPlan:
    """Plans an op list over a ShardLayout (the layout is updated in place)."""

    def __init__(self, layout: ShardLayout):
        self.L = layout

    def _free_local(self, avoid, next_use) -> int:
        """The local physical bit to give up for a global qubit: its qubit is not
        in `avoid`, and among those it is the one a non-diagonal operation needs
        again latest (never, for qubits whose Hadamards are done); bits 0-2 (the
        shard's contiguous rows) only when nothing else is free."""
        L = self.L
        cands = [p for p in range(L.local_n) if L.qubit_at(p) not in avoid]
        if not cands:
            raise ValueError("no local qubit is free for an exchange")
        high = [p for p in cands if p >= 3] or cands
        return max(high, key=lambda p: (next_use(L.qubit_at(p)), p))

    def plan(self, ops: Sequence[SOp]):
        L = self.L
        steps = []
        run = []

        def flush():
            if run:
                steps.append(("local", list(run), None))
                run.clear()

        ops = list(ops)
        # For each qubit, the op indexes that need it local (non-diagonal ops).
        uses = {}
        for i, op in enumerate(ops):
            if op.kind in (OP_H, OP_X, OP_CNOT, OP_GATE):
                for q in _op_qubits(op):
                    uses.setdefault(q, []).append(i)
        cursor = [0]

        def next_use(q):
            for j in uses.get(q, ()):
                if j > cursor[0]:
                    return j
            return len(ops) + 1

        for i, op in enumerate(ops):
            cursor[0] = i
            qs = _op_qubits(op)
            if op.kind == OP_SWAP:
                # A swap of two qubits is a relabelling of their bit positions:
                # no amplitude moves (the reference's three CNOTs permute
                # amplitudes without arithmetic, so this is exact).  Ops already
                # in the run keep the indices they were given.
                L.swap_positions(op.q0, op.q1)
                continue
            if op.kind == OP_PHASE_FLIP:
                flush()
                owner, local = self._locate(op.state)
                steps.append(("local", [SOp(OP_PHASE_FLIP, state=local)], {"rank": owner}))
                continue
            if op.kind == OP_CPHASE and any(L.is_global(q) for q in qs):
                flush()
                c, t = op.q0, op.q1
                gq = [q for q in (c, t) if L.is_global(q)]
                bits = {L.pos[q] - L.local_n: 1 for q in gq}
                if len(gq) == 2:
                    steps.append(("scale", cmath.exp(1j * op.theta), {"bits": bits}))
                else:
                    lq = t if gq[0] == c else c
                    ph = cmath.exp(1j * op.theta)
                    gate = SOp(OP_GATE, matrix=(1, 0, 0, ph), qubits=(L.local_qubit(lq),))
                    steps.append(("local", [gate], {"bits": bits}))
                continue
            # Non-diagonal ops: bring global qubits local first.
            need = [q for q in qs if L.is_global(q)]
            if need:
                flush()
                for q in need:
                    p_local = self._free_local(set(qs), next_use)
                    p_global = L.pos[q]
                    steps.append(("swap", p_global - L.local_n, p_local))
                    L.swap_positions(q, L.qubit_at(p_local))
            run.append(self._to_local(op))
        flush()
        return steps

    def _locate(self, state: int):
        """(rank, local index) of logical basis state `state`."""
        L = self.L
        phys = 0
        for q in range(L.n):
            if (state >> (L.n - 1 - q)) & 1:
                phys |= 1 << L.pos[q]
        return phys >> L.local_n, phys & ((1 << L.local_n) - 1)

    def _to_local(self, op: SOp) -> SOp:
        L = self.L
        if op.kind == OP_GATE:
            return SOp(OP_GATE, matrix=op.matrix, qubits=tuple(L.local_qubit(q) for q in op.qubits))
        return SOp(op.kind, q0=L.local_qubit(op.q0), q1=L.local_qubit(op.q1) if op.kind in (OP_CNOT, OP_CPHASE, OP_SWAP) else 0,
                   theta=op.theta)


def rank_selected(rank: int, filt, local_n: int) -> bool:
    if filt is None:
        return True
    if "rank" in filt:
        return rank == filt["rank"]
    return all(((rank >> j) & 1) == v for j, v in filt["bits"].items())


def exchange_half(shard, rank: int, gbit: int, lbit: int, group=None):
    """Swaps physical bits (global gbit, local lbit) of the sharded state: this
    rank trades the half of its shard whose local bit lbit differs from its
    own global bit with the partner rank (rank ^ (1 << gbit)).  `shard` is a
    1-D tensor of interleaved complex amplitudes [re0, im0, ...] (host or
    device), updated in place."""
    import torch
    import torch.distributed as dist

    partner = rank ^ (1 << gbit)
    mine = (rank >> gbit) & 1
    amps = shard.view(-1, 2)
    n_local = amps.shape[0]
    hi = n_local >> (lbit + 1)
    v = amps.view(hi, 2, 1 << lbit, 2)
    half = v[:, 1 - mine].contiguous()
    recv = torch.empty_like(half)
    reqs = dist.batch_isend_irecv([dist.P2POp(dist.isend, half, partner, group),
                                   dist.P2POp(dist.irecv, recv, partner, group)])
    for r in reqs:
        r.wait()
    v[:, 1 - mine].copy_(recv)


def exchange_half_in_process(shards, gbit: int, lbit: int):
    """exchange_half for all ranks' shards held by one process (one GPU, or the
    host): the same data movement, as plain copies."""
    import torch

    for r in range(len(shards)):
        partner = r ^ (1 << gbit)
        if partner < r:
            continue
        mine = (r >> gbit) & 1
        va = shards[r].view(-1, 2)
        vb = shards[partner].view(-1, 2)
        hi = va.shape[0] >> (lbit + 1)
        a = va.view(hi, 2, 1 << lbit, 2)
        b = vb.view(hi, 2, 1 << lbit, 2)
        tmp = a[:, 1 - mine].clone()
        a[:, 1 - mine].copy_(b[:, mine])
        b[:, mine].copy_(tmp)
        del tmp
    torch.cuda.synchronize() if shards[0].is_cuda else None


def run_sharded(steps, shard, rank: int, local_n: int, apply_local: Callable, scale_shard: Callable, group=None):
    """Executes planned steps on this rank's shard."""
    for st in steps:
        if st[0] == "local":
            if rank_selected(rank, st[2], local_n):
                apply_local(shard, st[1])
        elif st[0] == "swap":
            exchange_half(shard, rank, st[1], st[2], group)
        elif st[0] == "scale":
            if rank_selected(rank, st[2], local_n):
                scale_shard(shard, st[1])
        else:
            raise ValueError(st[0])
