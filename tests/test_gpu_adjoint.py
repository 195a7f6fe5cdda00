"""The adjoint gradient (tmfqs_gpu_adjoint_gradient) against the FP64 oracle.

dE/dtheta of E = <psi|O|psi> for a diagonal Z-string observable, with respect
to every controlled-phase angle, checked against
  * central finite differences (h = 1e-6) of the FP64 oracle's forward,
  * the parameter-shift rule on the reference's own Dense forward
    (tests/golden/adjoint_ps_n24.json, made by tests/golden/make_adjoint_golden.py)
    at the full 24-qubit, 20-layer size,
  * torch.autograd through the thin binding in tmfqsfullstate_b200.autograd.
Tolerances: 1e-8 for the complex128 forms; 1e-5 for complex64.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "adjoint_ps_n24.json")


def oracle_op(o):
    if o.kind == tq.OP_H:
        return O.h(o.q0)
    if o.kind == tq.OP_X:
        return O.x(o.q0)
    if o.kind == tq.OP_CNOT:
        return O.cnot(o.q0, o.q1)
    if o.kind == tq.OP_CPHASE:
        return O.cphase(o.q0, o.q1, o.theta)
    if o.kind == tq.OP_SWAP:
        return O.swap(o.q0, o.q1)
    if o.kind == tq.OP_PHASE_FLIP:
        return O.phase_flip(o.state)
    raise ValueError(o.kind)


def diag_values(n, masks, weights):
    x = np.arange(1 << n, dtype=np.uint64)
    o = np.zeros(1 << n)
    for m, w in zip(masks, weights):
        par = np.zeros(1 << n, dtype=np.uint64)
        y = x & np.uint64(m)
        while np.any(y):
            par ^= y & np.uint64(1)
            y >>= np.uint64(1)
        o += w * (1.0 - 2.0 * par.astype(np.float64))
    return o


def energy(n, oracle_ops, o):
    r = O.OracleRegister(n, basis=0)
    r.run(oracle_ops)
    a = r.amplitudes()
    return float(np.dot(a[0::2] ** 2 + a[1::2] ** 2, o))


def fd_grad(n, build, thetas, o, h=1e-6):
    g = np.zeros(len(thetas))
    for i in range(len(thetas)):
        tp, tm = thetas.copy(), thetas.copy()
        tp[i] += h
        tm[i] -= h
        g[i] = (energy(n, build(tp), o) - energy(n, build(tm), o)) / (2 * h)
    return g


def layered_oracle(n):
    return lambda th: [oracle_op(op) for op in tq.layered_cphase_ops(n, th)]


def test_parameter_shift_rule_on_oracle():
    """The shift rule used for the reference fixture equals finite differences (CPU)."""
    n, layers = 6, 2
    th = tq.random_angles(n * layers, 99)
    masks, weights = tq.zz_ring_observable(n)
    o = diag_values(n, masks, weights)
    build = layered_oracle(n)
    fd = fd_grad(n, build, th, o)
    half = np.pi / 2
    for i in range(len(th)):
        tp, tm = th.copy(), th.copy()
        tp[i] += half
        tm[i] -= half
        ps = (energy(n, build(tp), o) - energy(n, build(tm), o)) / 2
        assert abs(ps - fd[i]) < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("prec,exact,tol", [(tq.FP64, 1, 1e-8), (tq.FP64, 0, 1e-8), (tq.FP32, 1, 1e-5)])
def test_adjoint_layered_matches_fd(prec, exact, tol):
    n, layers = 8, 3
    th = tq.random_angles(n * layers, 123456)
    masks, weights = tq.zz_ring_observable(n)
    o = diag_values(n, masks, weights)
    with tq.GpuState(prec) as g:
        g.set_option(tq.OPT_EXACT, exact)
        g.init_basis(n, 0)
        e, grads = g.adjoint_gradient(tq.layered_cphase_ops(n, th), masks, weights, 0)
    assert abs(e - energy(n, layered_oracle(n)(th), o)) < tol
    fd = fd_grad(n, layered_oracle(n), th, o)
    assert grads.shape == (n * layers,)
    assert np.max(np.abs(grads - fd)) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(tq.FP64, 1e-8), (tq.FP32, 1e-4)])
def test_adjoint_more_runs_than_pending_sums(prec, tol):
    """70 diagonal runs: the device-side partial sums are read back mid-call
    (every 64 passes) as well as at the end.  Complex64 over 910 ops: E drifts
    by about 1e-5 (|O| <= 6), hence 1e-4."""
    n, layers = 6, 70
    th = tq.random_angles(n * layers, 77)
    masks, weights = tq.zz_ring_observable(n)
    o = diag_values(n, masks, weights)
    with tq.GpuState(prec) as g:
        g.init_basis(n, 0)
        e, grads = g.adjoint_gradient(tq.layered_cphase_ops(n, th), masks, weights, 0)
    assert abs(e - energy(n, layered_oracle(n)(th), o)) < tol
    fd = fd_grad(n, layered_oracle(n), th, o)
    assert np.max(np.abs(grads - fd)) < tol


@pytest.mark.gpu
def test_adjoint_checkpoint_intervals_agree():
    n, layers = 10, 4
    th = tq.random_angles(n * layers, 5)
    masks, weights = tq.zz_ring_observable(n)
    ops = tq.layered_cphase_ops(n, th)
    res = []
    for every in (1, 7, 2 * n, 10 * n, len(ops), 0):
        with tq.GpuState(tq.FP64) as g:
            g.set_option(tq.OPT_EXACT, 0)
            g.init_basis(n, 0)
            res.append(g.adjoint_gradient(ops, masks, weights, every))
    for e, gr in res[1:]:
        assert abs(e - res[0][0]) < 1e-12
        assert np.max(np.abs(gr - res[0][1])) < 1e-10


@pytest.mark.gpu
def test_adjoint_general_circuit_matches_fd():
    """Every invertible op kind between the controlled phases; weighted single and multi-Z terms."""
    n = 7
    rng = np.random.default_rng(3)
    masks = [0b1, 0b1100000, 0b0010110, 0b1111111]
    weights = [0.7, -1.3, 2.0, 0.25]
    o = diag_values(n, masks, weights)
    u, _ = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
    m = np.empty(32)
    m[0::2], m[1::2] = u.real.ravel(), u.imag.ravel()
    qubits = np.array([2, 5], dtype=np.uint32)
    skeleton = []
    for step in range(40):
        q = [int(v) for v in rng.permutation(n)[:2]]
        kind = int(rng.integers(0, 7))
        skeleton.append((kind, q, int(rng.integers(0, 1 << n))))
    count = sum(1 for k, _, _ in skeleton if k == 3)
    th = rng.uniform(-np.pi, np.pi, count)

    def build(thetas, oracle):
        out, it = [], iter(thetas)
        lib = O if oracle else tq
        for kind, q, s in skeleton:
            if kind == 0:
                out.append(lib.h(q[0]))
            elif kind == 1:
                out.append(lib.x(q[0]))
            elif kind == 2:
                out.append(lib.cnot(q[0], q[1]))
            elif kind == 3:
                out.append(lib.cphase(q[0], q[1], float(next(it))))
            elif kind == 4:
                out.append(lib.swap(q[0], q[1]))
            elif kind == 5:
                out.append(lib.phase_flip(s))
            else:
                out.append(lib.gate(u, [2, 5]) if oracle else tq.gate(u, qubits))
        return out

    with tq.GpuState(tq.FP64) as g:
        g.init_basis(n, 0)
        g.apply_ops([tq.h(q) for q in range(n)])
        e, grads = g.adjoint_gradient(build(th, False), masks, weights, 9)

    def energy_from_plus(thetas):
        r = O.OracleRegister(n, basis=0)
        r.run([O.h(q) for q in range(n)] + build(thetas, True))
        a = r.amplitudes()
        return float(np.dot(a[0::2] ** 2 + a[1::2] ** 2, o))

    assert abs(e - energy_from_plus(th)) < 1e-10
    fd = np.array([(energy_from_plus(np.where(np.arange(count) == i, th + 1e-6, th)) -
                    energy_from_plus(np.where(np.arange(count) == i, th - 1e-6, th))) / 2e-6 for i in range(count)])
    assert np.max(np.abs(grads - fd)) < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("n,prec,tol", [(2, tq.FP64, 1e-8), (2, tq.FP32, 1e-5), (3, tq.FP64, 1e-8),
                                        (12, tq.FP64, 1e-8), (12, tq.FP32, 1e-5)])
def test_adjoint_long_diagonal_runs(n, prec, tol):
    """Diagonal runs of 40, 12 and 20 gates (gradient passes of 32, 8, 12 and 20
    entries: one to four phase tables), phase flips inside the runs, masks on
    the low three bits and above them, and registers of fewer than eight
    amplitudes."""
    rng = np.random.default_rng(17 + n)
    masks, weights = [0b1, (1 << n) - 1, 0b11 << (n - 2)], [0.6, -1.1, 0.9]
    o = diag_values(n, masks, weights)
    skeleton = [(0, [q], 0) for q in range(n)]
    for run_len in (40, 12, 20):
        for _ in range(run_len):
            q = [int(v) for v in rng.permutation(n)[:2]]
            skeleton.append((3 if rng.random() < 0.75 else 5, q, int(rng.integers(0, 1 << n))))
        skeleton += [(0, [int(rng.integers(0, n))], 0), (1, [int(rng.integers(0, n))], 0)]
    count = sum(1 for k, _, _ in skeleton if k == 3)
    th = rng.uniform(-np.pi, np.pi, count)

    def build(thetas, oracle):
        out, it = [], iter(thetas)
        lib = O if oracle else tq
        for kind, q, s in skeleton:
            if kind == 0:
                out.append(lib.h(q[0]))
            elif kind == 1:
                out.append(lib.x(q[0]))
            elif kind == 3:
                out.append(lib.cphase(q[0], q[1], float(next(it))))
            else:
                out.append(lib.phase_flip(s))
        return out

    with tq.GpuState(prec) as g:
        g.init_basis(n, 0)
        e, grads = g.adjoint_gradient(build(th, False), masks, weights, 0)
    assert abs(e - energy(n, build(th, True), o)) < tol
    fd = fd_grad(n, lambda t: build(t, True), th, o)
    assert np.max(np.abs(grads - fd)) < tol


@pytest.mark.gpu
def test_adjoint_torch_autograd():
    import torch

    from tmfqsfullstate_b200.autograd import CircuitExpectation

    n, layers = 6, 2
    masks, weights = tq.zz_ring_observable(n)

    def make_state():
        g = tq.GpuState(tq.FP64)
        g.init_basis(n, 0)
        return g

    th = torch.tensor(tq.random_angles(n * layers, 11), dtype=torch.float64, requires_grad=True)
    e = CircuitExpectation.apply(th, make_state, lambda v: tq.layered_cphase_ops(n, v), masks, weights)
    e.backward()
    o = diag_values(n, masks, weights)
    fd = fd_grad(n, layered_oracle(n), th.detach().numpy().copy(), o)
    assert np.max(np.abs(th.grad.numpy() - fd)) < 1e-8
    f = lambda t: CircuitExpectation.apply(t, make_state, lambda v: tq.layered_cphase_ops(n, v), masks, weights)
    assert torch.autograd.gradcheck(f, (th.detach().clone().requires_grad_(True),), eps=1e-6, atol=1e-6)


@pytest.mark.gpu
def test_adjoint_errors():
    with tq.GpuState(tq.FP64) as g:
        g.init_basis(4, 0)
        with pytest.raises(tq.InvalidArgument):
            g.adjoint_gradient([tq.h(0)], [], [], 0)
        with pytest.raises(tq.OutOfRange):
            g.adjoint_gradient([tq.h(0)], [1 << 4], [1.0], 0)
        with pytest.raises(tq.InvalidArgument):
            g.adjoint_gradient([tq.Op(kind=tq.OP_INVERSION)], [1], [1.0], 0)
        with pytest.raises(tq.InvalidArgument):
            g.adjoint_gradient([tq.cphase(1, 1, 0.3)], [1], [1.0], 0)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(tq.FP32, 1e-5), (tq.FP64, 1e-8)])
def test_adjoint_full_size_matches_reference_parameter_shift(prec, tol):
    """24 qubits, 20 layers, 480 angles; checkpoints every 48 ops (one layer)."""
    gold = json.load(open(GOLDEN))
    n, layers = gold["n"], gold["layers"]
    th = tq.random_angles(n * layers, gold["seed"])
    assert np.allclose(th[gold["indices"]], gold["thetas"], rtol=0, atol=0)
    masks, weights = tq.zz_ring_observable(n)
    with tq.GpuState(prec) as g:
        g.init_basis(n, 0)
        e, grads = g.adjoint_gradient(tq.layered_cphase_ops(n, th), masks, weights, 2 * n)
    assert abs(e - gold["expectation"]) < tol
    err = np.abs(grads[gold["indices"]] - np.array(gold["ps_grad"]))
    assert np.max(err) < tol, err


@pytest.mark.gpu
def test_adjoint_full_size_all_angles_match_fp64_central_differences():
    """24 qubits, 20 layers: the complex64 adjoint gradient on all 480 angles
    against FP64 central differences (h = 1e-6).  The 960 shifted forwards run
    on the GPU in the fast complex128 form (relative L2 <= 1e-12 from the
    reference); E of each is a device dot product of |a|^2 with the diagonal
    of O.  The complex128 adjoint is held to the same differences at 1e-7."""
    import torch

    gold = json.load(open(GOLDEN))
    n, layers = gold["n"], gold["layers"]
    th = tq.random_angles(n * layers, gold["seed"])
    masks, weights = tq.zz_ring_observable(n)
    dev = torch.device("cuda", 0)
    x = torch.arange(1 << n, dtype=torch.int64, device=dev)
    o = torch.zeros(1 << n, dtype=torch.float64, device=dev)
    for m, w in zip(masks, weights):
        par = torch.zeros_like(x)
        for b in range(n):
            if (m >> b) & 1:
                par ^= (x >> b) & 1
        o += w * (1.0 - 2.0 * par.double())
    del x
    grads = {}
    for prec in (tq.FP32, tq.FP64):
        with tq.GpuState(prec) as g:
            g.init_basis(n, 0)
            e, grads[prec] = g.adjoint_gradient(tq.layered_cphase_ops(n, th), masks, weights, 2 * n)
        assert abs(e - gold["expectation"]) < 1e-5
    fd = np.zeros(len(th))
    with tq.GpuState(tq.FP64) as f:
        f.set_option(tq.OPT_EXACT, 0)
        for i in range(len(th)):
            es = []
            for s in (1e-6, -1e-6):
                t = th.copy()
                t[i] += s
                f.init_basis(n, 0)
                f.apply_ops(tq.layered_cphase_ops(n, t))
                a = f.tensor().view(-1, 2)
                es.append(float(((a * a).sum(dim=1) * o).sum()))
            fd[i] = (es[0] - es[1]) / 2e-6
    err32 = np.abs(grads[tq.FP32] - fd)
    err64 = np.abs(grads[tq.FP64] - fd)
    assert np.max(err32) < 1e-5, (int(np.argmax(err32)), float(np.max(err32)))
    assert np.max(err64) < 1e-7, (int(np.argmax(err64)), float(np.max(err64)))
