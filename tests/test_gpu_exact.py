"""Parity of the FP64 CUDA path with the oracle, through the C ABI.

Bar: bit-identical amplitudes (np.array_equal; the reference's -0/+0 choices
compare equal), bit-identical totals, identical measured indices.  Sizes are
small enough for the C oracle to finish in seconds.
"""
import itertools

import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu


def rand_state(n, seed, zeros=0.0):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(2 << n)
    if zeros:
        mask = rng.random(1 << n) < zeros
        a.reshape(-1, 2)[mask] = 0.0
    nrm = np.sqrt(np.dot(a, a))
    return a / nrm if nrm else a


@pytest.fixture(scope="module")
def gpu():
    g = tq.GpuState(tq.FP64)
    yield g
    g.close()


def assert_same(a, b, what=""):
    assert a.shape == b.shape
    if not np.array_equal(a, b):
        d = np.flatnonzero(a != b)
        raise AssertionError(f"{what}: {d.size} mismatches, first at {d[0]}: {a[d[0]]!r} vs {b[d[0]]!r}")


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12])
def test_single_qubit_gates_every_qubit(gpu, n):
    L = O.lib()
    a = rand_state(n, 11 + n)
    gpu.load(n, a)
    ref = a.copy()
    for q in range(n):
        gpu.h(q)
        L.or_dense_h(O.dptr(ref), n, q)
        assert_same(gpu.export(), ref, f"H q={q}")
        gpu.x(q)
        L.or_dense_x(O.dptr(ref), n, q)
        assert_same(gpu.export(), ref, f"X q={q}")


@pytest.mark.parametrize("n", [2, 3, 5, 8, 12])
def test_two_qubit_gates_every_pair(gpu, n):
    L = O.lib()
    a = rand_state(n, 21 + n)
    gpu.load(n, a)
    ref = a.copy()
    rng = np.random.default_rng(n)
    for c, t in itertools.permutations(range(n), 2):
        theta = float(rng.uniform(-7, 7))
        gpu.cphase(c, t, theta)
        L.or_dense_cphase(O.dptr(ref), n, c, t, theta)
        gpu.cnot(c, t)
        L.or_dense_cnot(O.dptr(ref), n, c, t)
        if c < t:
            gpu.swap(c, t)
            for cc, tt in ((c, t), (t, c), (c, t)):
                L.or_dense_cnot(O.dptr(ref), n, cc, tt)
    assert_same(gpu.export(), ref, "cphase/cnot/swap sweep")


def test_zero_pairs_and_sparse_states(gpu):
    L = O.lib()
    n = 10
    a = rand_state(n, 5, zeros=0.7)
    gpu.load(n, a)
    ref = a.copy()
    for q in range(n):
        gpu.h(q)
        L.or_dense_h(O.dptr(ref), n, q)
        gpu.cphase((q + 3) % n, q, 0.3 * q + 0.1)
        L.or_dense_cphase(O.dptr(ref), n, (q + 3) % n, q, 0.3 * q + 0.1)
    assert_same(gpu.export(), ref, "sparse H/CP")


@pytest.mark.parametrize("k", [0, 1, 2, 3, 4, 6])
def test_generic_gate(gpu, k):
    n = 9
    rng = np.random.default_rng(100 + k)
    a = rand_state(n, 7 + k)
    for trial in range(3):
        qubits = [int(v) for v in rng.permutation(n)[:k]]
        m = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
        gpu.load(n, a)
        gpu.gate(m, qubits)
        ref = a.copy()
        op = O.gate(m, qubits)
        assert O.lib().or_dense_gate(O.dptr(ref), n, op.matrix, op.qubits, k) == 0
        assert_same(gpu.export(), ref, f"gate k={k} q={qubits}")


def test_flip_inversion_affine(gpu):
    L = O.lib()
    n = 11
    a = rand_state(n, 3)
    gpu.load(n, a)
    ref = a.copy()
    gpu.phase_flip(77)
    L.or_dense_phase_flip(O.dptr(ref), 77)
    gpu.inversion_mean(0.0123, -0.0456)
    L.or_dense_inversion_mean(O.dptr(ref), n, 0.0123, -0.0456)
    gpu.affine((0.3, -0.7), (1e-3, 2e-3))
    L.or_dense_affine(O.dptr(ref), n, 0.3, -0.7, 1e-3, 2e-3)
    gpu.inversion()
    L.or_dense_inversion(O.dptr(ref), n)
    assert_same(gpu.export(), ref, "flip/inversion/affine")


def spike_state(n):
    a = rand_state(n, 4) * 1e-3
    a[2 * ((1 << n) // 3)] = 1.0
    return a


STATES = {
    "gauss": lambda n: rand_state(n, 1),
    "sparse": lambda n: rand_state(n, 2, zeros=0.9),
    "uniform": lambda n: np.tile([2.0 ** (-n / 2), 0.0], 1 << n),
    "spike": spike_state,
    "pow2": lambda n: np.ldexp(1.0, -np.random.default_rng(9).integers(1, 60, 2 << n)).astype(np.float64),
}


@pytest.mark.parametrize("kind", sorted(STATES))
@pytest.mark.parametrize("n", [0, 1, 7, 10, 15, 20])
def test_total_probability_and_sums_bitexact(gpu, kind, n):
    a = np.ascontiguousarray(STATES[kind](n), dtype=np.float64)
    gpu.load(n, a)
    L = O.lib()
    tp = gpu.total_probability()
    assert tp == L.or_dense_total_probability(O.dptr(a), n)
    sr, si = gpu.amplitude_sum()
    rr, ri = O.ctypes.c_double(), O.ctypes.c_double()
    L.or_dense_amplitude_sum(O.dptr(a), n, O.ctypes.byref(rr), O.ctypes.byref(ri))
    assert (sr, si) == (rr.value, ri.value)


@pytest.mark.parametrize("kind", sorted(STATES))
@pytest.mark.parametrize("n", [1, 9, 16, 20])
def test_sample_matches_sequential_cdf(gpu, kind, n):
    a = np.ascontiguousarray(STATES[kind](n), dtype=np.float64)
    gpu.load(n, a)
    L = O.lib()
    total = L.or_dense_total_probability(O.dptr(a), n)
    rng = np.random.default_rng(n)
    rnds = list(rng.random(25) * min(total, 0.999999)) + [0.0]
    # Draws exactly on cumulative values (the ties of `rnd <= cumulative`).
    cum = np.cumsum(a[0::2] ** 2 + a[1::2] ** 2)
    for k in rng.integers(0, 1 << n, 5):
        out = O.ctypes.c_uint64()
        probe = float(cum[k])
        if probe < 1.0:
            rnds.append(probe)
    for r in rnds:
        out = O.ctypes.c_uint64()
        rc = L.or_dense_sample(O.dptr(a), n, r, O.ctypes.byref(out))
        if rc == 0:
            assert gpu.sample(r) == out.value, r
        else:
            with pytest.raises(tq.RuntimeFailure):
                gpu.sample(r)


def test_sample_rejects_bad_draws(gpu):
    gpu.init_basis(3, 0)
    for r in (-0.1, 1.0, float("nan")):
        with pytest.raises(tq.InvalidArgument):
            gpu.sample(r)


@pytest.mark.parametrize("n", [8, 14, 19])
def test_overlay_reductions(gpu, n):
    a = rand_state(n, 31)
    gpu.load(n, a)
    scale, bias = (-0.8, 0.1), (2e-4, -1e-4)
    r = O.OracleRegister(n, amps=a)
    r.inversion_mean(-bias[0] / 2.0, -bias[1] / 2.0, False)  # overlay scale -1, bias = 2*mean
    st = r.state
    scale, bias = st["scale"], st["bias"]
    assert gpu.overlay_total_probability(scale, bias) == r.total_probability()
    tot = r.total_probability()
    for rnd in np.random.default_rng(1).random(10) * min(tot, 0.99):
        assert gpu.overlay_sample(scale, bias, float(rnd)) == r.measure(float(rnd))


def ops_equal_run(gpu, n, a, ops):
    gpu.load(n, a)
    gpu.apply_ops(ops)
    r = O.OracleRegister(n, amps=a)
    r.run([O.Op(kind=o.kind, q0=o.q0, q1=o.q1, theta=o.theta, state=o.state) for o in ops])
    return gpu.export(), r.amplitudes()


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 12, 13, 16])
def test_fused_qft_bitexact(gpu, n):
    a = rand_state(n, 40 + n)
    got, ref = ops_equal_run(gpu, n, a, tq.qft_ops(n))
    assert_same(got, ref, f"QFT n={n}")
    st = gpu.stats()
    assert st["kernel_launches"] > 0


@pytest.mark.parametrize("kind", ["sparse", "pattern", "basis"])
def test_fused_qft_zero_inputs_bitexact(gpu, kind):
    """QFT-16 through the register-stage pass on inputs with exact zeros (all-zero
    pairs skipped by whole warps, zero amplitudes taking no phase), compared bit
    for bit, signs of zeros included."""
    n = 16
    if kind == "sparse":
        a = rand_state(n, 77, zeros=0.7)
    else:
        a = np.zeros(2 << n)
        if kind == "pattern":
            a[0::2 << 4] = 2.0 ** (-(n - 4) / 2)  # uniform over the multiples of 2^4
        else:
            a[2 * 5] = 1.0
    got, ref = ops_equal_run(gpu, n, a, tq.qft_ops(n))
    assert_same(got.view(np.uint64), ref.view(np.uint64), f"QFT-16 {kind} (bits)")


@pytest.mark.parametrize("seed", range(6))
def test_fused_random_circuits_bitexact(gpu, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 15))
    ops = []
    for _ in range(int(rng.integers(5, 80))):
        k = int(rng.integers(0, 6))
        q = [int(v) for v in rng.permutation(n)[:2]]
        if k == 0:
            ops.append(tq.h(q[0]))
        elif k == 1:
            ops.append(tq.x(q[0]))
        elif k == 2:
            ops.append(tq.cnot(q[0], q[1]))
        elif k == 3:
            ops.append(tq.cphase(q[0], q[1], float(rng.uniform(-4, 4))))
        elif k == 4:
            ops.append(tq.swap(q[0], q[1]))
        else:
            ops.append(tq.phase_flip(int(rng.integers(0, 1 << n))))
    a = rand_state(n, seed)
    got, ref = ops_equal_run(gpu, n, a, ops)
    assert_same(got, ref, f"random circuit seed={seed}")


def test_long_diagonal_pass_bitexact(gpu):
    """1500 diagonal ops in one fused pass: its program (84 KB) is larger than
    a pinned upload slot and goes up synchronously; the next batches reuse the
    slots."""
    n = 10
    rng = np.random.default_rng(99)
    ops = [tq.h(q) for q in range(n)]
    for _ in range(1500):
        q = [int(v) for v in rng.permutation(n)[:2]]
        if rng.random() < 0.8:
            ops.append(tq.cphase(q[0], q[1], float(rng.uniform(-4, 4))))
        else:
            ops.append(tq.phase_flip(int(rng.integers(0, 1 << n))))
    ops += [tq.h(q) for q in range(n)]
    a = rand_state(n, 98)
    for rep in range(2):
        got, ref = ops_equal_run(gpu, n, a, ops)
        assert_same(got, ref, f"long diagonal pass, run {rep}")
        small, sref = ops_equal_run(gpu, n, a, tq.qft_ops(n))
        assert_same(small, sref, f"QFT after the long pass, run {rep}")


def test_apply_ops_error_leaves_prefix_applied(gpu):
    n = 4
    a = rand_state(n, 8)
    gpu.load(n, a)
    with pytest.raises(tq.OutOfRange):
        gpu.apply_ops([tq.h(0), tq.h(1), tq.h(9)])
    r = O.OracleRegister(n, amps=a)
    r.run([O.h(0), O.h(1)])
    assert_same(gpu.export(), r.amplitudes(), "prefix")
    with pytest.raises(tq.InvalidArgument):
        gpu.apply_ops([tq.cnot(1, 1)])


@pytest.mark.parametrize("materialized", [True, False])
@pytest.mark.parametrize("n,marked", [(2, [2]), (5, [3]), (10, [1000]), (12, [5, 77, 3000])])
def test_grover_register_semantics(gpu, n, marked, materialized):
    gpu.init_basis(n, 0)
    gpu.apply_ops([tq.h(q) for q in range(n)])
    view = tq.RegisterView.fresh()
    iters = O.lib().or_grover_iterations(1 << n, len(set(marked)))
    gpu.grover_run(view, marked, iters, materialized)
    r = O.OracleRegister(n)
    r.run(O.grover_ops(n, marked, materialized))
    st = r.state
    assert bool(view.has_sum) == st["has_sum"] and (view.sum_re, view.sum_im) == st["sum"]
    assert bool(view.overlay) == st["overlay"]
    if view.overlay:
        assert (view.scale_re, view.scale_im) == st["scale"] and (view.bias_re, view.bias_im) == st["bias"]
    assert_same(gpu.export(), r.raw(), "backend amplitudes")
    tot = r.total_probability()
    if view.overlay:
        g_tot = gpu.overlay_total_probability((view.scale_re, view.scale_im), (view.bias_re, view.bias_im))
    else:
        g_tot = gpu.total_probability()
    assert g_tot == tot


@pytest.mark.parametrize("materialized", [True, False])
def test_grover20_golden(gpu, materialized):
    """grover 20 524287: P(marked), total probability and the seeded measurement."""
    n, s = 20, 524287
    gpu.init_basis(n, 0)
    gpu.apply_ops([tq.h(q) for q in range(n)])
    view = tq.RegisterView.fresh()
    gpu.grover_run(view, [s], 804, materialized)
    re, im = gpu.amplitude(s)
    if view.overlay:
        sc, bi = (view.scale_re, view.scale_im), (view.bias_re, view.bias_im)
        re, im = (sc[0] * re - sc[1] * im) + bi[0], (sc[0] * im + sc[1] * re) + bi[1]
        tot = gpu.overlay_total_probability(sc, bi)
        meas = gpu.overlay_sample(sc, bi, float(O.mt_unit(123456, 1)[0]))
    else:
        tot = gpu.total_probability()
        meas = gpu.sample(float(O.mt_unit(123456, 1)[0]))
    p = re * re + im * im
    if materialized:
        assert p == 0.9999997569653617 and tot == 1.0000000000201612
    else:
        assert p == 0.99999975696536192 and tot == 1.0000000000201614
    assert meas == s


def test_init_io_cache_and_errors(gpu):
    n = 6
    with tq.GpuState(tq.FP64) as g:
        with pytest.raises(tq.LogicError):
            g.h(0)
        g.init_uniform(n, [3, 9, 3, 60])
        r = O.OracleRegister(n, uniform=[3, 9, 3, 60])
        assert_same(g.export(), r.amplitudes(), "uniform")
        with pytest.raises(tq.OutOfRange):
            g.init_uniform(n, [64])
        with pytest.raises(tq.InvalidArgument):
            g.init_uniform(n, [])
        g.init_basis(n, 5, (0.5, -0.25))
        assert g.amplitude(5) == (0.5, -0.25) and g.amplitude(4) == (0.0, 0.0)
        g.set_amplitude(4, 1.0, 2.0)
        g.phase_flip(4)
        assert g.amplitude(4) == (-1.0, -2.0)
        full = g.export()
        assert full[8] == -1.0 and full[9] == -2.0 and full[10] == 0.5
        with pytest.raises(tq.OutOfRange):
            g.amplitude(64)
        with pytest.raises(tq.OutOfRange):
            g.h(6)
        with pytest.raises(tq.InvalidArgument):
            g.cnot(2, 2)
        c = g.clone()
        g.x(0)
        assert_same(c.export(), full, "clone is a deep copy")
        a = rand_state(n, 12)
        g.load(n, a)
        assert_same(g.export_chunk(10, 20), a[20:60], "export chunk")
        g.load_chunk(3, a[100:110])
        b = a.copy()
        b[6:16] = a[100:110]
        assert_same(g.export(), b, "load chunk")
        c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [10, 16, 21])
def test_load_apply_ops_equals_load_then_apply(n):
    """tmfqs_gpu_load_apply_ops (copy in slabs overlapped with the first pass)
    gives the same bytes as load + apply_ops, for the QFT and a circuit whose
    first pass is not a fused pass; and the same error after the same prefix."""
    amps = O.random_phase(n, 40 + n)
    for ops in (tq.qft_ops(n), [tq.swap(0, n - 1), tq.h(1)] + tq.qft_ops(n)):
        with tq.GpuState(tq.FP64) as a, tq.GpuState(tq.FP64) as b:
            a.load_apply_ops(n, amps, ops)
            b.load(n, amps)
            b.apply_ops(ops)
            assert np.array_equal(a.export(), b.export())
            assert a.total_probability() == b.total_probability()
    bad = tq.qft_ops(n)[:5] + [tq.h(n)] + tq.qft_ops(n)
    with tq.GpuState(tq.FP64) as a, tq.GpuState(tq.FP64) as b:
        with pytest.raises(tq.OutOfRange):
            a.load_apply_ops(n, amps, bad)
        b.load(n, amps)
        with pytest.raises(tq.OutOfRange):
            b.apply_ops(bad)
        assert np.array_equal(a.export(), b.export())
    with tq.GpuState(tq.FP32) as a, tq.GpuState(tq.FP32) as b:
        a.load_apply_ops(n, amps, tq.qft_ops(n))
        b.load(n, amps)
        b.apply_ops(tq.qft_ops(n))
        assert np.array_equal(a.export(), b.export())
