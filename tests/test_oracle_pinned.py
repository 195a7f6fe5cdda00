"""The C oracle is pinned to the reference (CPU only, no GPU).

1. Against the committed golden fixtures (tests/golden/golden.json, produced
   by tests/golden/make_golden.py from the reference library itself) --
   these always run.
2. Against the reference library compiled from its sources (oracle/_ref),
   bit for bit, on random circuits -- where that library was built.
"""
import hashlib
import json
import math
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))["cases"]
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def test_qft3_known_answers():
    for s in (0, 5):
        r = O.OracleRegister(3, basis=s)
        r.run(O.qft_ops(3))
        got = r.amplitudes()
        assert got.tolist() == GOLDEN[f"qft3_basis{s}"]
        # The reference test's analytic form, QFT|x> = 8^-1/2 sum_y e^{+2 pi i x y / 8} |y>.
        for y in range(8):
            ang = 2 * math.pi * s * y / 8
            assert abs(got[2 * y] - math.cos(ang) / math.sqrt(8)) < 1e-12
            assert abs(got[2 * y + 1] - math.sin(ang) / math.sqrt(8)) < 1e-12


def test_inversion_fixture():
    fx = GOLDEN["inversion_fixture"]
    a = np.array(fx["amps_in"])
    r = O.OracleRegister(3, amps=a)
    r.inversion_mean(fx["mean"][0], fx["mean"][1], False)
    assert r.amplitudes().tolist() == fx["logical_after_lazy_inversion"]
    assert r.total_probability() == fx["total_probability"]
    assert r.measure(fx["total_probability"] * 0.5) == fx["measure_half_total"]
    r2 = O.OracleRegister(3, amps=a)
    r2.run([O.inversion(False)])
    assert r2.amplitudes().tolist() == fx["logical_after_inversion_default"]


def test_grover_seeded_draws():
    cases = {"grover5_3": (5, [3], range(100, 120)), "grover2_2": (2, [2], range(200, 232)),
             "grover3_1_6": (3, [1, 6], range(300, 332)), "grover3_2_5_2": (3, [2, 5, 2], range(400, 416))}
    for name, (n, marked, seeds) in cases.items():
        ops = O.grover_ops(n, marked, False)
        r = O.OracleRegister(n)
        r.run(ops)
        got = [r.measure(float(O.mt_unit(s, 1)[0])) for s in seeds]
        assert got == GOLDEN["grover_draws"][name], name
    # The reference tests' own assertions on those draws.
    assert all(v == 2 for v in GOLDEN["grover_draws"]["grover2_2"])
    assert all(v in (1, 6) for v in GOLDEN["grover_draws"]["grover3_1_6"])


@pytest.mark.parametrize("n", [12, 16])
def test_random_phase_qft(n):
    g = GOLDEN[f"qft{n}_random_phase"]
    a = O.random_phase(n, 123456)
    assert digest(a) == g["input_sha256"]
    r = O.OracleRegister(n, amps=a)
    r.run(O.qft_ops(n))
    assert digest(r.amplitudes()) == g["sha256"]
    assert r.total_probability() == g["total"]
    assert r.measure(float(O.mt_unit(123456, 1)[0])) == g["measured"]


@pytest.mark.parametrize("name", ["grover10_mat", "grover10_lazy", "grover12_mat", "grover12_lazy"])
def test_grover_runs(name):
    g = GOLDEN[name]
    n = int(name[6:8])
    r = O.OracleRegister(n)
    r.run(O.grover_ops(n, g["marked"], name.endswith("mat")))
    assert digest(r.amplitudes()) == g["sha256"]
    assert r.total_probability() == g["total"]
    assert r.measure(float(O.mt_unit(123456, 1)[0])) == g["measured"]


def test_iteration_counts_and_rng():
    assert O.lib().or_grover_iterations(1 << 20, 1) == GOLDEN["grover_iterations"]["2^20,1"] == 804
    assert O.lib().or_grover_iterations(1 << 30, 4) == GOLDEN["grover_iterations"]["2^30,4"] == 12867
    assert O.mt_unit(123456, 8).tolist() == GOLDEN["mt19937_123456_first8"]


def test_oracle_error_contracts():
    r = O.OracleRegister(2)
    with pytest.raises(IndexError):
        r.apply(O.h(2))
    with pytest.raises(ValueError):
        r.apply(O.cnot(1, 1))
    with pytest.raises(ValueError):
        O.grover_ops(3, [8], True)
    with pytest.raises(ValueError):
        O.OracleRegister(3, uniform=[])


@needs_ref
@pytest.mark.parametrize("seed", range(8))
def test_oracle_matches_reference_random_circuits(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 10))
    a = rng.standard_normal(2 << n)
    a /= np.linalg.norm(a)
    ops = []
    for _ in range(60):
        q = [int(v) for v in rng.permutation(n)[:2]]
        k = int(rng.integers(0, 9))
        if k == 0:
            ops.append(O.h(q[0]))
        elif k == 1:
            ops.append(O.x(q[0]))
        elif k == 2:
            ops.append(O.cnot(*q))
        elif k == 3:
            ops.append(O.cphase(q[0], q[1], float(rng.uniform(-5, 5))))
        elif k == 4:
            ops.append(O.swap(*q))
        elif k == 5:
            ops.append(O.phase_flip(int(rng.integers(0, 1 << n))))
        elif k == 6:
            ops.append(O.inversion(bool(rng.integers(0, 2))))
        else:
            kk = int(rng.integers(1, min(n, 3) + 1))
            m = rng.standard_normal((1 << kk, 1 << kk)) + 1j * rng.standard_normal((1 << kk, 1 << kk))
            ops.append(O.gate(m, [int(v) for v in rng.permutation(n)[:kk]]))
    mine, ref = O.OracleRegister(n, amps=a), O.RefRegister(n, amps=a)
    for op in ops:
        mine.apply(op)
        ref.apply(op)
    assert np.array_equal(mine.amplitudes(), ref.amplitudes())
    assert mine.total_probability() == ref.total_probability()
    for rnd in rng.random(5) * 0.9:
        assert mine.measure(float(rnd)) == ref.measure(float(rnd))


@needs_ref
def test_oracle_matches_reference_inputs_and_builders():
    assert np.array_equal(O.random_phase(11, 99), O.RefState(11, "random_phase", seed=99).amplitudes())
    assert np.array_equal(O.mt_unit(7, 64), O.ref_mt_unit(7, 64))
    for n in (1, 5, 9):
        a, b = O.qft_ops(n), O.ref_qft_ops(n)
        assert [(o.kind, o.q0, o.q1, o.theta) for o in a] == [(o.kind, o.q0, o.q1, o.theta) for o in b]
    a, b = O.grover_ops(6, [9, 3, 9], True), O.ref_grover_ops(6, [9, 3, 9], True)
    assert [(o.kind, o.q0, o.state, o.materialized) for o in a] == [(o.kind, o.q0, o.state, o.materialized) for o in b]


def test_product_input_generator_matches_golden_digests():
    """tmfqs_random_phase (the product's host input generator) against the
    reference's QuantumState::randomPhase (src/tmfqs/state/quantum_state.cpp:264-277),
    through the committed digests of the reference's own inputs."""
    import tmfqsfullstate_b200 as tq

    for n in (12, 16):
        assert digest(tq.random_phase(n, 123456)) == GOLDEN[f"qft{n}_random_phase"]["input_sha256"]


def test_product_input_generator_matches_golden_qft28_digest():
    """The 28-qubit bench input, bit for bit (4 GiB on the host, about 15 s)."""
    import tmfqsfullstate_b200 as tq

    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "qft28_ref.json")))
    assert digest(tq.random_phase(28, gold["seed"])) == gold["input_sha256"]


@needs_ref
@pytest.mark.parametrize("n,seed", [(1, 0), (3, 5), (10, 99), (14, 123456), (17, 4242)])
def test_product_input_generator_matches_reference(n, seed):
    import tmfqsfullstate_b200 as tq

    assert np.array_equal(tq.random_phase(n, seed), O.RefState(n, "random_phase", seed=seed).amplitudes())
    assert np.array_equal(tq.mt19937_unit(seed, 100), O.ref_mt_unit(seed, 100))
