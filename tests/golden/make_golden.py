#!/usr/bin/env python3
"""Generates tests/golden/golden.json from the reference itself.

Runs the reference library compiled from its sources (oracle/_ref, built by
`make -C oracle`) through its public API and records small known answers for
the dense path: the cases of the reference's own tests
(tests/integration/circuit/test_circuit.cpp, tests/integration/storage/
test_storage_parity.cpp) plus QFT/Grover runs whose outputs are summarised by
exact values and checksums.  Re-run only where the reference sources exist:

    make -C oracle && python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def main():
    g = {"source": "reference library compiled from its sources (oracle/_ref)", "cases": {}}
    c = g["cases"]

    # test_circuit.cpp:76-87, :89-106 -- QFT of |0> and |5> on 3 qubits.
    for s in (0, 5):
        st = O.RefState(3, "basis", basis=s)
        c[f"qft3_basis{s}"] = st.run(O.ref_qft_ops(3))["amps"].tolist()

    # test_circuit.cpp:128-137 / test_storage_parity.cpp:155-164 -- the 8-amplitude fixture.
    fixture = [0.20, 0.10, -0.15, 0.05, 0.30, -0.20, 0.00, 0.10, -0.25, -0.15, 0.18, 0.12, -0.08, 0.04, 0.22, -0.06]
    a = np.array(fixture)
    r = O.RefRegister(3, amps=a)
    mean = (sum(a[0::2]) / 8.0, sum(a[1::2]) / 8.0)
    mr = mi = 0.0
    for k in range(8):
        mr += a[2 * k]
        mi += a[2 * k + 1]
    mean = (mr / 8.0, mi / 8.0)
    r.inversion_mean(mean[0], mean[1], False)
    tot = r.total_probability()
    c["inversion_fixture"] = {
        "amps_in": fixture,
        "mean": list(mean),
        "logical_after_lazy_inversion": r.amplitudes().tolist(),
        "total_probability": tot,
        "measure_half_total": r.measure(tot * 0.5),
    }
    r2 = O.RefRegister(3, amps=a)
    r2.run([O.inversion(False)])
    c["inversion_fixture"]["logical_after_inversion_default"] = r2.amplitudes().tolist()

    # Grover success draws of test_circuit.cpp:102-123, 240-258.
    draws = {}
    for name, n, marked, seeds in (("grover5_3", 5, [3], range(100, 120)), ("grover2_2", 2, [2], range(200, 232)),
                                   ("grover3_1_6", 3, [1, 6], range(300, 332)), ("grover3_2_5_2", 3, [2, 5, 2], range(400, 416))):
        st = O.RefState(n, "basis")
        ops = O.ref_grover_ops(n, marked, False)
        draws[name] = [st.run(ops, want_amps=False, seed=s)["measured"] for s in seeds]
    c["grover_draws"] = draws

    # Random-phase QFT on 12 and 16 qubits: exact totals, measured index, digest.
    for n in (12, 16):
        st = O.RefState(n, "random_phase", seed=123456)
        res = st.run(O.ref_qft_ops(n), seed=123456)
        c[f"qft{n}_random_phase"] = {"total": res["total"], "measured": res["measured"], "amp0": res["amps"][:2].tolist(),
                                     "sha256": digest(res["amps"]), "input_sha256": digest(st.amplitudes())}

    # Grover runs, both diffusion forms.
    for n, marked in ((10, [1000]), (12, [5, 77, 3000])):
        for mat in (True, False):
            st = O.RefState(n, "basis")
            res = st.run(O.ref_grover_ops(n, marked, mat), seed=123456)
            c[f"grover{n}_{'mat' if mat else 'lazy'}"] = {"marked": marked, "total": res["total"],
                                                        "measured": res["measured"], "sha256": digest(res["amps"])}

    c["grover_iterations"] = {"2^20,1": O.ref().ref_grover_iterations(1 << 20, 1),
                              "2^30,4": O.ref().ref_grover_iterations(1 << 30, 4)}
    c["mt19937_123456_first8"] = O.ref_mt_unit(123456, 8).tolist()

    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(out, "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
