#!/usr/bin/env python3
"""Generates tests/golden/qft28_ref.json: the whole-state answer of the QFT on
28 qubits, from the reference itself.

Runs the reference library compiled from its sources (oracle/_ref, built by
`make -C oracle`) through its public API: QuantumState::randomPhase(28,
123456) (src/tmfqs/state/quantum_state.cpp:264-277, the qftG input of
examples/qftG.cpp:70-81), then sim::Simulator::run of circuit::appendQft(28)
(src/tmfqs/circuit/circuit.cpp:87-100) on the Dense backend, measured with
Mt19937RandomSource(123456).  The 4 GiB output does not fit in the tree, so it
is summarised by values that pin it completely or by sampling:

  sha256 / input_sha256   digests of the output and input amplitude bytes
  chunk_sha256            digests of the 64 equal chunks of the output
  argmax, max_probability first index of the largest |a|^2 and its value
  norm2                   sum of re^2 + im^2 (numpy pairwise sum)
  samples                 the amplitudes at 256 fixed indices
  total, measured         totalProbability() and measure() of the register

About four minutes of one core and 16 GB of host memory.  Re-run only where the
reference sources exist:

    make -C oracle && python tests/golden/make_qft28_golden.py
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

N_QUBITS = 28
SEED = 123456
CHUNKS = 64


def sample_indices(n: int) -> np.ndarray:
    """256 fixed indices: 0, the top index, and 254 drawn with numpy's PCG64(7)."""
    rng = np.random.default_rng(7)
    idx = rng.integers(0, 1 << n, size=254, dtype=np.uint64)
    return np.unique(np.concatenate([idx, np.array([0, (1 << n) - 1], dtype=np.uint64)]))


def main():
    n = N_QUBITS
    t0 = time.time()
    st = O.RefState(n, "random_phase", seed=SEED)
    inp = st.amplitudes()
    res = st.run(O.ref_qft_ops(n), seed=SEED)
    amps = res["amps"]
    prob = amps[0::2] * amps[0::2] + amps[1::2] * amps[1::2]
    arg = int(np.argmax(prob))
    idx = sample_indices(n)
    chunk = amps.size // CHUNKS
    out = {
        "source": "reference library compiled from its sources (oracle/_ref): QuantumState::randomPhase(28, 123456), "
                  "Simulator::run(appendQft(28)) on the Dense backend, measure(Mt19937RandomSource(123456))",
        "n_qubits": n,
        "seed": SEED,
        "sha256": hashlib.sha256(amps.tobytes()).hexdigest(),
        "input_sha256": hashlib.sha256(inp.tobytes()).hexdigest(),
        "chunk_sha256": [hashlib.sha256(amps[i * chunk:(i + 1) * chunk].tobytes()).hexdigest() for i in range(CHUNKS)],
        "argmax": arg,
        "max_probability": float(prob[arg]),
        "norm2": float(np.sum(prob)),
        "total": res["total"],
        "measured": res["measured"],
        "reference_seconds": res["seconds"],
        "sample_indices": [int(i) for i in idx],
        "samples": [[float(amps[2 * int(i)]), float(amps[2 * int(i) + 1])] for i in idx],
    }
    path = os.path.join(ROOT, "tests", "golden", "qft28_ref.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(f"wrote {path} in {time.time() - t0:.1f} s (reference Simulator {res['seconds']:.1f} s)")


if __name__ == "__main__":
    main()
