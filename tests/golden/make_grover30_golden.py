#!/usr/bin/env python3
"""Known answers of the 30-qubit, 4-marked-state Grover benchmark from the
reference itself (oracle/_ref, the reference compiled from its sources):
tests/golden/grover30_ref.json.

Marked states: 4 distinct draws of std::uniform_int_distribution<uint64_t>(0,
2^30 - 1) over std::mt19937_64(123456) (tmfqs_uniform_states).  Circuit: the
prefix of circuit::appendGrover(30, marked, materialized) made of the H layer
and the first 10 iterations (phase flips, then inversion about the mean),
run through the reference's Simulator on a Dense register, for both diffusion
forms.  Recorded: each marked amplitude, the total probability and the index
measured with Mt19937RandomSource(123456).  Needs ~40 GB of host memory and a
few minutes on one core per form:

    make -C oracle && python tests/golden/make_grover30_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
import tmfqsfullstate_b200 as tq  # noqa: E402

N, SEED, ITERS = 30, 123456, 10


def main():
    marked = [int(v) for v in tq.uniform_states(SEED, 4, 0, (1 << N) - 1)]
    out = {"source": "reference Dense path (oracle/_ref), Simulator::run", "n": N, "seed": SEED, "marked": marked,
           "iterations": ITERS, "forms": {}}
    for mat in (True, False):
        ops = O.ref_grover_ops(N, marked, mat)
        per_iter = len(sorted(set(marked))) + 1
        ops = ops[:N + ITERS * per_iter]
        st = O.RefState(N, "basis", basis=0)
        res = st.run(ops, want_amps=True, seed=SEED)
        a = res["amps"]
        out["forms"]["materialized" if mat else "lazy"] = {
            "amplitudes": {str(s): [float(a[2 * s]), float(a[2 * s + 1])] for s in marked},
            "total_probability": res["total"], "measured": res["measured"], "seconds": res["seconds"]}
        del a, res, st
        print("form", "materialized" if mat else "lazy", "done", flush=True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "grover30_ref.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
