#!/usr/bin/env python3
"""Parameter-shift gradients of the layered controlled-phase circuit from the
reference's own Dense forward (oracle/_ref, the reference compiled from its
sources), for the adjoint-gradient tests: tests/golden/adjoint_ps_n24.json.

Circuit: n=24 qubits from |0...0>, 20 layers of (H on every qubit, then
controlledPhase(q, q+1 mod 24, theta[l, q]) for q = 0..23), then a final H
layer.  Angles: std::uniform_real_distribution<double>(0, 2*pi) over
std::mt19937(123456), in (l, q) order.  Observable E = sum_q <Z_q Z_{q+1 mod 24}>
from the amplitudes.  controlledPhase(theta) = diag(1, 1, 1, e^{i theta}) has
generator |11><11| (eigenvalues 0 and 1), so
    dE/dtheta = [E(theta + pi/2) - E(theta - pi/2)] / 2.
32 angles are sampled (numpy default_rng(2024)).  Each forward takes the
reference several seconds on one core; the script spreads them over a spawn
pool.  Re-run only where the reference sources exist:

    make -C oracle && python tests/golden/make_adjoint_golden.py
"""
import json
import multiprocessing as mp
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

N, LAYERS, SEED, NSAMPLE = 24, 20, 123456, 32


def angles():
    import oracle as O

    return 2.0 * np.arccos(-1.0) * O.ref_mt_unit(SEED, N * LAYERS)


def circuit(thetas):
    import oracle as O

    ops = []
    for layer in np.asarray(thetas).reshape(LAYERS, N):
        ops += [O.h(q) for q in range(N)]
        ops += [O.cphase(q, (q + 1) % N, float(layer[q])) for q in range(N)]
    ops += [O.h(q) for q in range(N)]
    return ops


def zz_ring_diag():
    x = np.arange(1 << N, dtype=np.uint32)
    o = np.zeros(1 << N, dtype=np.float64)
    for q in range(N):
        a, b = N - 1 - q, N - 1 - (q + 1) % N
        o += 1.0 - 2.0 * (((x >> a) ^ (x >> b)) & 1)
    return o


def energy(thetas):
    import oracle as O

    st = O.RefState(N, "basis", basis=0)
    a = st.run(circuit(thetas))["amps"]
    p = a[0::2] ** 2 + a[1::2] ** 2
    return float(np.dot(p, zz_ring_diag()))


def main():
    th = angles()
    idx = sorted(int(i) for i in np.random.default_rng(2024).choice(N * LAYERS, NSAMPLE, replace=False))
    tasks = [th]
    half = np.arccos(-1.0) / 2.0
    for i in idx:
        for s in (+1, -1):
            t = th.copy()
            t[i] += s * half
            tasks.append(t)
    with mp.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
        es = pool.map(energy, tasks)
    e0 = es[0]
    ps = [(es[1 + 2 * k] - es[2 + 2 * k]) / 2.0 for k in range(NSAMPLE)]
    out = {"source": "reference Dense forward (oracle/_ref), parameter-shift rule", "n": N, "layers": LAYERS,
           "seed": SEED, "angles": "2*pi*generate_canonical(mt19937(seed)), (l, q) order", "observable": "sum_q Z_q Z_{q+1 mod n}",
           "expectation": e0, "indices": idx, "thetas": [float(th[i]) for i in idx], "ps_grad": ps}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "adjoint_ps_n24.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, "E =", e0)


if __name__ == "__main__":
    main()
