"""The 30-qubit benchmark configurations at full size.

* Grover search on 30 qubits with 4 marked states (tmfqs_uniform_states: 4
  distinct draws of uniform_int_distribution over mt19937_64(123456)): the
  plain complex128 form reproduces the reference's own amplitudes, total
  probability and seeded measurement after the H layer and 10 iterations
  (tests/golden/grover30_ref.json, made by tests/golden/make_grover30_golden.py
  from the reference compiled from its sources), for both diffusion forms; and
  the complex64 form tracks complex128 over all 12867 iterations (marked-state
  probability within 1e-6, whole-state fidelity >= 1 - 1e-6).
* QFT of the uniform state over k = 0 mod 2^10 on 30 qubits in complex64
  against its analytic answer (2^-5 at multiples of 2^20, 0 elsewhere): the
  largest deviation within 1e-6.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "grover30_ref.json")
N30 = 30


def marked30():
    return [int(v) for v in tq.uniform_states(123456, 4, 0, (1 << N30) - 1)]


def logical(g, view, s):
    re, im = g.amplitude(s)
    if view.overlay:
        re, im = ((view.scale_re * re - view.scale_im * im) + view.bias_re,
                  (view.scale_re * im + view.scale_im * re) + view.bias_im)
    return re, im


@pytest.mark.parametrize("form", ["materialized", "lazy"])
def test_grover30_reference_prefix(form):
    gold = json.load(open(GOLDEN))
    marked = marked30()
    assert marked == gold["marked"]
    ref = gold["forms"][form]
    with tq.GpuState(tq.FP64) as g:
        g.init_basis(N30, 0)
        g.apply_ops([tq.h(q) for q in range(N30)])
        view = tq.RegisterView.fresh()
        g.grover_run(view, marked, gold["iterations"], form == "materialized")
        for s in marked:
            assert list(logical(g, view, s)) == ref["amplitudes"][str(s)], s
        rnd = float(O.mt_unit(123456, 1)[0])
        if view.overlay:
            sc, bi = (view.scale_re, view.scale_im), (view.bias_re, view.bias_im)
            tot, meas = g.overlay_total_probability(sc, bi), g.overlay_sample(sc, bi, rnd)
        else:
            tot, meas = g.total_probability(), g.sample(rnd)
        assert tot == ref["total_probability"]
        assert meas == ref["measured"]


@pytest.mark.parametrize("materialized", [False, True])
def test_grover30_c64_tracks_c128(materialized):
    """All 12867 iterations: the complex64 form's marked-state probability
    within 1e-6 of complex128, and the fidelity of its whole logical state
    (the lazy overlay materialised) >= 1 - 1e-6."""
    import torch

    marked = marked30()
    iters = int(math.floor(math.pi / 4.0 * math.sqrt((1 << N30) / len(marked))))
    assert iters == 12867
    p, held = {}, {}
    try:
        for prec in (tq.FP32, tq.FP64):
            g = tq.GpuState(prec)
            held[prec] = g
            g.init_basis(N30, 0)
            g.apply_ops([tq.h(q) for q in range(N30)])
            view = tq.RegisterView.fresh()
            g.grover_run(view, marked, iters, materialized)
            p[prec] = sum(a * a + b * b for a, b in (logical(g, view, s) for s in marked))
            p[(prec, "u")] = logical(g, view, 12345)  # an unmarked amplitude as well
            if view.overlay:
                g.affine((view.scale_re, view.scale_im), (view.bias_re, view.bias_im))
        assert p[tq.FP64] > 0.999
        assert abs(p[tq.FP32] - p[tq.FP64]) < 1e-6
        assert abs(p[(tq.FP32, "u")][0] - p[(tq.FP64, "u")][0]) < 1e-9
        a, b = held[tq.FP64].tensor(), held[tq.FP32].tensor()
        dre = dim = na = nb = 0.0
        step = 1 << 26
        for i in range(0, a.numel(), step):
            x = a[i:i + step].view(-1, 2)
            y = b[i:i + step].double().view(-1, 2)
            dre += float((x[:, 0] * y[:, 0] + x[:, 1] * y[:, 1]).sum())
            dim += float((x[:, 0] * y[:, 1] - x[:, 1] * y[:, 0]).sum())
            na += float((x * x).sum())
            nb += float((y * y).sum())
        del a, b, x, y
        assert (dre * dre + dim * dim) / (na * nb) >= 1.0 - 1e-6
    finally:
        for g in held.values():
            g.close()
        torch.cuda.empty_cache()


def test_qft30_pattern_known_answer_c64():
    import torch

    n, m = N30, 10
    with tq.GpuState(tq.FP32) as g:
        g.init_uniform(n, np.arange(0, 1 << n, 1 << m, dtype=np.uint64))
        g.apply_ops(tq.qft_ops(n))
        t = g.tensor().view(-1, 2)
        re, im = t[:, 0].double(), t[:, 1]
        idx = torch.arange(1 << n, device=t.device)
        expect = torch.where(idx % (1 << (n - m)) == 0, torch.full_like(re, 2.0 ** (-m / 2)), torch.zeros_like(re))
        err = max(float((re - expect).abs().max()), float(im.abs().max()))
        del t, re, im, idx, expect
    assert err < 1e-6
