"""The headline workload at full size: the QFT on 28 qubits of the random-phase
input QuantumState::randomPhase(28, 123456), checked on the whole 4 GiB state
against the reference's own answer (tests/golden/qft28_ref.json, made by
tests/golden/make_qft28_golden.py from the reference compiled from its
sources: Simulator::run of appendQft(28) on the Dense backend).

* plain FP64 form: the output bytes have the reference's SHA-256 (bit for bit,
  every amplitude), the same argmax, total probability and seeded measurement;
* fast FP64 form (TMFQS_OPT_EXACT=0): relative L2 <= 1e-12 against the
  reference (formula of src/tmfqs/experiment/comparison.cpp:59-60, computed on
  the device against the plain result, which is the reference's vector), the
  same argmax and measured index;
* complex64 form: fidelity >= 1 - 1e-6 against the reference.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "qft28_ref.json")


@pytest.fixture(scope="module")
def gold():
    return json.load(open(GOLDEN))


@pytest.fixture(scope="module")
def qft28(gold):
    """The plain result, computed once; kept on the device for the other forms."""
    import torch

    n = gold["n_qubits"]
    inp = tq.random_phase(n, gold["seed"])
    g = tq.GpuState(tq.FP64)
    g.load(n, inp)
    g.apply_ops(tq.qft_ops(n))
    yield n, inp, g
    g.close()
    torch.cuda.empty_cache()


def _argmax(t):
    import torch

    a = t.view(-1, 2).double()
    p = (a * a).sum(dim=1)
    i = int(torch.argmax(p))
    return i, float(p[i])


def test_qft28_plain_is_the_reference_vector(gold, qft28):
    n, _, g = qft28
    rnd = float(tq.mt19937_unit(gold["seed"], 1)[0])
    out = g.export()
    mv = memoryview(out).cast("B")
    chunk = mv.nbytes // len(gold["chunk_sha256"])
    bad = [i for i, d in enumerate(gold["chunk_sha256"]) if hashlib.sha256(mv[i * chunk:(i + 1) * chunk]).hexdigest() != d]
    assert bad == [], f"chunks differing from the reference: {bad}"
    assert hashlib.sha256(mv).hexdigest() == gold["sha256"]
    idx = np.array(gold["sample_indices"], dtype=np.int64)
    got = np.stack([out[2 * idx], out[2 * idx + 1]], axis=1)
    assert got.tolist() == gold["samples"]
    assert _argmax(g.tensor()) == (gold["argmax"], gold["max_probability"])
    assert g.total_probability() == gold["total"]
    assert g.sample(rnd) == gold["measured"]


def _rel_l2(ref, got):
    """sqrt(sum |got - ref|^2 / sum |ref|^2) over interleaved device vectors, FP64 (comparison.cpp:59-60)."""
    num = den = 0.0
    step = 1 << 26
    for i in range(0, ref.numel(), step):
        r = ref[i:i + step].double()
        d = got[i:i + step].double() - r
        num += float((d * d).sum())
        den += float((r * r).sum())
    return (num / den) ** 0.5


def _fidelity(ref, got):
    dre = dim = na = nb = 0.0
    step = 1 << 26
    for i in range(0, ref.numel(), step):
        x = ref[i:i + step].double().view(-1, 2)
        y = got[i:i + step].double().view(-1, 2)
        dre += float((x[:, 0] * y[:, 0] + x[:, 1] * y[:, 1]).sum())
        dim += float((x[:, 0] * y[:, 1] - x[:, 1] * y[:, 0]).sum())
        na += float((x * x).sum())
        nb += float((y * y).sum())
    return (dre * dre + dim * dim) / (na * nb)


@pytest.mark.parametrize("prec,exact", [(tq.FP64, 0), (tq.FP32, 1)])
def test_qft28_fast_forms_against_the_reference(gold, qft28, prec, exact):
    n, inp, plain = qft28
    rnd = float(tq.mt19937_unit(gold["seed"], 1)[0])
    with tq.GpuState(prec) as g:
        g.set_option(tq.OPT_EXACT, exact)
        g.load(n, inp)
        g.apply_ops(tq.qft_ops(n))
        ref_t, got_t = plain.tensor(), g.tensor()
        fid = _fidelity(ref_t, got_t)
        if prec == tq.FP64:
            assert _rel_l2(ref_t, got_t) <= 1e-12
            assert _argmax(got_t)[0] == gold["argmax"]
            assert g.sample(rnd) == gold["measured"]
        assert fid >= 1.0 - 1e-6
        del ref_t, got_t
