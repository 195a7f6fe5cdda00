"""Device experiment::compareStates (tmfqs_gpu_compare) against the reference's own.

Every field of the report -- including the three left-to-right FP64 sums
behind rmse, relL2 and the total-probability difference -- must equal the
reference's compareStates (oracle/_ref, the reference compiled from its
sources) on the same amplitudes, bit for bit; candidates in complex64 are
compared through their exact double values.  Without oracle/_ref the sums are
checked against a left-to-right Python restatement of comparison.cpp:12-62.
"""
import math

import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu


def restated(ref, got):
    """comparison.cpp:12-62 in Python floats (IEEE double, left to right)."""
    out = dict(bitwise_equal=True, max_abs_amplitude_error=0.0, max_abs_component_error=0.0,
               max_abs_probability_error=0.0, worst_state=0)
    dn = rn = rt = gt = 0.0
    for s in range(len(ref) // 2):
        rr, ri, gr, gi = float(ref[2 * s]), float(ref[2 * s + 1]), float(got[2 * s]), float(got[2 * s + 1])
        if rr != gr or ri != gi:
            out["bitwise_equal"] = False
        dr, di = gr - rr, gi - ri
        sq = dr * dr + di * di
        e = math.sqrt(sq)
        if e > out["max_abs_amplitude_error"]:
            out["max_abs_amplitude_error"] = e
            out["worst_state"] = s
        out["max_abs_component_error"] = max(out["max_abs_component_error"], max(abs(dr), abs(di)))
        dn += sq
        rn += rr * rr + ri * ri
        pr, pg = rr * rr + ri * ri, gr * gr + gi * gi
        rt += pr
        gt += pg
        out["max_abs_probability_error"] = max(out["max_abs_probability_error"], abs(pg - pr))
    n = len(ref) // 2
    out["rmse_amplitude"] = math.sqrt(dn / n)
    out["rel_l2"] = 0.0 if rn == 0.0 else math.sqrt(dn / rn)
    out["total_probability_diff"] = abs(gt - rt)
    return out


def reference_report(n, a, b):
    if O.ref_available():
        return O.ref_compare_full(n, a, b)
    return restated(a, b)


def cases():
    rng = np.random.default_rng(17)
    for n in (9, 13, 17):
        a = rng.standard_normal(2 << n)
        a /= np.linalg.norm(a)
        yield n, a, a + 1e-7 * rng.standard_normal(2 << n), tq.FP64, "perturbed"
        yield n, a, a.copy(), tq.FP64, "identical"
        yield n, a, a, tq.FP32, "complex64"
        b = a.copy()
        b[2 * 5] += 3e-3  # two states tie for the largest error: the first one counts
        b[2 * 77] += 3e-3
        yield n, a, b, tq.FP64, "tie"


@pytest.mark.parametrize("case", list(cases()), ids=lambda c: f"n{c[0]}-{c[4]}")
def test_compare_matches_reference(case):
    n, a, b, prec_b, _ = case
    with tq.GpuState(tq.FP64) as ga, tq.GpuState(prec_b) as gb:
        ga.load(n, a)
        gb.load(n, b)
        got = ga.compare(gb)
        b_exact = gb.export()  # the candidate's stored values (complex64 rounding included)
    want = reference_report(n, a, b_exact)
    for k in O.COMPARE_FIELDS:
        assert got[k] == want[k], (k, got[k], want[k])


def test_compare_errors():
    with tq.GpuState(tq.FP64) as ga, tq.GpuState(tq.FP64) as gb:
        ga.init_basis(4, 0)
        gb.init_basis(5, 0)
        with pytest.raises(tq.InvalidArgument):
            ga.compare(gb)
