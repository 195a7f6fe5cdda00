"""The allocation-free measurement entry point (tmfqs_sample_static).

Some callers cannot let this library call cudaMalloc -- for example an
application whose own caching allocator already holds almost all of the
GPU's memory, or a tight loop that must not pay the device-wide
synchronisation that cudaMalloc/cudaFree bring.  tmfqs_sample_static serves
them: it measures a state that lives in the caller's own device buffer and
keeps its working tables in a fixed 2 MiB array inside the library
(states up to 24 qubits).

This file is collected last so that a run stopping at the first failure has
already run every other test.  It checks the new entry point against the
handle-based tmfqs_gpu_sample on the same states, two calls in a row each
time; the bar is the same as for every measurement test here: the identical
index.
"""
import pytest

import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu


def _prepared_state(n, seed, prec=tq.FP64):
    g = tq.GpuState(prec)
    g.load(n, tq.random_phase(n, seed))
    g.apply_ops(tq.qft_ops(n))
    return g


@pytest.mark.parametrize("prec", [tq.FP64, tq.FP32])
@pytest.mark.parametrize("n", [1, 12, 20, 24])
def test_static_sample_matches_handle_sample_twice_in_a_row(n, prec):
    with _prepared_state(n, 123 + n, prec) as g:
        ptr, nbytes = g.device_buffer()
        assert nbytes == (16 if prec == tq.FP64 else 8) << n
        stream = g.stream()
        draws = [float(v) for v in tq.mt19937_unit(123456 + n, 2)]
        got = [tq.sample_static(ptr, prec, n, r, stream) for r in draws]
        want = [g.sample(r) for r in draws]
        assert got == want


def test_static_sample_reuses_the_array_across_sizes():
    """A big state, then a small one, then the big one again: stale tables must not leak."""
    with _prepared_state(22, 5) as big, _prepared_state(10, 6) as small:
        r = 0.6180339887498949
        first = tq.sample_static(big.device_buffer()[0], tq.FP64, 22, r, big.stream())
        small_idx = tq.sample_static(small.device_buffer()[0], tq.FP64, 10, r, small.stream())
        again = tq.sample_static(big.device_buffer()[0], tq.FP64, 22, r, big.stream())
        assert first == again == big.sample(r)
        assert small_idx == small.sample(r)


def test_static_sample_rejects_oversized_states_and_bad_draws():
    with _prepared_state(4, 1) as g:
        ptr = g.device_buffer()[0]
        with pytest.raises(tq.InvalidArgument, match="24 qubits"):
            tq.sample_static(ptr, tq.FP64, 25, 0.5, g.stream())
        with pytest.raises(tq.InvalidArgument):
            tq.sample_static(ptr, tq.FP64, 4, 1.0, g.stream())
