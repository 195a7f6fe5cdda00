"""Failure paths of the device backend, injected on the host (no GPU fault):
device out-of-memory through tmfqs_debug_fail_allocations, which makes the
library's next allocation report cudaErrorMemoryAllocation without calling
cudaMalloc.  Each failing call returns TMFQS_ERR_NOMEM (DeviceOutOfMemory in
Python; std::runtime_error through the C++ binding, checked by
bin/test_host_api), leaves the handle usable, and the same call succeeds once
the knob is spent.  Mirrors the reference's convention that resource failures
are std::runtime_error (src/tmfqs/storage/factory/storage_strategy_registry.cpp:99-108).
"""
import numpy as np
import pytest

import oracle as O
import tmfqsfullstate_b200 as tq

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def disarm():
    yield
    tq.debug_fail_allocations(0, 0)


def test_state_allocation_failure_is_reported_and_recoverable():
    with tq.GpuState(tq.FP64) as g:
        tq.debug_fail_allocations(0, 1)
        with pytest.raises(tq.DeviceOutOfMemory):
            g.init_zero(20)
        with pytest.raises(tq.LogicError):
            g.total_probability()  # nothing was initialised
        g.init_basis(20, 0)
        assert g.total_probability() == 1.0


def test_scratch_failure_leaves_the_state_intact():
    n = 12
    amps = O.random_phase(n, 7)
    with tq.GpuState(tq.FP64) as g:
        g.load(n, amps)
        tq.debug_fail_allocations(0, 1)  # the exact-reduction scratch of the first sum
        with pytest.raises(tq.DeviceOutOfMemory):
            g.total_probability()
        reg = O.OracleRegister(n, amps=amps)
        assert g.total_probability() == reg.total_probability()
        assert np.array_equal(g.export(), amps)


def test_clone_failure_keeps_the_original():
    with tq.GpuState(tq.FP64) as g:
        g.init_basis(10, 5)
        tq.debug_fail_allocations(0, 1)
        with pytest.raises(tq.DeviceOutOfMemory):
            g.clone()
        c = g.clone()
        assert c.amplitude(5) == (1.0, 0.0)
        c.close()


def test_pass_program_failure_then_success():
    n = 14
    amps = O.random_phase(n, 3)
    with tq.GpuState(tq.FP64) as g:
        g.load(n, amps)
        tq.debug_fail_allocations(0, 4)
        with pytest.raises(tq.DeviceOutOfMemory):
            g.apply_ops(tq.qft_ops(n))
        tq.debug_fail_allocations(0, 0)
        g.load(n, amps)
        g.apply_ops(tq.qft_ops(n))
        reg = O.OracleRegister(n, amps=amps)
        reg.run(O.qft_ops(n))
        assert np.array_equal(g.export(), reg.amplitudes())
