"""The C-ABI library loads and exports every entry point include/tmfqs_b200.h declares."""
import ctypes
import re

import pytest

import tmfqsfullstate_b200 as tq


def declared_symbols():
    text = open(tq.HEADER).read()
    return sorted(set(re.findall(r"TMFQS_API\s+[\w\s\*]+?\b(tmfqs_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 35
    assert "tmfqs_gpu_apply_ops" in names and "tmfqs_gpu_sample" in names


def test_library_exports_every_declared_symbol():
    L = tq.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
        assert name in tq.SIGNATURES, f"binding missing for {name}"


def test_binding_covers_only_declared_symbols():
    assert set(tq.SIGNATURES) == set(declared_symbols())


def test_struct_layouts_match_header():
    # tmfqs_op: int, 2 x unsigned, double, uint64, int, 2 pointers, unsigned.
    assert ctypes.sizeof(tq.Op) == 64
    assert ctypes.sizeof(tq.RegisterView) == 64
    # tmfqs_stats: seven uint64 counters.
    assert ctypes.sizeof(tq.Stats) == 56


def test_create_without_gpu_fails_loudly():
    from tests.conftest import HAS_GPU

    if HAS_GPU:
        pytest.skip("a GPU is present")
    with pytest.raises(tq.CudaError):
        tq.GpuState(tq.FP64)


def test_last_error_is_a_string():
    assert isinstance(tq.lib().tmfqs_gpu_last_error(), bytes)
