"""tmfqsfullstate_b200 -- B200 dense state-vector engine for TMFQS.

The product is native: ``libtmfqs_b200.so`` (hand-written sm_100a CUDA
kernels behind the C ABI in ``include/tmfqs_b200.h``) and the C++17 host
library that mirrors the reference's ``tmfqs::`` API on top of it
(``host/``: ``QuantumRegister``, ``circuit::Circuit``, ``sim::Simulator`` with
the ``gpu`` storage strategy, and the ``grover``/``groverLazy``/``qftG``
CLIs).  This module is a thin ``ctypes`` binding of the C ABI, used by the
tests, the smoke check and the benchmark.  There is no CPU fallback: if the
shared library is missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtmfqs_b200.so")
HOST_LIB_PATH = os.path.join(HERE, "host", "libtmfqs.so")
BIN_DIR = os.path.join(HERE, "host", "bin")
HEADER = os.path.join(os.path.dirname(HERE), "include", "tmfqs_b200.h")

FP64, FP32 = 0, 1
OP_H, OP_X, OP_CNOT, OP_CPHASE, OP_SWAP, OP_GATE, OP_PHASE_FLIP, OP_INVERSION = range(8)
OPT_FUSION, OPT_FUSED_QUBITS, OPT_GROVER_FUSION = range(3)


class TmfqsError(RuntimeError):
    """A failed C-ABI call; ``status`` is the tmfqs_status code."""

    status = 0


class OutOfRange(TmfqsError, IndexError):
    status = 1


class InvalidArgument(TmfqsError, ValueError):
    status = 2


class LogicError(TmfqsError):
    status = 3


class RuntimeFailure(TmfqsError):
    status = 4


class CudaError(TmfqsError):
    status = 5


class DeviceOutOfMemory(TmfqsError, MemoryError):
    status = 6


_ERRORS = {c.status: c for c in (OutOfRange, InvalidArgument, LogicError, RuntimeFailure, CudaError, DeviceOutOfMemory)}


class Op(ctypes.Structure):
    """tmfqs_op (include/tmfqs_b200.h)."""

    _fields_ = [
        ("kind", ctypes.c_int),
        ("q0", ctypes.c_uint),
        ("q1", ctypes.c_uint),
        ("theta", ctypes.c_double),
        ("state", ctypes.c_uint64),
        ("materialized", ctypes.c_int),
        ("matrix", ctypes.POINTER(ctypes.c_double)),
        ("qubits", ctypes.POINTER(ctypes.c_uint)),
        ("k", ctypes.c_uint),
    ]


class RegisterView(ctypes.Structure):
    """tmfqs_register_view: QuantumRegister's cached sum and affine overlay."""

    _fields_ = [
        ("has_sum", ctypes.c_int),
        ("sum_re", ctypes.c_double),
        ("sum_im", ctypes.c_double),
        ("overlay", ctypes.c_int),
        ("scale_re", ctypes.c_double),
        ("scale_im", ctypes.c_double),
        ("bias_re", ctypes.c_double),
        ("bias_im", ctypes.c_double),
    ]

    @classmethod
    def fresh(cls):
        return cls(0, 0.0, 0.0, 0, 1.0, 0.0, 0.0, 0.0)


class KernelTime(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_uint64), ("ms", ctypes.c_double), ("bytes", ctypes.c_double)]


KT_NAMES = ("fused", "permute", "gate", "reduce", "grover", "adjoint")
OPT_KERNEL_TIMING = 3
OPT_EXACT = 4
OPT_RADIX = 5
OPT_TENSOR = 6
OPT_QFT_PASS = 7


class PassRecord(ctypes.Structure):
    """tmfqs_pass_record: one timed device pass."""

    _fields_ = [("kind", ctypes.c_int), ("op_count", ctypes.c_uint), ("segment", ctypes.c_uint64),
                ("first_op", ctypes.c_uint64), ("ms", ctypes.c_double), ("bytes", ctypes.c_double)]


class StateComparison(ctypes.Structure):
    _fields_ = [("bitwise_equal", ctypes.c_int), ("max_abs_amplitude_error", ctypes.c_double),
                ("max_abs_component_error", ctypes.c_double), ("rmse_amplitude", ctypes.c_double),
                ("rel_l2", ctypes.c_double), ("max_abs_probability_error", ctypes.c_double),
                ("total_probability_diff", ctypes.c_double), ("worst_state", ctypes.c_uint64)]


class Stats(ctypes.Structure):
    _fields_ = [
        ("kernel_launches", ctypes.c_uint64),
        ("fused_passes", ctypes.c_uint64),
        ("gate_passes", ctypes.c_uint64),
        ("reduction_passes", ctypes.c_uint64),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
        ("qft_passes", ctypes.c_uint64),
    ]


# Every entry point declared in include/tmfqs_b200.h, with its signature.
_H = ctypes.c_void_p
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_U64 = ctypes.c_uint64
_U64P = ctypes.POINTER(ctypes.c_uint64)
_UI = ctypes.c_uint
SIGNATURES = {
    "tmfqs_gpu_create": [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_H)],
    "tmfqs_gpu_destroy": [_H],
    "tmfqs_gpu_clone": [_H, ctypes.POINTER(_H)],
    "tmfqs_gpu_last_error": None,
    "tmfqs_gpu_init_zero": [_H, _UI],
    "tmfqs_gpu_init_basis": [_H, _UI, _U64, _D, _D],
    "tmfqs_gpu_init_uniform": [_H, _UI, _U64P, ctypes.c_size_t],
    "tmfqs_gpu_load": [_H, _UI, _DP],
    "tmfqs_gpu_load_chunk": [_H, _U64, _DP, _U64],
    "tmfqs_gpu_export": [_H, _DP],
    "tmfqs_gpu_export_chunk": [_H, _U64, _DP, _U64],
    "tmfqs_gpu_get_amp": [_H, _U64, _DP, _DP],
    "tmfqs_gpu_set_amp": [_H, _U64, _D, _D],
    "tmfqs_gpu_num_qubits": [_H, ctypes.POINTER(_UI)],
    "tmfqs_gpu_precision": [_H, ctypes.POINTER(ctypes.c_int)],
    "tmfqs_gpu_total_probability": [_H, _DP],
    "tmfqs_gpu_sample": [_H, _D, _U64P],
    "tmfqs_gpu_amplitude_sum": [_H, _DP, _DP],
    "tmfqs_gpu_overlay_sum": [_H, _D, _D, _D, _D, _DP, _DP],
    "tmfqs_gpu_overlay_total_probability": [_H, _D, _D, _D, _D, _DP],
    "tmfqs_gpu_overlay_sample": [_H, _D, _D, _D, _D, _D, _U64P],
    "tmfqs_gpu_phase_flip": [_H, _U64],
    "tmfqs_gpu_inversion": [_H],
    "tmfqs_gpu_inversion_mean": [_H, _D, _D],
    "tmfqs_gpu_affine": [_H, _D, _D, _D, _D],
    "tmfqs_gpu_h": [_H, _UI],
    "tmfqs_gpu_x": [_H, _UI],
    "tmfqs_gpu_cphase": [_H, _UI, _UI, _D],
    "tmfqs_gpu_cnot": [_H, _UI, _UI],
    "tmfqs_gpu_gate": [_H, _DP, ctypes.POINTER(_UI), _UI],
    "tmfqs_gpu_swap": [_H, _UI, _UI],
    "tmfqs_gpu_apply_ops": [_H, ctypes.POINTER(Op), ctypes.c_size_t],
    "tmfqs_gpu_grover_run": [_H, ctypes.POINTER(RegisterView), _U64P, ctypes.c_size_t, _U64, ctypes.c_int],
    "tmfqs_gpu_adjoint_gradient": [_H, ctypes.POINTER(Op), ctypes.c_size_t, _U64P, _DP, _UI, ctypes.c_size_t, _DP,
                                   _DP],
    "tmfqs_gpu_compare": [_H, _H, ctypes.POINTER(StateComparison)],
    "tmfqs_gpu_sync": [_H],
    "tmfqs_gpu_stats": [_H, ctypes.POINTER(Stats)],
    "tmfqs_gpu_reset_stats": [_H],
    "tmfqs_gpu_set_option": [_H, ctypes.c_int, ctypes.c_long],
    "tmfqs_gpu_kernel_times": [_H, ctypes.POINTER(KernelTime)],
    "tmfqs_gpu_device_buffer": [_H, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)],
    "tmfqs_gpu_stream": [_H, ctypes.POINTER(ctypes.c_void_p)],
    "tmfqs_random_phase": [_UI, ctypes.c_uint32, _DP],
    "tmfqs_sample_static": [ctypes.c_void_p, ctypes.c_int, _UI, _D, ctypes.c_void_p, _U64P],
    "tmfqs_debug_fail_allocations": [_UI, _UI],
    "tmfqs_gpu_pass_mark": [_H, _U64P],
    "tmfqs_gpu_load_apply_ops": [_H, _UI, _DP, ctypes.c_void_p, ctypes.c_size_t],
    "tmfqs_gpu_pass_log": [_H, ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)],
    "tmfqs_mt19937_unit": [ctypes.c_uint32, _U64, _DP],
    "tmfqs_uniform_states": [_U64, _U64, _U64, _U64, _U64P],
}

_lib = None


def build(jobs: int = 8) -> None:
    """Compile libtmfqs_b200.so and the C++ host library for sm_100a, in-tree."""
    subprocess.run(["make", "-s", "-C", HERE, f"-j{jobs}"], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "host"), f"-j{jobs}"], check=True)


def lib() -> ctypes.CDLL:
    """The loaded C ABI.  Raises if the library was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            if name == "tmfqs_gpu_last_error":
                f.restype = ctypes.c_char_p
                f.argtypes = []
            else:
                f.restype = ctypes.c_int
                f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int):
    if rc:
        msg = lib().tmfqs_gpu_last_error().decode(errors="replace")
        raise _ERRORS.get(rc, TmfqsError)(msg)


def _dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_DP)


# ---- op constructors -------------------------------------------------------

def h(q):
    return Op(kind=OP_H, q0=q)


def x(q):
    return Op(kind=OP_X, q0=q)


def cnot(c, t):
    return Op(kind=OP_CNOT, q0=c, q1=t)


def cphase(c, t, theta):
    return Op(kind=OP_CPHASE, q0=c, q1=t, theta=theta)


def swap(a, b):
    return Op(kind=OP_SWAP, q0=a, q1=b)


def phase_flip(s):
    return Op(kind=OP_PHASE_FLIP, state=s)


def gate(matrix: np.ndarray, qubits):
    m = np.ascontiguousarray(np.stack([np.real(matrix), np.imag(matrix)], axis=-1).reshape(-1), dtype=np.float64)
    q = (ctypes.c_uint * max(1, len(qubits)))(*qubits)
    op = Op(kind=OP_GATE, matrix=_dptr(m), qubits=ctypes.cast(q, ctypes.POINTER(ctypes.c_uint)), k=len(qubits))
    op._buffers = (m, q)  # keep alive
    return op


PI = 3.14159265358979323846  # kPi (reference include/tmfqs/core/constants.h:6)


def qft_ops(n: int):
    """circuit::appendQft (reference src/tmfqs/circuit/circuit.cpp:87-100)."""
    ops = []
    for t in range(n):
        ops.append(h(t))
        for c in range(t + 1, n):
            ops.append(cphase(c, t, PI / float(1 << (c - t))))
    for l in range(n // 2):
        ops.append(swap(l, n - l - 1))
    return ops


def zz_ring_observable(n: int):
    """sum_q Z_q Z_{q+1 mod n} as (masks, weights); qubit q is index bit n-1-q."""
    masks = [(1 << (n - 1 - q)) | (1 << (n - 1 - (q + 1) % n)) for q in range(n)]
    return masks, [1.0] * n


def layered_cphase_ops(n: int, thetas):
    """len(thetas) // n layers of (H on every qubit, then cphase(q, q+1 mod n,
    theta[l, q]) for q = 0..n-1), then a final H layer.  The i-th CPHASE op
    carries thetas[i]."""
    thetas = np.asarray(thetas, dtype=np.float64).reshape(-1, n)
    ops = []
    for layer in thetas:
        ops += [h(q) for q in range(n)]
        ops += [cphase(q, (q + 1) % n, float(layer[q])) for q in range(n)]
    ops += [h(q) for q in range(n)]
    return ops


def uniform_states(seed: int, count: int, lo: int, hi: int) -> np.ndarray:
    """`count` distinct draws of std::uniform_int_distribution<uint64_t>(lo, hi) over std::mt19937_64(seed)."""
    out = np.zeros(max(1, count), dtype=np.uint64)
    _check(lib().tmfqs_uniform_states(seed, count, lo, hi, out.ctypes.data_as(_U64P)))
    return out[:count]


def random_angles(count: int, seed: int) -> np.ndarray:
    """std::uniform_real_distribution<double>(0, 2*pi) over std::mt19937(seed)."""
    return 2.0 * np.arccos(-1.0) * mt19937_unit(seed, count)


def random_phase(n: int, seed: int, out: np.ndarray | None = None) -> np.ndarray:
    """QuantumState::randomPhase(n, seed) input (host, std::mt19937)."""
    if out is None:
        out = np.empty(2 << n, dtype=np.float64)
    _check(lib().tmfqs_random_phase(n, seed, _dptr(out)))
    return out


def mt19937_unit(seed: int, count: int) -> np.ndarray:
    """Mt19937RandomSource(seed).nextUnitDouble() draws."""
    out = np.empty(count, dtype=np.float64)
    _check(lib().tmfqs_mt19937_unit(seed, count, _dptr(out)))
    return out


def sample_static(device_amps: int, precision: int, num_qubits: int, rnd: float, stream: int | None = None) -> int:
    """Exact measurement over a caller-owned device state without any device allocation.

    For callers that cannot let the library allocate: the working tables use a
    fixed 2 MiB device array inside libtmfqs_b200 (num_qubits <= 24); calls
    that overlap on the GPU share it and race.
    """
    out = ctypes.c_uint64()
    _check(lib().tmfqs_sample_static(ctypes.c_void_p(device_amps), precision, num_qubits, rnd,
                                     ctypes.c_void_p(stream) if stream else None, ctypes.byref(out)))
    return out.value


def debug_fail_allocations(skip: int, count: int) -> None:
    """Test hook: after `skip` more device allocations succeed, the next `count`
    fail as out of memory (no device memory is touched); (0, 0) disarms."""
    _check(lib().tmfqs_debug_fail_allocations(skip, count))


def op_array(ops):
    arr = (Op * max(1, len(ops)))()
    for i, op in enumerate(ops):
        arr[i] = op
    arr._keep = list(ops)
    return arr


class GpuState:
    """One register's state vector in HBM (a tmfqs_gpu_state handle)."""

    def __init__(self, precision: int = FP64, device: int = 0, _handle=None):
        self.device = device
        self._h = ctypes.c_void_p()
        if _handle is not None:
            self._h = _handle
        else:
            _check(lib().tmfqs_gpu_create(precision, device, ctypes.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().tmfqs_gpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- lifetime / IO --
    def clone(self) -> "GpuState":
        out = ctypes.c_void_p()
        _check(lib().tmfqs_gpu_clone(self._h, ctypes.byref(out)))
        return GpuState(device=self.device, _handle=out)

    def precision(self) -> int:
        v = ctypes.c_int()
        _check(lib().tmfqs_gpu_precision(self._h, ctypes.byref(v)))
        return v.value

    @property
    def num_qubits(self) -> int:
        v = ctypes.c_uint()
        _check(lib().tmfqs_gpu_num_qubits(self._h, ctypes.byref(v)))
        return v.value

    def init_zero(self, n):
        _check(lib().tmfqs_gpu_init_zero(self._h, n))

    def init_basis(self, n, s=0, amp=(1.0, 0.0)):
        _check(lib().tmfqs_gpu_init_basis(self._h, n, s, amp[0], amp[1]))

    def init_uniform(self, n, states):
        a = np.ascontiguousarray(np.array(states, dtype=np.uint64))
        _check(lib().tmfqs_gpu_init_uniform(self._h, n, a.ctypes.data_as(_U64P), len(a)))

    def load(self, n, amps: np.ndarray):
        a = np.ascontiguousarray(amps, dtype=np.float64)
        if a.size != 2 << n:
            raise ValueError("amplitude buffer size mismatch")
        _check(lib().tmfqs_gpu_load(self._h, n, _dptr(a)))

    def load_chunk(self, first, amps: np.ndarray):
        a = np.ascontiguousarray(amps, dtype=np.float64)
        _check(lib().tmfqs_gpu_load_chunk(self._h, first, _dptr(a), a.size // 2))

    def export(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(2 << self.num_qubits, dtype=np.float64)
        _check(lib().tmfqs_gpu_export(self._h, _dptr(out)))
        return out

    def export_chunk(self, first, count) -> np.ndarray:
        out = np.empty(2 * count, dtype=np.float64)
        _check(lib().tmfqs_gpu_export_chunk(self._h, first, _dptr(out), count))
        return out

    def amplitude(self, s):
        re, im = ctypes.c_double(), ctypes.c_double()
        _check(lib().tmfqs_gpu_get_amp(self._h, s, ctypes.byref(re), ctypes.byref(im)))
        return re.value, im.value

    def set_amplitude(self, s, re, im):
        _check(lib().tmfqs_gpu_set_amp(self._h, s, re, im))

    # -- reductions --
    def total_probability(self) -> float:
        v = ctypes.c_double()
        _check(lib().tmfqs_gpu_total_probability(self._h, ctypes.byref(v)))
        return v.value

    def sample(self, rnd: float) -> int:
        v = ctypes.c_uint64()
        _check(lib().tmfqs_gpu_sample(self._h, rnd, ctypes.byref(v)))
        return v.value

    def amplitude_sum(self):
        re, im = ctypes.c_double(), ctypes.c_double()
        _check(lib().tmfqs_gpu_amplitude_sum(self._h, ctypes.byref(re), ctypes.byref(im)))
        return re.value, im.value

    def overlay_sum(self, scale, bias):
        re, im = ctypes.c_double(), ctypes.c_double()
        _check(lib().tmfqs_gpu_overlay_sum(self._h, scale[0], scale[1], bias[0], bias[1], ctypes.byref(re), ctypes.byref(im)))
        return re.value, im.value

    def overlay_total_probability(self, scale, bias) -> float:
        v = ctypes.c_double()
        _check(lib().tmfqs_gpu_overlay_total_probability(self._h, scale[0], scale[1], bias[0], bias[1], ctypes.byref(v)))
        return v.value

    def overlay_sample(self, scale, bias, rnd) -> int:
        v = ctypes.c_uint64()
        _check(lib().tmfqs_gpu_overlay_sample(self._h, scale[0], scale[1], bias[0], bias[1], rnd, ctypes.byref(v)))
        return v.value

    # -- operations --
    def h(self, q):
        _check(lib().tmfqs_gpu_h(self._h, q))

    def x(self, q):
        _check(lib().tmfqs_gpu_x(self._h, q))

    def cnot(self, c, t):
        _check(lib().tmfqs_gpu_cnot(self._h, c, t))

    def cphase(self, c, t, theta):
        _check(lib().tmfqs_gpu_cphase(self._h, c, t, theta))

    def swap(self, a, b):
        _check(lib().tmfqs_gpu_swap(self._h, a, b))

    def gate(self, matrix: np.ndarray, qubits):
        op = gate(matrix, qubits)
        _check(lib().tmfqs_gpu_gate(self._h, op.matrix, op.qubits, op.k))

    def phase_flip(self, s):
        _check(lib().tmfqs_gpu_phase_flip(self._h, s))

    def inversion(self):
        _check(lib().tmfqs_gpu_inversion(self._h))

    def inversion_mean(self, re, im):
        _check(lib().tmfqs_gpu_inversion_mean(self._h, re, im))

    def affine(self, scale, bias):
        _check(lib().tmfqs_gpu_affine(self._h, scale[0], scale[1], bias[0], bias[1]))

    def apply_ops(self, ops):
        arr = op_array(ops)
        _check(lib().tmfqs_gpu_apply_ops(self._h, arr, len(ops)))

    def grover_run(self, view: RegisterView, marked, iterations: int, materialized: bool) -> RegisterView:
        a = np.ascontiguousarray(np.array(marked, dtype=np.uint64))
        _check(lib().tmfqs_gpu_grover_run(self._h, ctypes.byref(view), a.ctypes.data_as(_U64P), len(a), iterations,
                                          1 if materialized else 0))
        return view

    def adjoint_gradient(self, ops, obs_masks, obs_weights, checkpoint_every: int = 0):
        """Runs `ops` on the current state and returns (E, dE/dtheta) for the
        diagonal observable sum_j w_j Z(m_j): one derivative per CPHASE op, in
        op order.  The handle holds the final state afterwards."""
        arr = op_array(ops)
        m = np.ascontiguousarray(np.array(obs_masks, dtype=np.uint64))
        w = np.ascontiguousarray(np.array(obs_weights, dtype=np.float64))
        if len(m) != len(w):
            raise ValueError("observable masks and weights differ in length")
        nparams = sum(1 for o in ops if o.kind == OP_CPHASE)
        grads = np.zeros(max(1, nparams), dtype=np.float64)
        e = ctypes.c_double()
        _check(lib().tmfqs_gpu_adjoint_gradient(self._h, arr, len(ops), m.ctypes.data_as(_U64P), _dptr(w), len(m),
                                                checkpoint_every, ctypes.byref(e), _dptr(grads)))
        return e.value, grads[:nparams]

    def compare(self, candidate: "GpuState") -> dict:
        """experiment::compareStates(self, candidate) on the device, field for field."""
        out = StateComparison()
        _check(lib().tmfqs_gpu_compare(self._h, candidate._h, ctypes.byref(out)))
        d = {f: getattr(out, f) for f, _ in StateComparison._fields_}
        d["bitwise_equal"] = bool(d["bitwise_equal"])
        return d

    def tensor(self):
        """A torch tensor viewing the handle's device state (interleaved re, im;
        float64 for FP64 handles, float32 for FP32) without a copy.  It is valid
        until the state is re-allocated or the handle closed; queued work on the
        handle's stream must be synchronised before torch reads it."""
        import torch

        self.sync()
        ptr, nbytes = self.device_buffer()
        dt = "<f8" if self.precision() == FP64 else "<f4"
        elem = 8 if dt == "<f8" else 4

        class _View:
            __cuda_array_interface__ = {"shape": (nbytes // elem,), "typestr": dt, "data": (ptr, False), "version": 2}

        return torch.as_tensor(_View(), device=torch.device("cuda", self.device))

    def sync(self):
        _check(lib().tmfqs_gpu_sync(self._h))

    def stats(self) -> dict:
        s = Stats()
        _check(lib().tmfqs_gpu_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def reset_stats(self):
        _check(lib().tmfqs_gpu_reset_stats(self._h))

    def set_option(self, option: int, value: int):
        _check(lib().tmfqs_gpu_set_option(self._h, option, value))

    def kernel_times(self) -> dict:
        arr = (KernelTime * len(KT_NAMES))()
        _check(lib().tmfqs_gpu_kernel_times(self._h, arr))
        return {n: {"launches": arr[i].launches, "ms": arr[i].ms, "bytes": arr[i].bytes} for i, n in enumerate(KT_NAMES)}

    def load_apply_ops(self, n, amps: np.ndarray, ops):
        """load(n, amps) then apply_ops(ops), with the copy overlapped with the first pass."""
        assert amps.dtype == np.float64 and amps.size == 2 << n and amps.flags.c_contiguous
        arr = op_array(ops)
        _check(lib().tmfqs_gpu_load_apply_ops(self._h, n, _dptr(amps), ctypes.cast(arr, ctypes.c_void_p), len(ops)))

    def pass_mark(self) -> int:
        seg = ctypes.c_uint64()
        _check(lib().tmfqs_gpu_pass_mark(self._h, ctypes.byref(seg)))
        return seg.value

    def pass_log(self) -> list:
        """Timed passes since reset_stats (needs OPT_KERNEL_TIMING on while they ran)."""
        n = ctypes.c_size_t()
        _check(lib().tmfqs_gpu_pass_log(self._h, None, 0, ctypes.byref(n)))
        arr = (PassRecord * max(1, n.value))()
        _check(lib().tmfqs_gpu_pass_log(self._h, ctypes.cast(arr, ctypes.c_void_p), n.value, ctypes.byref(n)))
        return [{"kind": KT_NAMES[r.kind], "op_count": r.op_count, "segment": r.segment, "first_op": r.first_op,
                 "ms": r.ms, "bytes": r.bytes} for r in arr[:n.value]]

    def device_buffer(self):
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        _check(lib().tmfqs_gpu_device_buffer(self._h, ctypes.byref(p), ctypes.byref(n)))
        return p.value, n.value

    def stream(self):
        p = ctypes.c_void_p()
        _check(lib().tmfqs_gpu_stream(self._h, ctypes.byref(p)))
        return p.value
