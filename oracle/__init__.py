"""CPU oracle for the TMFQS dense path -- test infrastructure only.

Two CPU implementations of the reference algorithm live here:

* ``liboracle.so`` -- the plain-C restatement in ``tmfqs_oracle.c`` (each
  function cites the reference file:line it follows);
* ``_ref/libtmfqs_ref.so`` -- the reference library itself, compiled from its
  own sources by ``ref/Makefile`` (renamed namespace, C wrapper in
  ``ref/ref_capi.cpp``).  It is built wherever the reference sources exist and
  travels with the tree otherwise.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, always as the checker, never as the thing
measured or shipped.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "liboracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libtmfqs_ref.so")
# Where the reference sources are, for building _ref/; unset, the Makefile's own default is used.
REFERENCE_SRC = os.environ.get("TMFQS_REFERENCE_SRC")

OP_H, OP_X, OP_CNOT, OP_CPHASE, OP_SWAP, OP_GATE, OP_PHASE_FLIP, OP_INVERSION = range(8)
ERRORS = {1: IndexError, 2: ValueError, 3: RuntimeError, 4: RuntimeError, 5: MemoryError}
ERROR_NAMES = {0: "ok", 1: "out_of_range", 2: "invalid_argument", 3: "logic_error", 4: "runtime_error", 5: "other"}
PI = 3.14159265358979323846


class Op(ctypes.Structure):
    """One circuit operation; layout of ``or_op`` (tmfqs_oracle.h)."""

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


class _Reg(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint),
        ("N", ctypes.c_uint64),
        ("a", ctypes.POINTER(ctypes.c_double)),
        ("has_sum", ctypes.c_int),
        ("sum_re", ctypes.c_double),
        ("sum_im", ctypes.c_double),
        ("overlay", ctypes.c_int),
        ("scale_re", ctypes.c_double),
        ("scale_im", ctypes.c_double),
        ("bias_re", ctypes.c_double),
        ("bias_im", ctypes.c_double),
    ]


def build() -> None:
    """Compile liboracle.so and, when the reference sources exist, _ref/."""
    extra = [f"REF={REFERENCE_SRC}"] if REFERENCE_SRC else []
    subprocess.run(["make", "-s", "-C", _HERE] + extra, check=True)


_lib = None
_ref = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        dp = ctypes.POINTER(ctypes.c_double)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        rp = ctypes.POINTER(_Reg)
        opp = ctypes.POINTER(Op)
        sig = {
            "or_dense_h": (None, [dp, ctypes.c_uint, ctypes.c_uint]),
            "or_dense_x": (None, [dp, ctypes.c_uint, ctypes.c_uint]),
            "or_dense_cnot": (None, [dp, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint]),
            "or_dense_cphase": (None, [dp, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_double]),
            "or_dense_phase_flip": (None, [dp, ctypes.c_uint64]),
            "or_dense_inversion_mean": (None, [dp, ctypes.c_uint, ctypes.c_double, ctypes.c_double]),
            "or_dense_inversion": (None, [dp, ctypes.c_uint]),
            "or_dense_affine": (None, [dp, ctypes.c_uint] + [ctypes.c_double] * 4),
            "or_dense_total_probability": (ctypes.c_double, [dp, ctypes.c_uint]),
            "or_dense_sample": (ctypes.c_int, [dp, ctypes.c_uint, ctypes.c_double, u64p]),
            "or_dense_gate": (ctypes.c_int, [dp, ctypes.c_uint, dp, ctypes.POINTER(ctypes.c_uint), ctypes.c_uint]),
            "or_dense_amplitude_sum": (None, [dp, ctypes.c_uint, dp, dp]),
            "or_reg_init_basis": (ctypes.c_int, [rp, ctypes.c_uint, ctypes.c_uint64, ctypes.c_double, ctypes.c_double]),
            "or_reg_init_uniform": (ctypes.c_int, [rp, ctypes.c_uint, u64p, ctypes.c_size_t]),
            "or_reg_load": (ctypes.c_int, [rp, ctypes.c_uint, dp]),
            "or_reg_free": (None, [rp]),
            "or_reg_copy": (ctypes.c_int, [rp, rp]),
            "or_reg_apply": (ctypes.c_int, [rp, opp]),
            "or_reg_run": (ctypes.c_int, [rp, opp, ctypes.c_size_t]),
            "or_reg_amplitude": (ctypes.c_int, [rp, ctypes.c_uint64, dp, dp]),
            "or_reg_set_amplitude": (ctypes.c_int, [rp, ctypes.c_uint64, ctypes.c_double, ctypes.c_double]),
            "or_reg_export": (ctypes.c_int, [rp, dp]),
            "or_reg_total_probability": (ctypes.c_double, [rp]),
            "or_reg_measure": (ctypes.c_int, [rp, ctypes.c_double, u64p]),
            "or_reg_inversion_mean": (ctypes.c_int, [rp, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
            "or_qft_op_count": (ctypes.c_size_t, [ctypes.c_uint]),
            "or_build_qft": (ctypes.c_size_t, [ctypes.c_uint, opp]),
            "or_grover_iterations": (ctypes.c_uint, [ctypes.c_uint64, ctypes.c_size_t]),
            "or_build_grover": (ctypes.c_long, [ctypes.c_uint, u64p, ctypes.c_size_t, ctypes.c_int, u64p,
                                                ctypes.POINTER(ctypes.c_size_t), opp]),
            "or_random_phase": (None, [ctypes.c_uint, ctypes.c_uint32, dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> ctypes.CDLL:
    """The compiled reference (oracle/_ref).  Raises if it was never built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} missing: run `make -C oracle` where the reference sources exist")
        R = ctypes.CDLL(REF_SO)
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        opp = ctypes.POINTER(Op)
        szp = ctypes.POINTER(ctypes.c_size_t)
        sig = {
            "ref_last_error": (ctypes.c_char_p, []),
            "ref_reg_new_basis": (vp, [ctypes.c_uint, ctypes.c_uint64]),
            "ref_reg_new_amps": (vp, [ctypes.c_uint, dp]),
            "ref_reg_copy": (vp, [vp]),
            "ref_reg_free": (None, [vp]),
            "ref_reg_init_uniform": (ctypes.c_int, [vp, u64p, ctypes.c_size_t]),
            "ref_reg_apply": (ctypes.c_int, [vp, opp]),
            "ref_reg_run": (ctypes.c_int, [vp, opp, ctypes.c_size_t]),
            "ref_reg_inversion_mean": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
            "ref_reg_set_amplitude": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_double, ctypes.c_double]),
            "ref_reg_amplitude": (ctypes.c_int, [vp, ctypes.c_uint64, dp, dp]),
            "ref_reg_export": (ctypes.c_int, [vp, dp]),
            "ref_reg_total_probability": (ctypes.c_int, [vp, dp]),
            "ref_reg_measure_fixed": (ctypes.c_int, [vp, ctypes.c_double, u64p]),
            "ref_reg_measure_seed": (ctypes.c_int, [vp, ctypes.c_uint32, u64p]),
            "ref_state_new": (vp, [ctypes.c_uint, ctypes.c_int, ctypes.c_uint64, dp, u64p, ctypes.c_size_t,
                                   ctypes.c_uint32]),
            "ref_state_free": (None, [vp]),
            "ref_state_export": (ctypes.c_int, [vp, dp]),
            "ref_sim_run": (ctypes.c_int, [vp, opp, ctypes.c_size_t, dp, dp, ctypes.c_int, ctypes.c_uint32, u64p, dp]),
            "ref_build_qft": (ctypes.c_int, [ctypes.c_uint, opp, ctypes.c_size_t, szp]),
            "ref_build_grover": (ctypes.c_int, [ctypes.c_uint, u64p, ctypes.c_size_t, ctypes.c_int, opp,
                                                ctypes.c_size_t, szp]),
            "ref_grover_iterations": (ctypes.c_uint, [ctypes.c_uint64, ctypes.c_size_t]),
            "ref_mt_unit": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_size_t, dp]),
            "ref_compare": (ctypes.c_int, [ctypes.c_uint, dp, dp, dp, dp, u64p, ctypes.POINTER(ctypes.c_int)]),
            "ref_compare_full": (ctypes.c_int, [ctypes.c_uint, dp, dp, dp, u64p, ctypes.POINTER(ctypes.c_int)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(R, name)
            f.restype = res
            f.argtypes = args
        _ref = R
    return _ref


# --------------------------------------------------------------------------
# helpers
# --------------------------------------------------------------------------

def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def u64ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def op_array(ops) -> ctypes.Array:
    """Convert a list of Op (or tuples) to a ctypes array; keeps GATE buffers alive."""
    arr = (Op * max(1, len(ops)))()
    keep = []
    for i, op in enumerate(ops):
        arr[i] = op
        keep.append(op)
    arr._keep = keep  # type: ignore[attr-defined]
    return arr


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


def inversion(materialized):
    return Op(kind=OP_INVERSION, materialized=1 if materialized else 0)


def gate(matrix: np.ndarray, qubits):
    """matrix: complex (2^k, 2^k); returned Op holds references to its buffers."""
    m = np.ascontiguousarray(np.stack([matrix.real, matrix.imag], axis=-1).reshape(-1), dtype=np.float64)
    q = (ctypes.c_uint * len(qubits))(*qubits)
    op = Op(kind=OP_GATE, matrix=dptr(m), qubits=ctypes.cast(q, ctypes.POINTER(ctypes.c_uint)), k=len(qubits))
    op._buffers = (m, q)  # type: ignore[attr-defined]
    return op


def qft_ops(n: int):
    L = lib()
    cnt = L.or_qft_op_count(n)
    arr = (Op * cnt)()
    L.or_build_qft(n, arr)
    return list(arr)


def grover_ops(n: int, marked, materialized: bool):
    L = lib()
    mk = np.ascontiguousarray(np.array(marked, dtype=np.uint64))
    srt = np.zeros(len(mk), dtype=np.uint64)
    uniq = ctypes.c_size_t(0)
    cnt = L.or_build_grover(n, u64ptr(mk), len(mk), int(materialized), u64ptr(srt), ctypes.byref(uniq), None)
    if cnt < 0:
        raise ValueError("invalid Grover circuit")
    arr = (Op * cnt)()
    L.or_build_grover(n, u64ptr(mk), len(mk), int(materialized), u64ptr(srt), ctypes.byref(uniq), arr)
    return list(arr)


def random_phase(n: int, seed: int) -> np.ndarray:
    out = np.empty(2 << n, dtype=np.float64)
    lib().or_random_phase(n, seed, dptr(out))
    return out


def mt_unit(seed: int, k: int) -> np.ndarray:
    """First k Mt19937RandomSource(seed).nextUnitDouble() values (restatement)."""

    class MT(ctypes.Structure):
        _fields_ = [("mt", ctypes.c_uint32 * 624), ("idx", ctypes.c_int)]

    L = lib()
    L.or_mt_seed.argtypes = [ctypes.POINTER(MT), ctypes.c_uint32]
    L.or_mt_canonical.restype = ctypes.c_double
    L.or_mt_canonical.argtypes = [ctypes.POINTER(MT)]
    g = MT()
    L.or_mt_seed(ctypes.byref(g), seed)
    return np.array([L.or_mt_canonical(ctypes.byref(g)) for _ in range(k)])


def _check(rc):
    if rc:
        raise ERRORS.get(rc, RuntimeError)(ERROR_NAMES.get(rc, str(rc)))


class OracleRegister:
    """QuantumRegister semantics (overlay + cached sum) on the C restatement."""

    def __init__(self, n: int, basis: int = 0, amps: np.ndarray | None = None, uniform=None):
        self._r = _Reg()
        L = lib()
        if amps is not None:
            a = np.ascontiguousarray(amps, dtype=np.float64)
            assert a.size == 2 << n
            _check(L.or_reg_load(ctypes.byref(self._r), n, dptr(a)))
        elif uniform is not None:
            s = np.ascontiguousarray(np.array(uniform, dtype=np.uint64))
            _check(L.or_reg_init_uniform(ctypes.byref(self._r), n, u64ptr(s), len(s)))
        else:
            _check(L.or_reg_init_basis(ctypes.byref(self._r), n, basis, 1.0, 0.0))
        self.n = n

    def __del__(self):
        if getattr(self, "_r", None) is not None and self._r.a:
            lib().or_reg_free(ctypes.byref(self._r))

    def copy(self) -> "OracleRegister":
        other = OracleRegister.__new__(OracleRegister)
        other._r = _Reg()
        other.n = self.n
        _check(lib().or_reg_copy(ctypes.byref(other._r), ctypes.byref(self._r)))
        return other

    @property
    def state(self):
        r = self._r
        return dict(has_sum=bool(r.has_sum), sum=(r.sum_re, r.sum_im), overlay=bool(r.overlay),
                    scale=(r.scale_re, r.scale_im), bias=(r.bias_re, r.bias_im))

    def apply(self, op: Op):
        _check(lib().or_reg_apply(ctypes.byref(self._r), ctypes.byref(op)))

    def run(self, ops):
        arr = op_array(ops)
        _check(lib().or_reg_run(ctypes.byref(self._r), arr, len(ops)))

    def inversion_mean(self, re, im, materialized):
        _check(lib().or_reg_inversion_mean(ctypes.byref(self._r), re, im, int(materialized)))

    def amplitude(self, s):
        re, im = ctypes.c_double(), ctypes.c_double()
        _check(lib().or_reg_amplitude(ctypes.byref(self._r), s, ctypes.byref(re), ctypes.byref(im)))
        return re.value, im.value

    def set_amplitude(self, s, re, im):
        _check(lib().or_reg_set_amplitude(ctypes.byref(self._r), s, re, im))

    def amplitudes(self) -> np.ndarray:
        out = np.empty(2 << self.n, dtype=np.float64)
        _check(lib().or_reg_export(ctypes.byref(self._r), dptr(out)))
        return out

    def raw(self) -> np.ndarray:
        """Backend (pre-overlay) amplitudes."""
        return np.ctypeslib.as_array(self._r.a, shape=(2 << self.n,)).copy()

    def total_probability(self) -> float:
        return lib().or_reg_total_probability(ctypes.byref(self._r))

    def measure(self, rnd: float) -> int:
        out = ctypes.c_uint64()
        _check(lib().or_reg_measure(ctypes.byref(self._r), rnd, ctypes.byref(out)))
        return out.value


class RefRegister:
    """tmfqs::QuantumRegister of the compiled reference (Dense strategy)."""

    def __init__(self, n: int, basis: int = 0, amps: np.ndarray | None = None, handle=None):
        R = ref()
        if handle is not None:
            self._h = handle
        elif amps is not None:
            a = np.ascontiguousarray(amps, dtype=np.float64)
            self._h = R.ref_reg_new_amps(n, dptr(a))
        else:
            self._h = R.ref_reg_new_basis(n, basis)
        if not self._h:
            raise RuntimeError(R.ref_last_error().decode())
        self.n = n

    def __del__(self):
        if getattr(self, "_h", None):
            ref().ref_reg_free(self._h)

    def _rc(self, rc):
        if rc:
            raise ERRORS.get(rc, RuntimeError)(ref().ref_last_error().decode())

    def copy(self):
        return RefRegister(self.n, handle=ref().ref_reg_copy(self._h))

    def init_uniform(self, states):
        s = np.ascontiguousarray(np.array(states, dtype=np.uint64))
        self._rc(ref().ref_reg_init_uniform(self._h, u64ptr(s), len(s)))

    def apply(self, op: Op):
        self._rc(ref().ref_reg_apply(self._h, ctypes.byref(op)))

    def run(self, ops):
        arr = op_array(ops)
        self._rc(ref().ref_reg_run(self._h, arr, len(ops)))

    def inversion_mean(self, re, im, materialized):
        self._rc(ref().ref_reg_inversion_mean(self._h, re, im, int(materialized)))

    def set_amplitude(self, s, re, im):
        self._rc(ref().ref_reg_set_amplitude(self._h, s, re, im))

    def amplitude(self, s):
        re, im = ctypes.c_double(), ctypes.c_double()
        self._rc(ref().ref_reg_amplitude(self._h, s, ctypes.byref(re), ctypes.byref(im)))
        return re.value, im.value

    def amplitudes(self) -> np.ndarray:
        out = np.empty(2 << self.n, dtype=np.float64)
        self._rc(ref().ref_reg_export(self._h, dptr(out)))
        return out

    def total_probability(self) -> float:
        out = ctypes.c_double()
        self._rc(ref().ref_reg_total_probability(self._h, ctypes.byref(out)))
        return out.value

    def measure(self, rnd: float) -> int:
        out = ctypes.c_uint64()
        self._rc(ref().ref_reg_measure_fixed(self._h, rnd, ctypes.byref(out)))
        return out.value

    def measure_seed(self, seed: int) -> int:
        out = ctypes.c_uint64()
        self._rc(ref().ref_reg_measure_seed(self._h, seed, ctypes.byref(out)))
        return out.value


class RefState:
    """state::QuantumState built by the reference's factories."""

    def __init__(self, n, kind="basis", basis=0, amps=None, states=None, seed=0):
        R = ref()
        kinds = {"basis": 0, "amplitudes": 1, "uniform": 2, "random_phase": 3}
        a = np.ascontiguousarray(amps, dtype=np.float64) if amps is not None else None
        s = np.ascontiguousarray(np.array(states, dtype=np.uint64)) if states is not None else None
        self._h = R.ref_state_new(n, kinds[kind], basis, dptr(a) if a is not None else None,
                                  u64ptr(s) if s is not None else None, 0 if s is None else len(s), seed)
        if not self._h:
            raise RuntimeError(R.ref_last_error().decode())
        self.n = n

    def __del__(self):
        if getattr(self, "_h", None):
            ref().ref_state_free(self._h)

    def amplitudes(self) -> np.ndarray:
        out = np.empty(2 << self.n, dtype=np.float64)
        rc = ref().ref_state_export(self._h, dptr(out))
        if rc:
            raise RuntimeError(ref().ref_last_error().decode())
        return out

    def run(self, ops, want_amps=True, seed=None):
        """sim::Simulator(Dense).run; returns dict(amps, total, measured, seconds)."""
        R = ref()
        arr = op_array(ops)
        out = np.empty(2 << self.n, dtype=np.float64) if want_amps else None
        tot = ctypes.c_double()
        meas = ctypes.c_uint64()
        secs = ctypes.c_double()
        rc = R.ref_sim_run(self._h, arr, len(ops), dptr(out) if out is not None else None, ctypes.byref(tot),
                           0 if seed is None else 1, 0 if seed is None else seed, ctypes.byref(meas),
                           ctypes.byref(secs))
        if rc:
            raise ERRORS.get(rc, RuntimeError)(R.ref_last_error().decode())
        return dict(amps=out, total=tot.value, measured=meas.value if seed is not None else None,
                    seconds=secs.value)


def ref_qft_ops(n):
    R = ref()
    cnt = ctypes.c_size_t()
    R.ref_build_qft(n, None, 0, ctypes.byref(cnt))
    arr = (Op * cnt.value)()
    rc = R.ref_build_qft(n, arr, cnt.value, ctypes.byref(cnt))
    if rc:
        raise RuntimeError(R.ref_last_error().decode())
    return list(arr)


def ref_grover_ops(n, marked, materialized):
    R = ref()
    mk = np.ascontiguousarray(np.array(marked, dtype=np.uint64))
    cnt = ctypes.c_size_t()
    rc = R.ref_build_grover(n, u64ptr(mk), len(mk), int(materialized), None, 0, ctypes.byref(cnt))
    if rc:
        raise ERRORS.get(rc, RuntimeError)(R.ref_last_error().decode())
    arr = (Op * cnt.value)()
    R.ref_build_grover(n, u64ptr(mk), len(mk), int(materialized), arr, cnt.value, ctypes.byref(cnt))
    return list(arr)


def ref_mt_unit(seed, k):
    out = np.empty(k, dtype=np.float64)
    rc = ref().ref_mt_unit(seed, k, dptr(out))
    if rc:
        raise RuntimeError(ref().ref_last_error().decode())
    return out


def ref_compare(n, ref_amps, got_amps):
    """experiment::compareStates of the reference: (relL2, maxAbs, worstState, bitwiseEqual)."""
    rl2, mx = ctypes.c_double(), ctypes.c_double()
    worst, bw = ctypes.c_uint64(), ctypes.c_int()
    a = np.ascontiguousarray(ref_amps, dtype=np.float64)
    b = np.ascontiguousarray(got_amps, dtype=np.float64)
    rc = ref().ref_compare(n, dptr(a), dptr(b), ctypes.byref(rl2), ctypes.byref(mx), ctypes.byref(worst),
                           ctypes.byref(bw))
    if rc:
        raise RuntimeError(ref().ref_last_error().decode())
    return rl2.value, mx.value, worst.value, bool(bw.value)


COMPARE_FIELDS = ("bitwise_equal", "max_abs_amplitude_error", "max_abs_component_error", "rmse_amplitude", "rel_l2",
                  "max_abs_probability_error", "total_probability_diff", "worst_state")


def ref_compare_full(n, ref_amps, got_amps) -> dict:
    """Every field of the reference's experiment::compareStates (comparison.cpp:12-62)."""
    out = np.zeros(6)
    worst, bw = ctypes.c_uint64(), ctypes.c_int()
    a = np.ascontiguousarray(ref_amps, dtype=np.float64)
    b = np.ascontiguousarray(got_amps, dtype=np.float64)
    rc = ref().ref_compare_full(n, dptr(a), dptr(b), dptr(out), ctypes.byref(worst), ctypes.byref(bw))
    if rc:
        raise RuntimeError(ref().ref_last_error().decode())
    return {"bitwise_equal": bool(bw.value), "max_abs_amplitude_error": out[0], "max_abs_component_error": out[1],
            "rmse_amplitude": out[2], "rel_l2": out[3], "max_abs_probability_error": out[4],
            "total_probability_diff": out[5], "worst_state": worst.value}


def rel_l2(ref_amps: np.ndarray, got_amps: np.ndarray) -> float:
    """relL2 = sqrt(sum|got-ref|^2 / sum|ref|^2), experiment/comparison.cpp:60."""
    d = got_amps - ref_amps
    den = float(np.dot(ref_amps, ref_amps))
    return 0.0 if den == 0.0 else float(np.sqrt(np.dot(d, d) / den))
