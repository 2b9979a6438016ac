"""ctypes front-end of the two oracle legs.  TEST INFRASTRUCTURE ONLY.

* ``KetRef`` drives ``oracle/_ref/libketref.so`` -- the reference's own ket
  headers and bra fused-gate sources compiled unchanged (see oracle/Makefile and
  oracle/ketref_driver.cpp).  ``fast=True`` loads the build with the reference's
  release flags (-Ofast -fopenmp), used as the timed CPU baseline.
* ``COracle`` drives ``oracle/liboracle.so`` -- the project's C restatement
  (oracle/rbk_oracle.c).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs may import
this module, and only as the checker or the timed reference.  Circuits are the
instruction tuples ``(mnemonic, qubits, params)`` produced by
``riken-braket_b200/circuits.py``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

ORC = {
    "H": 1, "X": 2, "Y": 3, "Z": 4, "U1": 5, "U2": 6, "U3": 7, "CNOT": 8, "CZ": 9,
    "U": 10, "EY": 11, "EZ": 12, "SWAP": 13, "BEGIN FUSION": 14, "END FUSION": 15, "EX": 16,
}


class OracleOp(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int32), ("q", ctypes.c_int32 * 2), ("k", ctypes.c_int32),
                ("p", ctypes.c_double * 3)]


def encode(circuit):
    """Instruction tuples -> contiguous array of ``oracle_op`` records."""
    ops = (OracleOp * max(1, len(circuit)))()
    for i, (mnem, qubits, params) in enumerate(circuit):
        op = ops[i]
        op.code = ORC[mnem]
        for j, q in enumerate(qubits[:2]):
            op.q[j] = int(q)
        if mnem == "U":
            op.k = int(params[0])
        else:
            for j, p in enumerate(params[:3]):
                op.p[j] = float(p)
    return ops, len(circuit)


def _pauli_args(terms, n):
    """terms: list of (pauli_string_over_qubits_0..n-1, complex coeff)."""
    strings = b"".join(s.encode() for s, _ in terms)
    assert len(strings) == n * len(terms)
    coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
    return strings, coeffs


class KetRef:
    """The reference's own ket/bra code (oracle/_ref)."""

    def __init__(self, n, initial_index=0, threads=1, fast=False):
        name = "libketref_fast.so" if fast else "libketref.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle)")
        lib = ctypes.CDLL(path)
        lib.ketref_create.restype = ctypes.c_void_p
        lib.ketref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64]
        lib.ketref_destroy.argtypes = [ctypes.c_void_p]
        lib.ketref_apply.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.ketref_apply_timed.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.ketref_apply_timed.restype = ctypes.c_double
        lib.ketref_last_error.restype = ctypes.c_char_p
        for f in ("ketref_set_amplitudes", "ketref_get_amplitudes"):
            getattr(lib, f).argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.ketref_spins.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.ketref_expectation.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p,
                                           ctypes.c_void_p, ctypes.c_void_p]
        lib.ketref_inner_product.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ketref_seed.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        lib.ketref_gate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_void_p]
        lib.ketref_expectation_on.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p]
        lib.ketref_inner_product_on.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p]
        lib.ketref_generate_events.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p]
        lib.ketref_measure.argtypes = [ctypes.c_void_p]
        lib.ketref_measure.restype = ctypes.c_uint64
        lib.ketref_projective_measurement.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self.lib, self.n = lib, n
        self.h = lib.ketref_create(n, threads, initial_index)
        if not self.h:
            raise RuntimeError(lib.ketref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ketref_destroy(self.h)
            self.h = None

    def apply(self, circuit):
        ops, count = encode(circuit)
        if self.lib.ketref_apply(self.h, ops, count) != 0:
            raise RuntimeError(self.lib.ketref_last_error().decode())

    def apply_timed(self, circuit):
        ops, count = encode(circuit)
        t = self.lib.ketref_apply_timed(self.h, ops, count)
        if t < 0:
            raise RuntimeError(self.lib.ketref_last_error().decode())
        return t

    def set_amplitudes(self, amps):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        assert a.size == 1 << self.n
        self.lib.ketref_set_amplitudes(self.h, a.ctypes.data)

    def amplitudes(self):
        out = np.empty(1 << self.n, dtype=np.complex128)
        self.lib.ketref_get_amplitudes(self.h, out.ctypes.data)
        return out

    def spins(self):
        out = np.empty((self.n, 3), dtype=np.float64)
        self.lib.ketref_spins(self.h, out.ctypes.data)
        return out

    def expectation(self, terms):
        strings, coeffs = _pauli_args(terms, self.n)
        out = np.empty(2, dtype=np.float64)
        self.lib.ketref_expectation(self.h, len(terms), strings, coeffs.ctypes.data, out.ctypes.data)
        return complex(out[0], out[1])

    def inner_product(self, other):
        """ket::inner_product(self, other) = <other|self>."""
        out = np.empty(2, dtype=np.float64)
        self.lib.ketref_inner_product(self.h, other.h, out.ctypes.data)
        return complex(out[0], out[1])

    def seed(self, seed):
        self.lib.ketref_seed(self.h, seed)

    def gate(self, kind, targets=(), controls=(), params=(0.0, 0.0, 0.0)):
        """One gate of bra's wider instruction set (kinds KG_* of oracle_ops.h),
        dispatched as bra::nompi_state does."""
        t = np.ascontiguousarray(list(targets) or [0], dtype=np.int32)
        c = np.ascontiguousarray(list(controls) or [0], dtype=np.int32)
        p = np.zeros(3, dtype=np.float64)
        p[:len(params)] = params
        if self.lib.ketref_gate(self.h, kind, len(targets), t.ctypes.data, len(controls), c.ctypes.data, p.ctypes.data) != 0:
            raise RuntimeError(self.lib.ketref_last_error().decode())

    def expectation_on(self, pauli, qubits):
        """bra's EXPECTATION :PAULIS:<pauli> q_0 ... (character k acts on qubits[k])."""
        q = np.ascontiguousarray(list(qubits), dtype=np.int32)
        out = np.empty(2, dtype=np.float64)
        self.lib.ketref_expectation_on(self.h, pauli.encode(), len(qubits), q.ctypes.data, out.ctypes.data)
        return complex(out[0], out[1])

    def inner_product_on(self, other, pauli, qubits):
        """<other| P |self> with the Pauli string `pauli` on `qubits` (bra's INNERPROD n :PAULIS:<pauli> q ...)."""
        q = np.ascontiguousarray(list(qubits), dtype=np.int32)
        out = np.empty(2, dtype=np.float64)
        self.lib.ketref_inner_product_on(self.h, other.h, pauli.encode(), len(qubits), q.ctypes.data, out.ctypes.data)
        return complex(out[0], out[1])

    def generate_events(self, num, seed=-1):
        """Like the reference, this overwrites the amplitudes with prefix sums."""
        out = np.empty(num, dtype=np.uint64)
        self.lib.ketref_generate_events(self.h, num, seed, out.ctypes.data)
        return out

    def measure(self):
        return int(self.lib.ketref_measure(self.h))

    def projective_measurement(self, q):
        return int(self.lib.ketref_projective_measurement(self.h, q))


class COracle:
    """The project's C restatement (oracle/rbk_oracle.c)."""

    def __init__(self, n, initial_index=0):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle liboracle.so)")
        lib = ctypes.CDLL(path)
        lib.orc_create.restype = ctypes.c_void_p
        lib.orc_create.argtypes = [ctypes.c_int, ctypes.c_uint64]
        lib.orc_destroy.argtypes = [ctypes.c_void_p]
        lib.orc_apply.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        for f in ("orc_set_amplitudes", "orc_get_amplitudes", "orc_spins", "orc_probabilities"):
            getattr(lib, f).argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.orc_expectation.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
        lib.orc_inner_product.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.orc_seed.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        lib.orc_generate_events.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p]
        lib.orc_projective_measurement.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.orc_measure.argtypes = [ctypes.c_void_p]
        lib.orc_measure.restype = ctypes.c_uint64
        self.lib, self.n = lib, n
        self.h = lib.orc_create(n, initial_index)
        if not self.h:
            raise MemoryError("orc_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def apply(self, circuit):
        ops, count = encode(circuit)
        if self.lib.orc_apply(self.h, ops, count) != 0:
            raise ValueError("oracle: unsupported instruction")

    def set_amplitudes(self, amps):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        assert a.size == 1 << self.n
        self.lib.orc_set_amplitudes(self.h, a.ctypes.data)

    def amplitudes(self):
        out = np.empty(1 << self.n, dtype=np.complex128)
        self.lib.orc_get_amplitudes(self.h, out.ctypes.data)
        return out

    def probabilities(self):
        out = np.empty(1 << self.n, dtype=np.float64)
        self.lib.orc_probabilities(self.h, out.ctypes.data)
        return out

    def spins(self):
        out = np.empty((self.n, 3), dtype=np.float64)
        self.lib.orc_spins(self.h, out.ctypes.data)
        return out

    def expectation(self, terms):
        strings, coeffs = _pauli_args(terms, self.n)
        out = np.empty(2, dtype=np.float64)
        self.lib.orc_expectation(self.h, len(terms), strings, coeffs.ctypes.data, out.ctypes.data)
        return complex(out[0], out[1])

    def inner_product(self, other):
        """<other|self>, the ket::inner_product(self, other) convention."""
        out = np.empty(2, dtype=np.float64)
        self.lib.orc_inner_product(self.h, other.h, out.ctypes.data)
        return complex(out[0], out[1])

    def seed(self, seed):
        self.lib.orc_seed(self.h, seed)

    def generate_events(self, num, seed=-1):
        out = np.empty(num, dtype=np.uint64)
        if self.lib.orc_generate_events(self.h, num, seed, out.ctypes.data) != 0:
            raise MemoryError("orc_generate_events")
        return out

    def projective_measurement(self, q):
        return int(self.lib.orc_projective_measurement(self.h, q))

    def measure(self):
        return int(self.lib.orc_measure(self.h))
