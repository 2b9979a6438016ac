"""Python binding of the C ABI in include/rbk.h (librbk.so, loaded in place).

``State`` mirrors the gate methods of bra::state (bra/include/bra/state.hpp:712-1003)
and ket::gate::* names; every call goes straight to the CUDA library.  There is
no CPU path: if librbk.so is missing or no GPU is present, constructing a State
raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librbk.so")

C128, C64 = 0, 1
STATUS = {0: "RBK_OK", 1: "RBK_ERR_INVALID", 2: "RBK_ERR_CUDA", 3: "RBK_ERR_OOM",
          4: "RBK_ERR_TIMEOUT", 5: "RBK_ERR_UNSUPPORTED", 6: "RBK_ERR_STATE"}


class RbkError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


class Stats(ctypes.Structure):
    _fields_ = [("gates_issued", ctypes.c_uint64), ("passes", ctypes.c_uint64),
                ("gate_launches", ctypes.c_uint64), ("reduction_passes", ctypes.c_uint64),
                ("relabel_passes", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64)]


_lib = None
_P = ctypes.c_void_p
_U32P = ctypes.POINTER(ctypes.c_uint32)
_D = ctypes.c_double
_I = ctypes.c_int
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64

_SIGNATURES = {
    "rbk_last_error": ([], ctypes.c_char_p),
    "rbk_version": ([], _I),
    "rbk_pass_descriptor_bytes": ([ctypes.POINTER(_U64)], _I),
    "rbk_state_create": ([_I, _I, _U64, _I, ctypes.POINTER(_P)], _I),
    "rbk_state_destroy": ([_P], _I),
    "rbk_state_num_qubits": ([_P, ctypes.POINTER(_I)], _I),
    "rbk_state_precision": ([_P, ctypes.POINTER(_I)], _I),
    "rbk_state_reset": ([_P, _U64], _I),
    "rbk_state_upload": ([_P, _P, _U64, _U64], _I),
    "rbk_state_download": ([_P, _P, _U64, _U64], _I),
    "rbk_state_synchronize": ([_P], _I),
    "rbk_flush": ([_P], _I),
    "rbk_state_set_deferred": ([_P, _I], _I),
    "rbk_state_set_pass_budget": ([_P, _I], _I),
    "rbk_state_set_tile_shape": ([_P, _I], _I),
    "rbk_state_get_stats": ([_P, ctypes.POINTER(Stats)], _I),
    "rbk_state_reset_stats": ([_P], _I),
    "rbk_state_device_ms": ([_P, ctypes.POINTER(_D)], _I),
    "rbk_state_get_permutation": ([_P, _U32P], _I),
    "rbk_state_canonicalize": ([_P], _I),
    "rbk_state_set_permutation": ([_P, ctypes.POINTER(ctypes.c_uint32)], _I),
    "rbk_state_set_layout": ([_P, ctypes.POINTER(ctypes.c_uint32)], _I),
    "rbk_state_device_pointer": ([_P, ctypes.POINTER(_P)], _I),
    "rbk_begin_fusion": ([_P], _I),
    "rbk_end_fusion": ([_P], _I),
    "rbk_hadamard": ([_P, _U32, _U32P, _I], _I),
    "rbk_pauli_x": ([_P, _U32, _U32P, _I], _I),
    "rbk_pauli_y": ([_P, _U32, _U32P, _I], _I),
    "rbk_pauli_z": ([_P, _U32P, _I], _I),
    "rbk_phase_shift_coeff": ([_P, _D, _D, _U32P, _I], _I),
    "rbk_phase_shift": ([_P, _D, _U32P, _I], _I),
    "rbk_controlled_phase_shift_k": ([_P, _I, _U32P, _I], _I),
    "rbk_phase_shift2": ([_P, _D, _D, _U32, _U32P, _I], _I),
    "rbk_phase_shift3": ([_P, _D, _D, _D, _U32, _U32P, _I], _I),
    "rbk_exponential_pauli_x": ([_P, _D, _U32, _U32P, _I], _I),
    "rbk_exponential_pauli_y": ([_P, _D, _U32, _U32P, _I], _I),
    "rbk_exponential_pauli_z": ([_P, _D, _U32, _U32P, _I], _I),
    "rbk_swap": ([_P, _U32, _U32, _U32P, _I], _I),
    "rbk_apply_matrix2": ([_P, ctypes.POINTER(_D), _U32, _U32P, _I], _I),
    "rbk_apply_diagonal2": ([_P, ctypes.POINTER(_D), _U32, _U32P, _I], _I),
    "rbk_norm2": ([_P, ctypes.POINTER(_D)], _I),
    "rbk_probabilities": ([_P, _P, _U64, _U64], _I),
    "rbk_spin_expectation_values": ([_P, _P], _I),
    "rbk_expectation_pauli": ([_P, _I, ctypes.c_char_p, _P, _P], _I),
    "rbk_inner_product": ([_P, _P, _P], _I),
    "rbk_fidelity": ([_P, _P, ctypes.POINTER(_D)], _I),
    "rbk_inner_product_pauli": ([_P, _P, _I, ctypes.c_char_p, _P, _P], _I),
    "rbk_fidelity_pauli": ([_P, _P, _I, ctypes.c_char_p, _P, ctypes.POINTER(_D)], _I),
    "rbk_x_rotation_half_pi": ([_P, _I, _U32, _U32P, _I], _I),
    "rbk_y_rotation_half_pi": ([_P, _I, _U32, _U32P, _I], _I),
    "rbk_sqrt_pauli_x": ([_P, _I, _U32, _U32P, _I], _I),
    "rbk_sqrt_pauli_y": ([_P, _I, _U32, _U32P, _I], _I),
    "rbk_sqrt_pauli_z": ([_P, _I, _U32P, _I, _U32P, _I], _I),
    "rbk_pauli_string": ([_P, ctypes.c_char_p, _U32P, _I, _U32P, _I], _I),
    "rbk_exponential_pauli_string": ([_P, _D, ctypes.c_char_p, _U32P, _I, _U32P, _I], _I),
    "rbk_exponential_swap": ([_P, _D, _U32, _U32, _U32P, _I], _I),
    "rbk_clear": ([_P, _U32], _I),
    "rbk_set": ([_P, _U32], _I),
    "rbk_shor_box": ([_P, _U32, _U64, _U64], _I),
    "rbk_apply_unitary": ([_P, ctypes.POINTER(_D), _U32P, _I], _I),
    "rbk_state_set_fusion_mode": ([_P, _I], _I),
    "rbk_state_seed": ([_P, _U64], _I),
    "rbk_generate_events": ([_P, _I, ctypes.c_int64, _P], _I),
    "rbk_measure": ([_P, ctypes.POINTER(_U64)], _I),
    "rbk_projective_measurement": ([_P, _U32, ctypes.POINTER(_I)], _I),
}


def lib():
    """Loads librbk.so once; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is not built (run __graft_entry__.build() or make -C riken-braket_b200)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def pass_descriptor_bytes():
    """Bytes of the parameter block one fused-pass launch carries from the host."""
    v = _U64()
    _check(lib().rbk_pass_descriptor_bytes(ctypes.byref(v)))
    return v.value


def _check(rc):
    if rc != 0:
        raise RbkError(rc, lib().rbk_last_error().decode())


def _qarr(qs):
    qs = [int(q) for q in qs]
    if not qs:
        return None, 0
    return (ctypes.c_uint32 * len(qs))(*qs), len(qs)


class State:
    """A state vector in GPU memory, |initial_index> at creation."""

    def __init__(self, num_qubits, precision=C128, initial_index=0, device=0):
        h = ctypes.c_void_p()
        _check(lib().rbk_state_create(num_qubits, precision, initial_index, device, ctypes.byref(h)))
        self.h = h
        self.n = num_qubits
        self.precision = precision
        self.dtype = np.complex128 if precision == C128 else np.complex64

    @classmethod
    def adopt(cls, handle, num_qubits, precision):
        """Wraps an rbk_state* created elsewhere (e.g. by rbk_qcx_run); the wrapper owns it."""
        s = cls.__new__(cls)
        s.h = handle if isinstance(handle, ctypes.c_void_p) else ctypes.c_void_p(handle)
        s.n = num_qubits
        s.precision = precision
        s.dtype = np.complex128 if precision == C128 else np.complex64
        return s

    def close(self):
        if getattr(self, "h", None):
            lib().rbk_state_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- lifecycle / data ---------------------------------------------------
    def reset(self, index=0):
        _check(lib().rbk_state_reset(self.h, index))

    def upload(self, amps, offset=0):
        a = np.ascontiguousarray(amps, dtype=self.dtype)
        _check(lib().rbk_state_upload(self.h, a.ctypes.data, offset, a.size))

    def amplitudes(self, offset=0, count=None):
        count = (1 << self.n) - offset if count is None else count
        out = np.empty(count, dtype=self.dtype)
        _check(lib().rbk_state_download(self.h, out.ctypes.data, offset, count))
        return out

    def synchronize(self):
        _check(lib().rbk_state_synchronize(self.h))

    def flush(self):
        _check(lib().rbk_flush(self.h))

    def set_deferred(self, on):
        _check(lib().rbk_state_set_deferred(self.h, 1 if on else 0))

    def set_pass_budget(self, budget):
        _check(lib().rbk_state_set_pass_budget(self.h, budget))

    def set_tile_shape(self, shape):
        _check(lib().rbk_state_set_tile_shape(self.h, shape))

    def stats(self):
        s = Stats()
        _check(lib().rbk_state_get_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def reset_stats(self):
        _check(lib().rbk_state_reset_stats(self.h))

    def device_ms(self):
        v = ctypes.c_double()
        _check(lib().rbk_state_device_ms(self.h, ctypes.byref(v)))
        return v.value

    def permutation(self):
        out = (ctypes.c_uint32 * self.n)()
        _check(lib().rbk_state_get_permutation(self.h, out))
        return list(out)

    def canonicalize(self):
        _check(lib().rbk_state_canonicalize(self.h))

    def set_permutation(self, perm):
        """Declares the layout map (logical q on physical bit perm[q]) without moving data."""
        arr = (ctypes.c_uint32 * self.n)(*[int(x) for x in perm])
        _check(lib().rbk_state_set_permutation(self.h, arr))

    def set_layout(self, perm):
        """Moves the data so that the layout map becomes perm; the logical state is unchanged."""
        arr = (ctypes.c_uint32 * self.n)(*[int(x) for x in perm])
        _check(lib().rbk_state_set_layout(self.h, arr))

    def device_pointer(self):
        p = ctypes.c_void_p()
        _check(lib().rbk_state_device_pointer(self.h, ctypes.byref(p)))
        return p.value

    # -- bra::state gate methods ---------------------------------------------
    def begin_fusion(self):
        _check(lib().rbk_begin_fusion(self.h))

    def end_fusion(self):
        _check(lib().rbk_end_fusion(self.h))

    def hadamard(self, t, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_hadamard(self.h, t, c, nc))

    def pauli_x(self, t, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_pauli_x(self.h, t, c, nc))

    def pauli_y(self, t, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_pauli_y(self.h, t, c, nc))

    def pauli_z(self, *qubits):
        q, nq = _qarr(qubits)
        _check(lib().rbk_pauli_z(self.h, q, nq))

    def phase_shift_coeff(self, coeff, *qubits):
        q, nq = _qarr(qubits)
        coeff = complex(coeff)
        _check(lib().rbk_phase_shift_coeff(self.h, coeff.real, coeff.imag, q, nq))

    def phase_shift(self, phase, *qubits):
        q, nq = _qarr(qubits)
        _check(lib().rbk_phase_shift(self.h, phase, q, nq))

    def controlled_phase_shift_k(self, k, *qubits):
        q, nq = _qarr(qubits)
        _check(lib().rbk_controlled_phase_shift_k(self.h, int(k), q, nq))

    def u2(self, phi, lam, t, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_phase_shift2(self.h, phi, lam, t, c, nc))

    def u3(self, theta, phi, lam, t, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_phase_shift3(self.h, theta, phi, lam, t, c, nc))

    def exponential_pauli_x(self, phase, t, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_exponential_pauli_x(self.h, phase, t, c, nc))

    def exponential_pauli_y(self, phase, t, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_exponential_pauli_y(self.h, phase, t, c, nc))

    def exponential_pauli_z(self, phase, t, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_exponential_pauli_z(self.h, phase, t, c, nc))

    def swap(self, q1, q2, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_swap(self.h, q1, q2, c, nc))

    def apply_matrix2(self, m, t, controls=()):
        m = np.asarray(m, dtype=np.complex128).reshape(2, 2)
        arr = (ctypes.c_double * 8)(*[v for z in m.ravel() for v in (z.real, z.imag)])
        c, nc = _qarr(controls)
        _check(lib().rbk_apply_matrix2(self.h, arr, t, c, nc))

    def apply_diagonal2(self, d0, d1, t, controls=()):
        d0, d1 = complex(d0), complex(d1)
        arr = (ctypes.c_double * 4)(d0.real, d0.imag, d1.real, d1.imag)
        c, nc = _qarr(controls)
        _check(lib().rbk_apply_diagonal2(self.h, arr, t, c, nc))

    def apply(self, ops):
        """Applies bra instruction tuples (see circuits.py)."""
        for mnem, q, p in ops:
            if mnem == "H":
                self.hadamard(q[0])
            elif mnem == "X":
                self.pauli_x(q[0])
            elif mnem == "Y":
                self.pauli_y(q[0])
            elif mnem == "Z":
                self.pauli_z(q[0])
            elif mnem == "U1":
                self.phase_shift(p[0], q[0])
            elif mnem == "U2":
                self.u2(p[0], p[1], q[0])
            elif mnem == "U3":
                self.u3(p[0], p[1], p[2], q[0])
            elif mnem == "CNOT":
                self.pauli_x(q[1], controls=(q[0],))
            elif mnem == "CZ":
                self.pauli_z(q[0], q[1])
            elif mnem == "U":
                self.controlled_phase_shift_k(int(p[0]), q[0], q[1])
            elif mnem == "EY":
                self.exponential_pauli_y(p[0], q[0])
            elif mnem == "EZ":
                self.exponential_pauli_z(p[0], q[0])
            elif mnem == "EX":
                self.exponential_pauli_x(p[0], q[0])
            elif mnem == "SWAP":
                self.swap(q[0], q[1])
            elif mnem == "BEGIN FUSION":
                self.begin_fusion()
            elif mnem == "END FUSION":
                self.end_fusion()
            else:
                raise ValueError(f"unsupported instruction {mnem}")

    # -- further gate families ---------------------------------------------
    def x_rotation_half_pi(self, t, controls=(), adjoint=False):
        c, nc = _qarr(controls)
        _check(lib().rbk_x_rotation_half_pi(self.h, int(adjoint), t, c, nc))

    def y_rotation_half_pi(self, t, controls=(), adjoint=False):
        c, nc = _qarr(controls)
        _check(lib().rbk_y_rotation_half_pi(self.h, int(adjoint), t, c, nc))

    def sqrt_pauli_x(self, t, controls=(), adjoint=False):
        c, nc = _qarr(controls)
        _check(lib().rbk_sqrt_pauli_x(self.h, int(adjoint), t, c, nc))

    def sqrt_pauli_y(self, t, controls=(), adjoint=False):
        c, nc = _qarr(controls)
        _check(lib().rbk_sqrt_pauli_y(self.h, int(adjoint), t, c, nc))

    def sqrt_pauli_z(self, targets, controls=(), adjoint=False):
        t, nt = _qarr(targets)
        c, nc = _qarr(controls)
        _check(lib().rbk_sqrt_pauli_z(self.h, int(adjoint), t, nt, c, nc))

    def pauli_string(self, paulis, targets, controls=()):
        t, nt = _qarr(targets)
        c, nc = _qarr(controls)
        _check(lib().rbk_pauli_string(self.h, paulis.encode(), t, nt, c, nc))

    def exponential_pauli_string(self, phase, paulis, targets, controls=()):
        t, nt = _qarr(targets)
        c, nc = _qarr(controls)
        _check(lib().rbk_exponential_pauli_string(self.h, phase, paulis.encode(), t, nt, c, nc))

    def exponential_swap(self, phase, q1, q2, controls=()):
        c, nc = _qarr(controls)
        _check(lib().rbk_exponential_swap(self.h, phase, q1, q2, c, nc))

    def apply_unitary(self, u, qubits):
        """Dense 2^k x 2^k unitary u[r][c] = <r|U|c>, bit i of the index = qubits[i]."""
        u = np.ascontiguousarray(u, dtype=np.complex128)
        q, nq = _qarr(qubits)
        assert u.shape == (1 << nq, 1 << nq)
        _check(lib().rbk_apply_unitary(self.h, u.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), q, nq))

    def set_fusion_mode(self, mode):
        """1: complex<float> fusion blocks of 5-6 qubits run as tensor-core unitaries."""
        _check(lib().rbk_state_set_fusion_mode(self.h, mode))

    def clear(self, q):
        _check(lib().rbk_clear(self.h, q))

    def set(self, q):
        _check(lib().rbk_set(self.h, q))

    def shor_box(self, num_exponent_qubits, divisor, base):
        _check(lib().rbk_shor_box(self.h, num_exponent_qubits, divisor, base))

    # -- observables -----------------------------------------------------------
    def norm2(self):
        v = ctypes.c_double()
        _check(lib().rbk_norm2(self.h, ctypes.byref(v)))
        return v.value

    def probabilities(self, offset=0, count=None):
        count = (1 << self.n) - offset if count is None else count
        out = np.empty(count, dtype=np.float64)
        _check(lib().rbk_probabilities(self.h, out.ctypes.data, offset, count))
        return out

    def spins(self):
        out = np.empty((self.n, 3), dtype=np.float64)
        _check(lib().rbk_spin_expectation_values(self.h, out.ctypes.data))
        return out

    def expectation(self, terms):
        strings = b"".join(s.encode() for s, _ in terms)
        coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
        out = np.empty(2, dtype=np.float64)
        _check(lib().rbk_expectation_pauli(self.h, len(terms), strings, coeffs.ctypes.data, out.ctypes.data))
        return complex(out[0], out[1])

    def inner_product(self, other):
        """ket::inner_product(self, other) = <other|self>."""
        out = np.empty(2, dtype=np.float64)
        _check(lib().rbk_inner_product(self.h, other.h, out.ctypes.data))
        return complex(out[0], out[1])

    def fidelity(self, other):
        v = ctypes.c_double()
        _check(lib().rbk_fidelity(self.h, other.h, ctypes.byref(v)))
        return v.value

    def inner_product_pauli(self, other, terms):
        """<other| H |self> for H = sum of (string, coeff) terms (strings over all qubits)."""
        strings = b"".join(s.encode() for s, _ in terms)
        coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
        out = np.empty(2, dtype=np.float64)
        _check(lib().rbk_inner_product_pauli(self.h, other.h, len(terms), strings, coeffs.ctypes.data, out.ctypes.data))
        return complex(out[0], out[1])

    def fidelity_pauli(self, other, terms):
        """|<other| H |self>|^2."""
        strings = b"".join(s.encode() for s, _ in terms)
        coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
        v = ctypes.c_double()
        _check(lib().rbk_fidelity_pauli(self.h, other.h, len(terms), strings, coeffs.ctypes.data, ctypes.byref(v)))
        return v.value

    # -- sampling and measurement ------------------------------------------------
    def seed(self, seed):
        """Re-seeds the state's std::mt19937_64 (bra's initial seed is 1)."""
        _check(lib().rbk_state_seed(self.h, seed))

    def generate_events(self, num, seed=-1):
        """ket::generate_events: num basis indices drawn from |a|^2.  seed < 0
        draws from the state's generator; otherwise a fresh one seeded `seed`.
        The amplitudes are left unchanged."""
        out = np.empty(num, dtype=np.uint64)
        _check(lib().rbk_generate_events(self.h, num, seed, out.ctypes.data))
        return out

    def measure(self):
        """ket::measure: one sampled basis index; the state collapses onto it."""
        v = ctypes.c_uint64()
        _check(lib().rbk_measure(self.h, ctypes.byref(v)))
        return v.value

    def projective_measurement(self, qubit):
        """ket::gate::projective_measurement: outcome 0/1, state renormalised."""
        v = ctypes.c_int()
        _check(lib().rbk_projective_measurement(self.h, qubit, ctypes.byref(v)))
        return v.value
