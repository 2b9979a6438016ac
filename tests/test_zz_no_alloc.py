"""rbk_expectation_pauli_noalloc: the expectation value for callers that
cannot allocate device memory (host callbacks, a fully reserved HBM, loops
that must not synchronise the device).  Called through the C ABI on a state
the library owns, twice in a row, it must agree with rbk_expectation_pauli to
the FP64 tolerance of the other GPU tests.  This file is collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _noalloc(lib):
    f = lib.rbk_expectation_pauli_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("precision,tol", [(0, TOL64), (1, 1e-5)])
def test_noalloc_expectation_matches_allocating_entry_point(pkg, precision, tol):
    n = 16
    C = pkg.circuits
    lib = pkg.rbk.lib()
    noalloc = _noalloc(lib)
    terms = C.ansatz_hamiltonian(n) + [("XYZ" + "I" * (n - 3), 0.3 + 0.1j), ("Y" * n, 1.0),
                                       ("I" * (n - 2) + "YX", -0.5j)]
    strings = b"".join(s.encode() for s, _ in terms)
    coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
    with pkg.State(n, precision) as s:
        s.apply(C.random_circuit(n, 200, seed=5))
        want = s.expectation(terms)          # allocating entry point (state-owned scratch)
        s.canonicalize()                     # logical order in device memory
        ptr = s.device_pointer()
        for _ in range(2):                   # the shared scratch keeps the last call's contents
            out = np.zeros(2, dtype=np.float64)
            rc = noalloc(ptr, n, precision, len(terms), strings, coeffs.ctypes.data, out.ctypes.data, None)
            assert rc == 0, lib.rbk_last_error().decode()
            assert abs(complex(out[0], out[1]) - want) <= tol
        # a second, different state reuses the same scratch
        s.apply(C.random_circuit(n, 50, seed=6))
        want2 = s.expectation(terms)
        s.canonicalize()
        out = np.zeros(2, dtype=np.float64)
        assert noalloc(s.device_pointer(), n, precision, len(terms), strings, coeffs.ctypes.data,
                       out.ctypes.data, None) == 0
        assert abs(complex(out[0], out[1]) - want2) <= tol


def test_noalloc_rejects_bad_arguments(pkg):
    lib = pkg.rbk.lib()
    noalloc = _noalloc(lib)
    out = np.zeros(2, dtype=np.float64)
    coeffs = np.array([1.0, 0.0])
    with pkg.State(12) as s:
        ptr = s.device_pointer()
        assert noalloc(ptr, 40, 0, 1, b"Z" * 40, coeffs.ctypes.data, out.ctypes.data, None) == 1
        assert noalloc(ptr, 12, 0, 1, b"Q" * 12, coeffs.ctypes.data, out.ctypes.data, None) == 1
        assert noalloc(None, 12, 0, 1, b"Z" * 12, coeffs.ctypes.data, out.ctypes.data, None) == 1
        many = [("I" * k + "X" + "I" * (11 - k)) for k in range(12)]
        many += [("I" * a + "X" + "I" * (b - a - 1) + "X" + "I" * (11 - b)) for a in range(12) for b in range(a + 1, 12)]
        cs = np.tile([1.0, 0.0], len(many))
        assert len(many) > 64
        assert noalloc(ptr, 12, 0, len(many), "".join(many).encode(), cs.ctypes.data, out.ctypes.data, None) == 1
