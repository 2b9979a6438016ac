"""rbk_expectation_pauli_noalloc: the expectation value for callers that
cannot allocate device memory when they need it (HBM reserved in full by
another allocator, loops that must not synchronise the device through
cudaMalloc / cudaFree).  Called through the C ABI on a state the library owns,
twice in a row, it must agree with rbk_expectation_pauli to the FP64
tolerance of the other GPU tests, and a warmed-up call must leave the device's
free memory unchanged.  This file is collected last."""
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


def _args(terms):
    strings = b"".join(s.encode() for s, _ in terms)
    coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
    return strings, coeffs


def _call(lib, noalloc, ptr, n, precision, terms):
    strings, coeffs = _args(terms)
    out = np.zeros(2, dtype=np.float64)
    rc = noalloc(ptr, n, precision, len(terms), strings, coeffs.ctypes.data, out.ctypes.data, None)
    assert rc == 0, lib.rbk_last_error().decode()
    return complex(out[0], out[1])


def _logical_pointer(s):
    """Logical-order device pointer of a library state, with every queued pass
    finished: the state's stream is non-blocking, so the entry point's stream
    (the legacy default one here) is ordered after it only through this wait."""
    s.canonicalize()
    ptr = s.device_pointer()
    s.synchronize()
    return ptr


def _term_sets(n):
    mixed = [("XYZ" + "I" * (n - 3), 0.3 + 0.1j), ("Y" * n, 1.0), ("I" * (n - 2) + "YX", -0.5j)]
    # 70 strings of Z and I only: one flip mask, split into groups of at most 64 strings
    rng = np.random.Generator(np.random.PCG64(70))
    zs = ["".join("Z" if b else "I" for b in rng.integers(0, 2, size=n)) for _ in range(70)]
    diag = [(z, complex(w)) for z, w in zip(zs, rng.uniform(-1, 1, size=70))]
    # exactly 64 distinct X/Y positions, the limit of the fixed scratch
    flips = []
    for k in range(1, 65):
        s = ["I"] * n
        for b in range(7):
            if (k >> b) & 1:
                s[b] = "X" if b % 2 else "Y"
        s[n - 1] = "Z" if k % 3 else "I"
        flips.append(("".join(s), complex(1.0 / k, 0.1 * (k % 5))))
    return {"mixed": mixed, "ham+mixed": None, "70 diagonal strings": diag, "64 flip masks": flips}


@pytest.mark.parametrize("precision,tol", [(0, TOL64), (1, 1e-5)])
def test_noalloc_expectation_matches_allocating_entry_point(pkg, precision, tol):
    n = 16
    C = pkg.circuits
    lib = pkg.rbk.lib()
    noalloc = _noalloc(lib)
    sets = _term_sets(n)
    sets["ham+mixed"] = C.ansatz_hamiltonian(n) + sets["mixed"]
    def flip_masks(terms):
        return {sum(1 << k for k, c in enumerate(p) if c in "XY") for p, _ in terms}
    assert len(flip_masks(sets["64 flip masks"])) == 64
    assert len(flip_masks(sets["70 diagonal strings"])) == 1
    with pkg.State(n, precision) as s:
        s.apply(C.random_circuit(n, 200, seed=5))
        want = {name: s.expectation(terms) for name, terms in sets.items()}  # allocating entry point
        ptr = _logical_pointer(s)
        for name, terms in sets.items():
            for _ in range(2):  # the shared scratch keeps the last call's contents
                got = _call(lib, noalloc, ptr, n, precision, terms)
                assert abs(got - want[name]) <= tol, (name, got, want[name])
        # a second, different state reuses the same scratch
        s.apply(C.random_circuit(n, 50, seed=6))
        want2 = s.expectation(sets["ham+mixed"])
        ptr = _logical_pointer(s)
        assert abs(_call(lib, noalloc, ptr, n, precision, sets["ham+mixed"]) - want2) <= tol


def test_noalloc_leaves_device_memory_unchanged(pkg):
    """Once a call has loaded the library's device code on the device, further
    calls allocate nothing: the device's free memory is the same before and
    after them."""
    import torch

    n = 18
    lib = pkg.rbk.lib()
    noalloc = _noalloc(lib)
    terms = pkg.circuits.ansatz_hamiltonian(n)
    with pkg.State(n) as s:
        s.apply(pkg.circuits.random_circuit(n, 100, seed=9))
        want = s.expectation(terms)
        ptr = _logical_pointer(s)
        _call(lib, noalloc, ptr, n, 0, terms)  # warm-up: module load, address lookup
        torch.cuda.synchronize(0)
        free0, _ = torch.cuda.mem_get_info(0)
        got = [_call(lib, noalloc, ptr, n, 0, terms) for _ in range(3)]
        torch.cuda.synchronize(0)
        free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert all(abs(g - want) <= TOL64 for g in got)


def test_noalloc_rejects_bad_arguments(pkg):
    lib = pkg.rbk.lib()
    noalloc = _noalloc(lib)
    out = np.zeros(2, dtype=np.float64)
    coeffs = np.array([1.0, 0.0])
    with pkg.State(12) as s:
        ptr = _logical_pointer(s)
        assert noalloc(ptr, 40, 0, 1, b"Z" * 40, coeffs.ctypes.data, out.ctypes.data, None) == 1
        assert noalloc(ptr, 12, 0, 1, b"Q" * 12, coeffs.ctypes.data, out.ctypes.data, None) == 1
        assert noalloc(None, 12, 0, 1, b"Z" * 12, coeffs.ctypes.data, out.ctypes.data, None) == 1
        many = [("I" * k + "X" + "I" * (11 - k)) for k in range(12)]
        many += [("I" * a + "X" + "I" * (b - a - 1) + "X" + "I" * (11 - b)) for a in range(12) for b in range(a + 1, 12)]
        cs = np.tile([1.0, 0.0], len(many))
        assert len(many) > 64
        assert noalloc(ptr, 12, 0, len(many), "".join(many).encode(), cs.ctypes.data, out.ctypes.data, None) == 1
