"""The wider gate families of the C ABI (rbk_x_rotation_half_pi ... rbk_shor_box)
against the reference's own ket functions, called the way bra's nompi_state
calls them (oracle.KetRef.gate), on random states.  n = 7 runs the per-gate
kernels, n = 14 the fused tile passes; c128 to 1e-12."""
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libketref.so")),
                                 reason="oracle/_ref not built (needs the reference sources)")]

TOL64 = 1e-12
KG = dict(SX=7, SX_ADJ=8, SY=9, SY_ADJ=10, SZ=11, SZ_ADJ=12, ROTX=21, ROTX_ADJ=22, ROTY=23, ROTY_ADJ=24, X=3, Y=4,
          Z=5, EX=25, EY=27, EZ=29, ESWAP=31, TOFFOLI=33, CLEAR=34, SET=35, SHORBOX=36)


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return a / np.linalg.norm(a)


def cases(n):
    q = lambda *xs: tuple(x % n for x in xs)  # noqa: E731
    t = lambda x: x % n  # noqa: E731
    return [
        ("x_rotation_half_pi", (t(3),), {}, "ROTX", q(3), ()),
        ("x_rotation_half_pi", (t(5), q(1, 6)), {"adjoint": True}, "ROTX_ADJ", q(5), q(1, 6)),
        ("y_rotation_half_pi", (t(0), q(4)), {}, "ROTY", q(0), q(4)),
        ("y_rotation_half_pi", (t(6),), {"adjoint": True}, "ROTY_ADJ", q(6), ()),
        ("sqrt_pauli_x", (t(2), q(n - 1)), {}, "SX", q(2), q(n - 1)),
        ("sqrt_pauli_x", (t(4),), {"adjoint": True}, "SX_ADJ", q(4), ()),
        ("sqrt_pauli_y", (t(1),), {}, "SY", q(1), ()),
        ("sqrt_pauli_y", (t(3), q(0, 5)), {"adjoint": True}, "SY_ADJ", q(3), q(0, 5)),
        ("sqrt_pauli_z", (q(2, 5),), {}, "SZ", q(2, 5), ()),
        ("sqrt_pauli_z", (q(1, 3, n - 2), q(6)), {"adjoint": True}, "SZ_ADJ", q(1, 3, n - 2), q(6)),
        ("pauli_string", ("XX", q(0, n - 1)), {}, "X", q(0, n - 1), ()),
        ("pauli_string", ("YYY", q(1, 4, 6), q(2)), {}, "Y", q(1, 4, 6), q(2)),
        ("pauli_string", ("ZZ", q(3, 5), q(0, 1)), {}, "Z", q(3, 5), q(0, 1)),
    ]


def exp_cases(n):
    q = lambda *xs: tuple(x % n for x in xs)  # noqa: E731
    return [
        ("XX", q(0, 3), (), "EX"), ("XXX", q(6, 1, n - 2), q(2,), "EX"), ("YY", q(2, 5), (), "EY"),
        ("YYY", q(0, 4, 6), q(1, 3), "EY"), ("ZZ", q(1, n - 1), (), "EZ"), ("ZZZ", q(2, 3, 5), q(0,), "EZ"),
    ]


@pytest.mark.parametrize("n", [7, 14])
def test_gate_families_vs_reference(pkg, n):
    init = random_state(n, n)
    for i, (method, args, kw, kind, targets, controls) in enumerate(cases(n)):
        with pkg.State(n) as s:
            s.upload(init)
            getattr(s, method)(*args, **kw)
            r = oracle.KetRef(n)
            r.set_amplitudes(init)
            r.gate(KG[kind], targets, controls)
            assert np.abs(s.amplitudes() - r.amplitudes()).max() <= TOL64, (method, args, kw)


@pytest.mark.parametrize("n", [7, 14])
def test_exponential_strings_and_swap_vs_reference(pkg, n):
    init = random_state(n, 100 + n)
    for paulis, targets, controls, kind in exp_cases(n):
        with pkg.State(n) as s:
            s.upload(init)
            s.exponential_pauli_string(0.731, paulis, targets, controls)
            r = oracle.KetRef(n)
            r.set_amplitudes(init)
            r.gate(KG[kind], targets, controls, (0.731,))
            assert np.abs(s.amplitudes() - r.amplitudes()).max() <= TOL64, (paulis, targets, controls)
    for q1, q2, controls in [(0, 1, ()), (n - 1, 2, ()), (3, 5, (0,)), (6, 1, (2, n - 2))]:
        with pkg.State(n) as s:
            s.upload(init)
            s.exponential_swap(-0.42, q1, q2, controls)
            r = oracle.KetRef(n)
            r.set_amplitudes(init)
            r.gate(KG["ESWAP"], (q1, q2), controls, (-0.42,))
            assert np.abs(s.amplitudes() - r.amplitudes()).max() <= TOL64


@pytest.mark.parametrize("n", [7, 14])
def test_clear_set_toffoli_vs_reference(pkg, n):
    init = random_state(n, 200 + n)
    for op, q in [("clear", 2), ("set", n - 1), ("clear", 0)]:
        with pkg.State(n) as s:
            s.upload(init)
            getattr(s, op)(q)
            r = oracle.KetRef(n)
            r.set_amplitudes(init)
            r.gate(KG[op.upper()], (q,))
            assert np.abs(s.amplitudes() - r.amplitudes()).max() <= TOL64
    with pkg.State(n) as s:
        s.upload(init)
        s.pauli_x(4, controls=(1, n - 1))
        r = oracle.KetRef(n)
        r.set_amplitudes(init)
        r.gate(KG["TOFFOLI"], (4,), (1, n - 1))
        assert np.abs(s.amplitudes() - r.amplitudes()).max() == 0.0


@pytest.mark.parametrize("n,nx,divisor,base", [(7, 3, 5, 2), (12, 7, 21, 2), (14, 8, 15, 7), (10, 10, 1, 3)])
def test_shor_box_vs_reference(pkg, n, nx, divisor, base):
    with pkg.State(n) as s:
        s.hadamard(0)
        s.shor_box(nx, divisor, base)
        r = oracle.KetRef(n)
        r.gate(KG["SHORBOX"], (), (), (nx, divisor, base))
        assert np.array_equal(s.amplitudes(), r.amplitudes())
