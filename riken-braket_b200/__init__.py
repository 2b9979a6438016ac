"""riken-braket_b200: B200-native state-vector gate application behind the
RIKEN-braket ket / bra interfaces.

The product is librbk.so (CUDA kernels for sm_100a + the C ABI of
include/rbk.h).  This package holds its Python binding (rbk.py), the seeded
workload generators (circuits.py), the adjoint-gradient harness, the .qcx
interpreter binding (qcx.py) and states sharded over ranks by global qubits
(global_qubits.py).  The
directory name is not a Python identifier; load it with ``load_package()``
from __graft_entry__.py (or importlib) under the name ``riken_braket_b200``.
"""
from . import adjoint, circuits, global_qubits, qcx, rbk  # noqa: F401
from .rbk import C64, C128, RbkError, State  # noqa: F401
