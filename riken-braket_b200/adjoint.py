"""Adjoint (reverse-sweep) gradients through the C ABI (rbk_adjoint_gradient).

The reference has no differentiation support; this is one of the engine's
extensions.  ``adjoint_gradient`` returns E(theta) = <psi|H|psi> and dE/dtheta
for a circuit whose EX/EY/EZ gates take parameters.  ``AnsatzEnergy`` wraps it
in a torch.autograd.Function; it exists only as a gradient-check harness
(torch.autograd.gradcheck), not as a compute path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import rbk

GATE = {"H": 1, "X": 2, "Y": 3, "Z": 4, "U1": 5, "U2": 6, "U3": 7, "CNOT": 8, "CZ": 9, "U": 10,
        "EX": 11, "EY": 12, "EZ": 13, "SWAP": 14}


class CircuitGate(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("qubits", ctypes.c_int32 * 2), ("param", ctypes.c_int32),
                ("scale", ctypes.c_double), ("angles", ctypes.c_double * 3)]


def gate_array(spec):
    """spec: list of (mnemonic, qubits, param_index or None, scale, angles)."""
    arr = (CircuitGate * max(1, len(spec)))()
    for i, (mnem, qubits, param, scale, angles) in enumerate(spec):
        g = arr[i]
        g.kind = GATE[mnem]
        for j, q in enumerate(qubits[:2]):
            g.qubits[j] = int(q)
        g.param = -1 if param is None else int(param)
        g.scale = float(scale)
        for j, a in enumerate(angles[:3]):
            g.angles[j] = float(a)
    return arr, len(spec)


def ansatz_spec(n, layers):
    """The hardware-efficient ansatz of circuits.ansatz as a parametrised gate
    list: RY(theta_k) = EY with scale -1/2, RZ(theta_k) = EZ with scale -1/2,
    then the CZ ring; parameter k in the same order as circuits.ansatz."""
    spec, k = [], 0
    for _ in range(layers):
        for q in range(n):
            spec.append(("EY", (q,), k, -0.5, ()))
            k += 1
        for q in range(n):
            spec.append(("EZ", (q,), k, -0.5, ()))
            k += 1
        for i in range(n):
            spec.append(("CZ", (i, (i + 1) % n), None, 0.0, ()))
    return spec, k


def _bind():
    lib = rbk.lib()
    f = lib.rbk_adjoint_gradient
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def adjoint_gradient(n, spec, theta, terms, precision=rbk.C128, device=0):
    """Returns (energy, gradient) for the parametrised gate list `spec`."""
    gates, count = gate_array(spec)
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    strings = b"".join(s.encode() for s, _ in terms)
    coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
    energy = ctypes.c_double()
    grad = np.zeros(theta.size, dtype=np.float64)
    rc = _bind()(n, precision, device, ctypes.cast(gates, ctypes.c_void_p), count, theta.ctypes.data, theta.size,
                 len(terms), strings, coeffs.ctypes.data, ctypes.addressof(energy), grad.ctypes.data)
    if rc != 0:
        raise rbk.RbkError(rc, rbk.lib().rbk_last_error().decode())
    return energy.value, grad


class BatchInstance(ctypes.Structure):
    _fields_ = [("num_qubits", ctypes.c_int32), ("num_gates", ctypes.c_int32), ("gates", ctypes.c_void_p),
                ("num_params", ctypes.c_int32), ("num_terms", ctypes.c_int32), ("strings", ctypes.c_char_p),
                ("coeffs", ctypes.c_void_p)]


class BatchStats(ctypes.Structure):
    _fields_ = [("num_small", ctypes.c_int), ("num_large", ctypes.c_int), ("threads", ctypes.c_int),
                ("small_ms", ctypes.c_float), ("last_run_ms", ctypes.c_double)]


class Batch:
    """Many parametrised circuits at once (rbk_batch_*): instances is a list of
    (num_qubits, spec, num_params, terms) with spec as for adjoint_gradient."""

    def __init__(self, instances, precision=rbk.C128, device=0):
        L = rbk.lib()
        L.rbk_batch_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.rbk_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.rbk_batch_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(BatchStats)]
        L.rbk_batch_destroy.argtypes = [ctypes.c_void_p]
        self._keep = []
        arr = (BatchInstance * max(1, len(instances)))()
        self.num_params = []
        for i, (n, spec, num_params, terms) in enumerate(instances):
            gates, count = gate_array(spec)
            strings = b"".join(t.encode() for t, _ in terms)
            coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
            self._keep += [gates, strings, coeffs]
            arr[i].num_qubits, arr[i].num_gates, arr[i].gates = n, count, ctypes.cast(gates, ctypes.c_void_p)
            arr[i].num_params, arr[i].num_terms = num_params, len(terms)
            arr[i].strings, arr[i].coeffs = strings, coeffs.ctypes.data
            self.num_params.append(num_params)
        h = ctypes.c_void_p()
        rc = L.rbk_batch_create(precision, device, len(instances), ctypes.cast(arr, ctypes.c_void_p), ctypes.byref(h))
        if rc != 0:
            raise rbk.RbkError(rc, L.rbk_last_error().decode())
        self.h = h
        self.count = len(instances)

    def run(self, thetas):
        """thetas: list of per-instance parameter arrays.  Returns (energies, list of gradients)."""
        flat = np.ascontiguousarray(np.concatenate([np.asarray(t, dtype=np.float64) for t in thetas])
                                    if thetas else np.zeros(0), dtype=np.float64)
        energies = np.zeros(self.count, dtype=np.float64)
        grads = np.zeros(max(1, flat.size), dtype=np.float64)
        rc = rbk.lib().rbk_batch_run(self.h, flat.ctypes.data, energies.ctypes.data, grads.ctypes.data)
        if rc != 0:
            raise rbk.RbkError(rc, rbk.lib().rbk_last_error().decode())
        out, k = [], 0
        for p in self.num_params:
            out.append(grads[k:k + p].copy())
            k += p
        return energies, out

    def set_workers(self, workers):
        L = rbk.lib()
        L.rbk_batch_set_workers.argtypes = [ctypes.c_void_p, ctypes.c_int]
        rc = L.rbk_batch_set_workers(self.h, workers)
        if rc != 0:
            raise rbk.RbkError(rc, L.rbk_last_error().decode())

    def stats(self):
        st = BatchStats()
        rbk.lib().rbk_batch_get_stats(self.h, ctypes.byref(st))
        return {f: getattr(st, f) for f, _ in BatchStats._fields_}

    def tuned_shapes(self, sizes):
        """{num_qubits: tile shape} that the autotuner picked (rbk_batch_tuned_shape; sizes left at the default omitted)."""
        L = rbk.lib()
        L.rbk_batch_tuned_shape.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        out = {}
        for n in sorted(set(sizes)):
            sh = ctypes.c_int(-1)
            if L.rbk_batch_tuned_shape(self.h, int(n), ctypes.byref(sh)) == 0 and sh.value >= 0:
                out[int(n)] = sh.value
        return out

    def close(self):
        if getattr(self, "h", None):
            rbk.lib().rbk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AdjointContext:
    """rbk_adjoint_create/run/destroy: repeated gradients of n-qubit circuits
    without re-allocating the two state vectors."""

    def __init__(self, n, precision=rbk.C128, device=0):
        L = rbk.lib()
        L.rbk_adjoint_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.rbk_adjoint_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.rbk_adjoint_destroy.argtypes = [ctypes.c_void_p]
        h = ctypes.c_void_p()
        rc = L.rbk_adjoint_create(n, precision, device, ctypes.byref(h))
        if rc != 0:
            raise rbk.RbkError(rc, L.rbk_last_error().decode())
        self.h, self.n = h, n

    def gradient(self, spec, theta, terms):
        gates, count = gate_array(spec)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        strings = b"".join(s.encode() for s, _ in terms)
        coeffs = np.array([[complex(c).real, complex(c).imag] for _, c in terms], dtype=np.float64).ravel()
        energy = ctypes.c_double()
        grad = np.zeros(theta.size, dtype=np.float64)
        rc = rbk.lib().rbk_adjoint_run(self.h, ctypes.cast(gates, ctypes.c_void_p), count, theta.ctypes.data, theta.size,
                                       len(terms), strings, coeffs.ctypes.data, ctypes.addressof(energy), grad.ctypes.data)
        if rc != 0:
            raise rbk.RbkError(rc, rbk.lib().rbk_last_error().decode())
        return energy.value, grad

    def close(self):
        if getattr(self, "h", None):
            rbk.lib().rbk_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_autograd_function():
    """torch.autograd.Function over adjoint_gradient (gradient-check harness only)."""
    import torch

    class AnsatzEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, n, spec, terms):
            e, g = adjoint_gradient(n, spec, theta.detach().cpu().numpy(), terms)
            ctx.save_for_backward(torch.from_numpy(g))
            return theta.new_tensor(e)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g.to(grad_out.dtype), None, None, None

    return AnsatzEnergy
