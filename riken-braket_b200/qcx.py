"""bra's .qcx interpreter on the engine (C ABI of include/rbk_qcx.h).

    text, state = qcx.run(open("circuit.qcx").read(), keep_state=True)

``run`` returns what bra prints for the program (bra/src/state.cpp:1980-2110)
and, on request, the final state as an ``rbk.State``.  ``parse`` gives the
parsed instruction list.  The command-line equivalent is bin/rbk-bra.
"""
from __future__ import annotations

import ctypes

from . import rbk

MAX_QUBITS = 40
MAX_VALUES = 40


class Instruction(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int32), ("kind", ctypes.c_int32), ("line", ctypes.c_int32),
                ("num_targets", ctypes.c_int32), ("num_controls", ctypes.c_int32), ("num_values", ctypes.c_int32),
                ("circuit", ctypes.c_int32), ("targets", ctypes.c_uint32 * MAX_QUBITS), ("controls", ctypes.c_uint32 * MAX_QUBITS),
                ("params", ctypes.c_double * 3), ("ints", ctypes.c_int64 * 2),
                ("values", ctypes.c_uint64 * MAX_VALUES), ("text", ctypes.c_char * 256)]

    def as_dict(self):
        return dict(op=self.op, kind=self.kind, line=self.line, circuit=self.circuit,
                    targets=list(self.targets[:self.num_targets]),
                    controls=list(self.controls[:self.num_controls]), params=list(self.params),
                    ints=list(self.ints), values=list(self.values[:min(self.num_values, MAX_VALUES)]),
                    text=self.text.decode())


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("device", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("deferred", ctypes.c_int), ("print_timing", ctypes.c_int)]


_bound = False


def _lib():
    global _bound
    L = rbk.lib()
    if not _bound:
        P = ctypes.c_void_p
        L.rbk_qcx_default_options.argtypes = [ctypes.POINTER(Options)]
        L.rbk_qcx_default_options.restype = None
        L.rbk_qcx_parse.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(P)]
        L.rbk_qcx_destroy.argtypes = [P]
        L.rbk_qcx_num_qubits.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
        L.rbk_qcx_num_circuits.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
        L.rbk_qcx_initial_state.argtypes = [P, ctypes.POINTER(ctypes.c_uint64)]
        L.rbk_qcx_num_instructions.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
        L.rbk_qcx_get_instruction.argtypes = [P, ctypes.c_int, ctypes.POINTER(Instruction)]
        L.rbk_qcx_run.argtypes = [P, ctypes.POINTER(Options), ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(P)]
        L.rbk_qcx_free_text.argtypes = [ctypes.c_void_p]
        L.rbk_qcx_free_text.restype = None
        for f in ("rbk_qcx_parse", "rbk_qcx_destroy", "rbk_qcx_num_qubits", "rbk_qcx_num_circuits", "rbk_qcx_initial_state",
                  "rbk_qcx_num_instructions", "rbk_qcx_get_instruction", "rbk_qcx_run"):
            getattr(L, f).restype = ctypes.c_int
        _bound = True
    return L


def _check(rc):
    if rc != 0:
        raise rbk.RbkError(rc, rbk.lib().rbk_last_error().decode())


class Program:
    """A parsed .qcx program."""

    def __init__(self, text):
        L = _lib()
        data = text.encode() if isinstance(text, str) else bytes(text)
        h = ctypes.c_void_p()
        _check(L.rbk_qcx_parse(data, len(data), ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            _lib().rbk_qcx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_qubits(self):
        v = ctypes.c_int()
        _check(_lib().rbk_qcx_num_qubits(self.h, ctypes.byref(v)))
        return v.value

    @property
    def num_circuits(self):
        v = ctypes.c_int()
        _check(_lib().rbk_qcx_num_circuits(self.h, ctypes.byref(v)))
        return v.value

    @property
    def initial_state(self):
        v = ctypes.c_uint64()
        _check(_lib().rbk_qcx_initial_state(self.h, ctypes.byref(v)))
        return v.value

    def instructions(self):
        L = _lib()
        count = ctypes.c_int()
        _check(L.rbk_qcx_num_instructions(self.h, ctypes.byref(count)))
        out = []
        for i in range(count.value):
            ins = Instruction()
            _check(L.rbk_qcx_get_instruction(self.h, i, ctypes.byref(ins)))
            out.append(ins.as_dict())
        return out

    def run(self, precision=rbk.C128, seed=1, deferred=True, timing=False, device=0, keep_state=False):
        """Returns (bra's output text, circuit 0's final State or None)."""
        L = _lib()
        opt = Options()
        L.rbk_qcx_default_options(ctypes.byref(opt))
        opt.precision, opt.seed, opt.deferred, opt.print_timing, opt.device = (
            precision, seed, int(deferred), int(timing), device)
        text = ctypes.c_void_p()
        st = ctypes.c_void_p()
        _check(L.rbk_qcx_run(self.h, ctypes.byref(opt), ctypes.byref(text), ctypes.byref(st) if keep_state else None))
        out = ctypes.string_at(text.value).decode()
        L.rbk_qcx_free_text(text)
        state = rbk.State.adopt(st, self.num_qubits, precision) if keep_state else None
        return out, state


def parse(text):
    return Program(text)


def run(text, **kw):
    prog = Program(text)
    try:
        return prog.run(**kw)
    finally:
        prog.close()
