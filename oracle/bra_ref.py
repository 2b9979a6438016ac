"""TEST INFRASTRUCTURE ONLY: bra's .qcx front end restated in Python, driving
the reference's own ket code (oracle/_ref/libketref.so through oracle.KetRef).

It checks the engine's C++ interpreter (riken-braket_b200/csrc/qcx.cpp) from
the other side: an independent parse of the same text (bra/src/interpreter.cpp:
372-826 and interpret_controlled_gates :3341-3508), executed gate by gate with
the ket calls bra's nompi_state makes (bra/src/nompi_state.cpp), printing what
bra::state prints (bra/src/state.cpp:1980-2110) without the timing lines.

Fusion blocks whose gates all have bra fused-gate classes in the reference
leg run through bra's fusion (ORC codes of oracle_ops.h); other blocks run
unfused (bra's fused and unfused results agree to rounding,
ket/test/fused_runtime_gate_numerical.cpp).
"""
from __future__ import annotations

import math

import numpy as np

import oracle

# Gate kinds (oracle_ops.h KG_*; the engine's RBK_QCX_* use the same numbers).
KG = dict(H=1, NOT=2, X=3, Y=4, Z=5, SWAP=6, SX=7, SX_ADJ=8, SY=9, SY_ADJ=10, SZ=11, SZ_ADJ=12, U1=13, U1_ADJ=14,
          U2=15, U2_ADJ=16, U3=17, U3_ADJ=18, R=19, R_ADJ=20, ROTX=21, ROTX_ADJ=22, ROTY=23, ROTY_ADJ=24, EX=25,
          EX_ADJ=26, EY=27, EY_ADJ=28, EZ=29, EZ_ADJ=30, ESWAP=31, ESWAP_ADJ=32, TOFFOLI=33, CLEAR=34, SET=35,
          SHORBOX=36)
OP = dict(GATE=1, BEGIN_FUSION=2, END_FUSION=3, MEASUREMENT=4, AMPLITUDES=5, GENERATE_EVENTS=6, EXIT=7,
          PROJECTIVE=8, EXPECTATION=9, PRINT=10, NOOP=11, INNERPROD=12, FIDELITY=13, VAR=14, LET=15)
LET_OPS = {":=": 0, "+=": 1, "-=": 2, "*=": 3, "/=": 4}
ALL, NONE = -1, -2  # INNERPROD / FIDELITY partner: every circuit, or nothing to do

CONSTANTS = {":REAL": 0.0, ":IMAG": 0.0, ":PI": math.pi, ":HALF_PI": math.pi / 2, ":TWO_PI": 2 * math.pi,
             ":ROOT_TWO": math.sqrt(2.0), ":HALF_ROOT_TWO": math.sqrt(0.5)}


class QcxError(Exception):
    pass


def _real(tok):
    if tok[0].isdigit() or tok[0] in "+-.":
        return float(tok)
    if tok in CONSTANTS:
        return CONSTANTS[tok]
    if tok.startswith(":REAL:") and len(tok) > 6 and (tok[6].isdigit() or tok[6] in "+-."):
        return float(tok[6:])
    raise QcxError(f"unsupported value {tok}")


def _count(body, letter):
    """'XXX' -> 3, 'X3' -> 3, else 0."""
    if not body or body[0] != letter:
        return 0
    if set(body) == {letter}:
        return len(body)
    if len(body) > 1 and body[1:].isdigit():
        return int(body[1:])
    return 0


def _operator(tok):
    """An operator column: (Pauli string, 0) for a :PAULIS:<s> literal,
    (NAME[:index], 1) for a PAULISS variable."""
    u = tok.upper()
    if u.startswith(":PAULIS:"):
        return u[len(":PAULIS:"):], 0
    return u, 1


def parse(text):
    """Returns (num_qubits, initial_state, instructions); each instruction is a
    dict with op, kind, targets, controls, params, ints, values, text, line, circuit."""
    return parse_program(text)[:3]


def parse_program(text):
    """parse() plus the number of circuits (CIRCUITS n)."""
    n, init, code = None, 0, []
    state = dict(circuit=0, in_circuit=False, num_circuits=1)

    def ins(op, line, **kw):
        d = dict(op=OP[op], kind=0, targets=[], controls=[], params=[0.0, 0.0, 0.0], ints=[0, 0], values=[], text="",
                 line=line, circuit=state["circuit"])
        d.update(kw)
        code.append(d)

    def qubit(tok):
        q = int(tok)
        if not tok.isdigit() or q >= n:
            raise QcxError(f"bad qubit {tok}")
        return q

    def gate(cols, line, kind, nc, nt, npar, exponent=False, all_controls=False):
        if len(cols) != 1 + nc + nt + npar:
            raise QcxError(f"line {line}: wrong operand count")
        qs = [qubit(t) for t in cols[1:1 + nc + nt]]
        if len(set(qs)) != len(qs):
            raise QcxError(f"line {line}: repeated qubit")
        ctl = qs if all_controls else qs[:nc]
        tgt = [] if all_controls else qs[nc:]
        params = [0.0, 0.0, 0.0]
        for k in range(npar):
            tok = cols[1 + nc + nt + k]
            params[k] = float(int(tok)) if exponent else _real(tok)
        ins("GATE", line, kind=KG[kind], targets=tgt, controls=ctl, params=params)

    def plain_or_controlled(cols, line, m, nc):
        adj = len(m) > 1 and m.endswith("+")
        base = m[:-1] if adj else m
        if base in ("I", "IC") and not adj:
            if len(cols) != 2 + nc:
                raise QcxError(f"line {line}: wrong operand count")
            [qubit(t) for t in cols[1:]]
            ins("NOOP", line)
            return True
        if not adj and _count(m, "I") >= 2:
            if len(cols) != 1 + nc + _count(m, "I"):
                raise QcxError("arity")
            ins("NOOP", line)
            return True
        if not adj and base in ("H", "NOT"):
            gate(cols, line, base, nc, 1, 0)
            return True
        if not adj and base == "Z":
            gate(cols, line, "Z", nc, 1, 0, all_controls=True)
            return True
        for letter in "XYZ":
            if not adj and _count(m, letter) >= 1:
                gate(cols, line, letter, nc, _count(m, letter), 0)
                return True
        if not adj and base == "SWAP":
            gate(cols, line, "SWAP", nc, 2, 0)
            return True
        suffix = "_ADJ" if adj else ""
        if base in ("S", "SZ"):
            gate(cols, line, "SZ" + suffix, nc, 1, 0, all_controls=True)
            return True
        if base.startswith("S") and _count(base[1:], "Z") >= 1:
            k = _count(base[1:], "Z")
            gate(cols, line, "SZ" + suffix, nc, k, 0, all_controls=(k == 1))
            return True
        if base == "T":
            gate(cols, line, "R" + suffix, nc, 1, 0, all_controls=True)
            code[-1]["params"][0] = 3.0
            return True
        if base in ("SX", "SY"):
            gate(cols, line, base + suffix, nc, 1, 0)
            return True
        if base == "U1":
            gate(cols, line, "U1" + suffix, nc, 1, 1, all_controls=True)
            return True
        if base in ("U2", "U3"):
            gate(cols, line, base + suffix, nc, 1, int(base[1]))
            return True
        if base == "R":
            gate(cols, line, "R" + suffix, nc, 1, 1, exponent=True, all_controls=True)
            return True
        rot = {"+X": "ROTX", "-X": "ROTX_ADJ", "+Y": "ROTY", "-Y": "ROTY_ADJ"}
        if not adj and base in rot:
            gate(cols, line, rot[base], nc, 1, 0)
            return True
        if base == "ESWAP":
            gate(cols, line, "ESWAP" + suffix, nc, 2, 1)
            return True
        if base.startswith("E"):
            for letter in "XYZ":
                k = _count(base[1:], letter)
                if k >= 1:
                    gate(cols, line, "E" + letter + suffix, nc, k, 1)
                    return True
        return False

    done = False
    for line_no, raw in enumerate(text.splitlines(), start=1):
        if done:
            break
        cols = raw.split("!", 1)[0].split()
        if not cols:
            continue
        m = cols[0].upper()
        word = lambda i: cols[i].upper() if i < len(cols) else ""  # noqa: E731
        if m == "QUBITS":
            n = int(cols[1])
            continue
        if m == "CIRCUITS":
            state["num_circuits"] = int(cols[1])
            continue
        if m == "INITIAL":
            init = int(cols[2])
            continue
        if m == "BIT" or m in ("MPIPROCESSES", "MPISWAPBUFFER"):
            continue
        if m == "EXIT":
            ins("EXIT", line_no)
            done = True
        elif m == "BEGIN":
            if word(1) == "MEASUREMENT":
                ins("MEASUREMENT", line_no, ints=[3, 0])
            elif word(1) == "FUSION":
                ins("BEGIN_FUSION", line_no)
            elif word(1) == "CIRCUIT":
                state["circuit"], state["in_circuit"] = int(cols[2]), True
            else:
                raise QcxError("BEGIN")
        elif m == "END":
            if word(1) == "CIRCUIT":
                state["circuit"], state["in_circuit"] = 0, False
            elif word(1) == "FUSION":
                ins("END_FUSION", line_no)
            else:
                raise QcxError("END")
        elif m in ("INNERPROD", "FIDELITY"):
            who = cols[1]
            if who[0].isdigit():
                partner = NONE if int(who) == state["circuit"] else int(who)
            else:
                partner = ALL if who.upper() == "ALL" else NONE
            text, is_var = _operator(cols[2]) if len(cols) >= 4 else ("", 0)
            ins(m, line_no, ints=[partner, is_var], text=text, targets=[qubit(t) for t in cols[3:]])
        elif m == "VAR":
            if cols[2].upper() != "PAULISS":
                raise QcxError(f"line {line_no}: only PAULISS variables")
            ins("VAR", line_no, text=cols[1].upper(), ints=[int(cols[3]) if len(cols) == 4 else 1, 0])
        elif m == "LET":
            ins("LET", line_no, text=cols[1].upper() + " " + cols[3].upper(), ints=[LET_OPS[cols[2]], 0])
        elif m == "DO":
            if word(1) == "MEASUREMENT":
                ins("MEASUREMENT", line_no, ints=[int(cols[2]) if len(cols) == 3 else 3, 0])
            elif word(1) == "AMPLITUDES":
                ins("AMPLITUDES", line_no, values=[int(t) for t in cols[2:]])
            else:
                raise QcxError("DO")
        elif m == "GENERATE":
            ins("GENERATE_EVENTS", line_no, ints=[int(cols[2]), int(cols[3])])
            done = True
        elif m == "EXPECTATION":
            text, is_var = _operator(cols[1])
            ins("EXPECTATION", line_no, text=text, ints=[0, is_var], targets=[qubit(t) for t in cols[2:]])
        elif m in ("PRINT", "PRINTLN"):
            ins("PRINT", line_no, text=" ".join(cols[1:]), ints=[int(m == "PRINTLN"), 0])
        elif m in ("U", "U+"):
            gate(cols, line_no, "R" if m == "U" else "R_ADJ", 0, 2, 1, exponent=True, all_controls=True)
        elif m == "TOFFOLI":
            gate(cols, line_no, "TOFFOLI", 2, 1, 0)
        elif m == "M":
            ins("PROJECTIVE", line_no, targets=[qubit(cols[1])])
        elif m in ("CLEAR", "SET"):
            gate(cols, line_no, m, 0, 1, 0)
        elif m == "SHORBOX":
            nx, div, base = (int(t) for t in cols[1:4])
            ins("GATE", line_no, kind=KG["SHORBOX"], params=[float(nx), float(div), float(base)], ints=[div, base])
        elif plain_or_controlled(cols, line_no, m, 0):
            pass
        elif m.startswith("C") and len(m) >= 2:
            cs = len(m) - len(m.lstrip("C"))
            j = 1
            while j < len(m) and m[j].isdigit():
                j += 1
            if cs > 1:
                nc, rest = cs, m[cs:]
            elif j > 1:
                nc, rest = int(m[1:j]), m[j:]
            else:
                nc, rest = 1, m[1:]
            if nc <= 0 or not rest or not plain_or_controlled(cols, line_no, rest, nc):
                raise QcxError(f"line {line_no}: unknown mnemonic {m}")
        else:
            raise QcxError(f"line {line_no}: unknown mnemonic {m}")
    if n is None:
        raise QcxError("no QUBITS")
    return n, init, code, state["num_circuits"]


# ---- execution on the reference ----------------------------------------------

_FUSIBLE = {"H", "X", "Y", "U2", "U3", "EX", "EY", "EZ", "SWAP"}
_NAME = {v: k for k, v in KG.items()}


def _as_core(g):
    """ORC instruction tuple of oracle.encode() if bra fuses this gate in the reference leg, else None."""
    name, t, c, p = _NAME[g["kind"]], g["targets"], g["controls"], g["params"]
    if name in ("NOT", "X") and len(t) == 1 and len(c) == 1:
        return ("CNOT", (c[0], t[0]), ())
    if name == "Z" and not t and len(c) == 1:
        return ("Z", (c[0],), ())
    if name == "Z" and not t and len(c) == 2:
        return ("CZ", (c[0], c[1]), ())
    if name == "U1" and len(c) == 1:
        return ("U1", (c[0],), (p[0],))
    if name in ("R", "R_ADJ") and len(c) == 2:
        k = int(p[0])
        return ("U", (c[0], c[1]), (-k if name == "R_ADJ" else k,))
    if name in _FUSIBLE and not c and len(t) == (2 if name == "SWAP" else 1):
        npar = {"U2": 2, "U3": 3, "EX": 1, "EY": 1, "EZ": 1}.get(name, 0)
        return (name, tuple(t), tuple(p[:npar]))
    if name == "NOT" and len(t) == 1 and not c:
        return ("X", tuple(t), ())
    return None


def _g(v, precision=6):
    """C++ ostream default floating output (printf %g) at the given precision."""
    return "%.*g" % (precision, v)


def _centre(s, width):
    pad = width - len(s)
    return s if pad <= 0 else " " * (pad // 2) + s + " " * (pad - pad // 2)


def _bits(v, n):
    return format(v, "0%db" % n) if n else ""


class _MT64:
    """std::mt19937_64 (the published MT19937-64 of Nishimura and Matsumoto:
    w = 64, n = 312, m = 156, r = 31), for the per-circuit seeds bra draws."""
    N, M = 312, 156
    MASK = (1 << 64) - 1

    def __init__(self, seed):
        self.mt = [seed & self.MASK]
        for i in range(1, self.N):
            prev = self.mt[-1]
            self.mt.append((6364136223846793005 * (prev ^ (prev >> 62)) + i) & self.MASK)
        self.i = self.N

    def __call__(self):
        if self.i >= self.N:
            upper, lower = 0xFFFFFFFF80000000, 0x7FFFFFFF
            for k in range(self.N):
                x = (self.mt[k] & upper) | (self.mt[(k + 1) % self.N] & lower)
                xa = (x >> 1) ^ (0xB5026F5AA96619E9 if x & 1 else 0)
                self.mt[k] = self.mt[(k + self.M) % self.N] ^ xa
            self.i = 0
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & self.MASK


# ---- PAULISS values (bra/include/bra/pauli_string_space.hpp:25-153; LET and
# variable lookup as bra/src/state.cpp:400-490, :977-998): (num_qubits, {string: coeff}).

def _new_space():
    return [0, {"": 0j}]


def _variable(c, ref):
    name, _, idx = ref.partition(":")
    if name not in c["vars"]:
        raise QcxError(f"{name} is not a PAULISS variable")
    return c["vars"][name][int(idx) if idx else 0]


def _space_value(c, rhs):
    if rhs.startswith(":PAULIS:"):
        s = rhs[len(":PAULIS:"):]
        return [len(s), {s: 1 + 0j}]
    v = _variable(c, rhs)
    return [v[0], dict(v[1])]


def _complex_value(c, rhs):
    fixed = {":COMPLEX": 0j, ":I": 1j, ":MINUS_I": -1j}
    if rhs in fixed:
        return fixed[rhs]
    if rhs == ":RESULT":
        return c["result"]
    if rhs.startswith(":COMPLEX:"):
        return complex(float(rhs[len(":COMPLEX:"):]), 0.0)
    raise QcxError(f"unsupported complex value {rhs}")


def _let(c, ins):
    lhs_ref, rhs = ins["text"].split(" ")
    lhs = _variable(c, lhs_ref)
    op = ins["ints"][0]
    if op == 0:
        lhs[:] = _space_value(c, rhs)
    elif op in (1, 2):
        for s, v in _space_value(c, rhs)[1].items():
            if len(s) != lhs[0]:
                raise QcxError(f"{s} has the wrong length")
            lhs[1][s] = lhs[1].get(s, 0j) + (v if op == 1 else -v)
    else:
        z = _complex_value(c, rhs)
        for s in lhs[1]:
            lhs[1][s] = lhs[1][s] * z if op == 3 else lhs[1][s] / z


def _terms(c, ins):
    """The operator of an instruction as [(string over the listed qubits, coefficient)]."""
    if not ins["ints"][1]:
        return [(ins["text"], 1 + 0j)]
    nq, terms = _variable(c, ins["text"])
    if nq != len(ins["targets"]):
        raise QcxError("operator length differs from the number of qubits")
    return list(terms.items())


def _overlap(a, b, ins, owner):
    """ket::inner_product(a, b[, P]) = <b| [P] |a> (squared modulus for FIDELITY) on the reference; the
    operator is circuit owner's."""
    if ins["text"]:
        v = sum(w * a.inner_product_on(b, s, ins["targets"]) for s, w in _terms(owner, ins))
    else:
        v = a.inner_product(b)
    return complex(abs(v) ** 2, 0.0) if ins["op"] == OP["FIDELITY"] else v


def _run_circuit(c, n, out):
    """Runs circuit context c until it finishes or waits (bra::interpreter::apply_circuit)."""
    r, code = c["r"], c["code"]
    while c["pc"] < len(code) and c["wait"] is None:
        i = c["pc"]
        ins = code[i]
        op = ins["op"]
        c["pc"] = i + 1
        if op == OP["BEGIN_FUSION"]:
            j = i + 1
            while j < len(code) and code[j]["op"] != OP["END_FUSION"]:
                j += 1
            block = code[i + 1:j]
            cores = [_as_core(g) if g["op"] == OP["GATE"] else None for g in block]
            if block and all(cores):
                r.apply([("BEGIN FUSION", (), ())] + cores + [("END FUSION", (), ())])
                c["pc"] = j + 1
            continue
        if op == OP["END_FUSION"] or op == OP["NOOP"]:
            pass
        elif op == OP["GATE"]:
            r.gate(ins["kind"], ins["targets"], ins["controls"], ins["params"])
        elif op == OP["MEASUREMENT"]:
            p = ins["ints"][0]
            spins = r.spins().reshape(n, 3)
            out.append("Expectation values of spins:\n")
            if p > 0:
                w = max(p + 3, 8)
                out.append(" ".join(_centre(s, w) for s in ("<Qx>", "<Qy>", "<Qz>")) + "\n")
                for q in range(n):
                    out.append(" ".join(_centre("% .*f" % (p, 0.5 - spins[q, k]), w) for k in range(3)) + "\n")
            else:
                out.append("<Qx> <Qy> <Qz>\n")
                prec = -p if p < 0 else 6
                for q in range(n):
                    out.append(" ".join(_g(0.5 - spins[q, k], prec) for k in range(3)) + "\n")
        elif op == OP["AMPLITUDES"]:
            a = r.amplitudes()
            idx = ins["values"] or range(1 << n)
            for k in idx:
                out.append("%s => %s + %s i\n" % (_bits(k, n), _g(a[k].real), _g(a[k].imag)))
        elif op == OP["GENERATE_EVENTS"]:
            ev = r.generate_events(ins["ints"][0], ins["ints"][1])
            out.append("Events:\n")
            out.extend("%d %s\n" % (k, _bits(int(e), n)) for k, e in enumerate(ev))
        elif op == OP["EXIT"]:
            out.append("Measurement result: %d\n" % r.measure())
        elif op == OP["PROJECTIVE"]:
            q = ins["targets"][0]
            c["outcomes"][q] = r.projective_measurement(q)
            c["last"] = q
        elif op == OP["EXPECTATION"]:
            c["result"] = sum(w * r.expectation_on(s, ins["targets"]) for s, w in _terms(c, ins))
        elif op == OP["VAR"]:
            if ins["text"] in c["vars"]:
                raise QcxError(f"variable {ins['text']} declared twice")
            c["vars"][ins["text"]] = [_new_space() for _ in range(ins["ints"][0])]
        elif op == OP["LET"]:
            _let(c, ins)
        elif op in (OP["INNERPROD"], OP["FIDELITY"]):
            if ins["ints"][0] != NONE:
                c["wait"] = ins
        elif op == OP["PRINT"]:
            parts = []
            result = c["result"]
            for a in ins["text"].split():
                if a[0].isdigit() or a[0] in "+-.":
                    parts.append(a)
                elif a == ":RESULT":
                    parts.append("(%s,%s)" % (_g(result.real), _g(result.imag)))
                elif a == ":OUTCOME":
                    parts.append(str(c["outcomes"][c["last"]]))
                elif a.startswith(":OUTCOMES:"):
                    parts.append(str(c["outcomes"][int(a[10:])]))
                elif a in CONSTANTS:
                    parts.append(_g(CONSTANTS[a]))
            out.append(" ".join(parts) + ("\n" if ins["ints"][0] else ""))


def _kind(w):
    return (2 if w["op"] == OP["FIDELITY"] else 0) + (1 if w["text"] else 0) + (4 if w["ints"][0] == ALL else 0)


def run(text, seed=1, threads=1):
    """Returns (output text without timing lines, circuit 0's final amplitudes,
    circuit 0's reference state).  Several circuits run as bra's nompi
    scheduler runs them (bra/src/bra.cpp:299-760): circuit 0 seeded with
    `seed`, circuit k >= 1 with the k-th draw of std::mt19937_64(seed); each
    runs until it waits on an INNERPROD / FIDELITY, then the pairs that wait
    on each other are evaluated in circuit order, or the ALL form once every
    circuit waits on it."""
    n, init, code, nc = parse_program(text)
    draws = _MT64(seed)
    ctx = []
    for k in range(nc):
        r = oracle.KetRef(n, initial_index=init, threads=threads)
        r.seed(seed if k == 0 else draws())
        ctx.append(dict(r=r, code=[i for i in code if i["circuit"] == k], pc=0, outcomes=[-1] * n, last=0,
                        result=0j, wait=None, vars={}))
    out = []
    while True:
        for c in ctx:
            if c["wait"] is None:
                _run_circuit(c, n, out)
        if all(c["wait"] is None for c in ctx):
            break
        progress, all_kind, all_same = False, None, True
        for k, c in enumerate(ctx):
            if c["wait"] is None:
                all_same = False
                continue
            kind = _kind(c["wait"])
            if kind >= 4:
                if all_kind is None:
                    all_kind = kind
                elif all_kind != kind:
                    all_same = False
                continue
            all_same = False
            o = ctx[c["wait"]["ints"][0]]
            if o["wait"] is None or _kind(o["wait"]) != kind or o["wait"]["ints"][0] != k:
                continue
            v = _overlap(c["r"], o["r"], c["wait"], c)
            c["result"], o["result"] = v, v.conjugate()
            c["wait"] = o["wait"] = None
            progress = True
        if not progress and all_same and all_kind is not None:
            w = ctx[0]["wait"]
            for c in ctx:
                c["result"] = _overlap(ctx[0]["r"], c["r"], w, ctx[0])
            for c in ctx:
                c["wait"] = None
            progress = True
        if not progress:
            raise QcxError("circuits wait on partners that never arrive")
    return "".join(out), ctx[0]["r"].amplitudes(), ctx[0]["r"]
