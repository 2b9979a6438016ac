"""Seeded synthetic workloads, as lists of bra .qcx instructions.

An instruction is ``(mnemonic, qubits, params)`` with the bra mnemonics of the
hot path (bra/src/interpreter.cpp:513-640): ``H t``, ``X t``, ``Y t``, ``Z c``,
``U1 c lambda``, ``U2 t phi lambda``, ``U3 t theta phi lambda``, ``CNOT c t``,
``CZ c1 c2``, ``U c1 c2 k``, ``EY t theta``, ``EZ t theta``, ``SWAP t1 t2``,
``BEGIN FUSION`` / ``END FUSION``.  The reference ships no benchmark suite for
this path, so all workloads are generated here from a seed; ``to_qcx`` prints a
circuit in bra's text format with round-trip exact angles.
"""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 2.0 * math.pi


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def brick(n, depth, seed=1, fuse_k=0):
    """H on every qubit, then `depth` brick layers: U3(theta, phi, lambda) on
    every qubit (angles i.i.d. uniform [0, 2 pi)), then CNOT c=i t=i+1 for even
    i on even layers and odd i on odd layers.

    fuse_k > 0 wraps the gates in BEGIN/END FUSION blocks of at most fuse_k
    qubits (each block: the U3s of its qubits, then its CNOTs; blocks of one
    layer act on disjoint qubits)."""
    rng = _rng(seed)
    ops = []
    if fuse_k:
        for a in range(0, n, fuse_k):
            ops.append(("BEGIN FUSION", (), ()))
            ops += [("H", (q,), ()) for q in range(a, min(n, a + fuse_k))]
            ops.append(("END FUSION", (), ()))
    else:
        ops += [("H", (q,), ()) for q in range(n)]
    for layer in range(depth):
        angles = rng.uniform(0.0, TWO_PI, size=(n, 3))
        start = layer % 2
        pairs = [(i, i + 1) for i in range(start, n - 1, 2)]
        if not fuse_k:
            ops += [("U3", (q,), tuple(float(x) for x in angles[q])) for q in range(n)]
            ops += [("CNOT", (c, t), ()) for c, t in pairs]
            continue
        # units: CNOT pairs and lone qubits, packed into blocks of <= fuse_k qubits
        units, q = [], 0
        while q < n:
            if (q, q + 1) in pairs:
                units.append((q, q + 1))
                q += 2
            else:
                units.append((q,))
                q += 1
        blocks, cur = [], []
        for u in units:
            if sum(len(x) for x in cur) + len(u) > fuse_k:
                blocks.append(cur)
                cur = []
            cur.append(u)
        if cur:
            blocks.append(cur)
        for blk in blocks:
            ops.append(("BEGIN FUSION", (), ()))
            for u in blk:
                for qq in u:
                    ops.append(("U3", (qq,), tuple(float(x) for x in angles[qq])))
            for u in blk:
                if len(u) == 2:
                    ops.append(("CNOT", u, ()))
            ops.append(("END FUSION", (), ()))
    return ops


def qft_brick(n, brick_layers=5, seed=1, fuse_k=0):
    """For j = 0..n-1: H j, then U m j k with k = m - j + 1 for every m > j
    (phase 2 pi / 2^k on |1_m 1_j>, all n(n-1)/2 pairs), then seeded brick layers.

    fuse_k > 0 groups the qubits in consecutive blocks of fuse_k: each block's H
    and in-block phases form one BEGIN/END FUSION block, followed by the block's
    phases towards later qubits (diagonal, so they commute with the rest of the
    block and may leave it); the brick layers come in fusion blocks as in brick()."""
    ops = []
    if not fuse_k:
        for j in range(n):
            ops.append(("H", (j,), ()))
            for m in range(j + 1, n):
                ops.append(("U", (m, j), (m - j + 1,)))
        ops += [op for op in brick(n, brick_layers, seed=seed)[n:]]
        return ops
    for a in range(0, n, fuse_k):
        b = min(n, a + fuse_k)
        ops.append(("BEGIN FUSION", (), ()))
        for j in range(a, b):
            ops.append(("H", (j,), ()))
            for m in range(j + 1, b):
                ops.append(("U", (m, j), (m - j + 1,)))
        ops.append(("END FUSION", (), ()))
        for j in range(a, b):
            for m in range(b, n):
                ops.append(("U", (m, j), (m - j + 1,)))
    layers = brick(n, brick_layers, seed=seed, fuse_k=fuse_k)
    first_layer = next(i for i, op in enumerate(layers) if op[0] == "U3") - 1  # skip the H blocks
    ops += layers[first_layer:]
    return ops


def ansatz(n, layers, seed=1, thetas=None):
    """Hardware-efficient ansatz: per layer RY(theta) on every qubit, RZ(theta)
    on every qubit, then CZ(i, i+1 mod n) for all i.  RY/RZ are written as bra's
    `EY t -theta/2` / `EZ t -theta/2` (exp(i phi P) with phi = -theta/2).
    Returns (ops, thetas) with 2*n*layers parameters uniform in [-pi, pi)."""
    if thetas is None:
        thetas = _rng(seed).uniform(-math.pi, math.pi, size=2 * n * layers)
    thetas = np.asarray(thetas, dtype=np.float64)
    ops, k = [], 0
    for _ in range(layers):
        for q in range(n):
            ops.append(("EY", (q,), (-0.5 * float(thetas[k]),)))
            k += 1
        for q in range(n):
            ops.append(("EZ", (q,), (-0.5 * float(thetas[k]),)))
            k += 1
        for i in range(n):
            ops.append(("CZ", (i, (i + 1) % n), ()))
    return ops, thetas


def ansatz_hamiltonian(n):
    """H = sum_i Z_i Z_{i+1} + 0.5 sum_i X_i (periodic), as (string, coeff)
    terms with character k acting on qubit k."""
    terms = []
    for i in range(n):
        s = ["I"] * n
        s[i] = "Z"
        s[(i + 1) % n] = "Z"
        terms.append(("".join(s), 1.0))
    for i in range(n):
        s = ["I"] * n
        s[i] = "X"
        terms.append(("".join(s), 0.5))
    return terms


def inverse(ops):
    """The exact inverse of an instruction list: gates reversed and each
    replaced by its adjoint (U3(t, p, l)^-1 = U3(-t, -l, -p), U m j k -> U m j -k,
    EX/EY/EZ and U1 with the negated angle; H, X, Y, Z, CNOT, CZ, SWAP are their
    own inverses).  Fusion markers keep their places around the reversed gates."""
    out = []
    for mnem, q, p in reversed(ops):
        if mnem == "BEGIN FUSION":
            out.append(("END FUSION", (), ()))
        elif mnem == "END FUSION":
            out.append(("BEGIN FUSION", (), ()))
        elif mnem == "U3":
            out.append(("U3", q, (-p[0], -p[2], -p[1])))
        elif mnem == "U":
            out.append(("U", q, (-p[0],)))
        elif mnem in ("U1", "EX", "EY", "EZ"):
            out.append((mnem, q, (-p[0],)))
        elif mnem == "U2":
            out.append(("U3", q, (-math.pi / 2, -p[1], -p[0])))
        elif mnem in ("H", "X", "Y", "Z", "CNOT", "CZ", "SWAP"):
            out.append((mnem, q, p))
        else:
            raise ValueError(f"no inverse for {mnem}")
    return out


def batch_instances(count=4096, n_min=10, n_max=24, depth_min=4, depth_max=16, seed_base=1):
    """Config-5 style batch: instance i draws, from its own generator seeded
    seed_base + i, a qubit count n = round(exp(U[ln n_min, ln n_max])), a depth
    U{depth_min..depth_max} and 2 n depth ansatz parameters U[-pi, pi).
    Returns a list of (n, layers, thetas)."""
    out = []
    for i in range(count):
        rng = _rng(seed_base + i)
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        layers = int(rng.integers(depth_min, depth_max + 1))
        thetas = rng.uniform(-math.pi, math.pi, size=2 * n * layers)
        out.append((n, layers, thetas))
    return out


def random_circuit(n, count, seed=1, kinds=None):
    """Random mix of the hot-path instructions (parity tests)."""
    rng = _rng(seed)
    kinds = kinds or ["H", "X", "Y", "Z", "U1", "U2", "U3", "CNOT", "CZ", "U", "EX", "EY", "EZ", "SWAP"]
    ops = []
    for _ in range(count):
        k = kinds[int(rng.integers(len(kinds)))]
        q = [int(x) for x in rng.permutation(n)[:2]]
        a = [float(x) for x in rng.uniform(0.0, TWO_PI, size=3)]
        if k in ("H", "X", "Y", "Z"):
            ops.append((k, (q[0],), ()))
        elif k in ("U1", "EX", "EY", "EZ"):
            ops.append((k, (q[0],), (a[0],)))
        elif k == "U2":
            ops.append((k, (q[0],), (a[0], a[1])))
        elif k == "U3":
            ops.append((k, (q[0],), tuple(a)))
        elif k in ("CNOT", "CZ", "SWAP"):
            ops.append((k, (q[0], q[1]), ()))
        elif k == "U":
            kk = int(rng.integers(1, n + 1))
            ops.append((k, (q[0], q[1]), (kk if rng.random() < 0.7 else -kk,)))
    return ops


def reference_passes(ops):
    """State passes the reference takes for a circuit: one per fusion block and
    one per gate outside a block (bra/src/nompi_state.cpp:1285-1357)."""
    passes, in_block = 0, False
    for mnem, _, _ in ops:
        if mnem == "BEGIN FUSION":
            in_block = True
        elif mnem == "END FUSION":
            in_block = False
            passes += 1
        elif not in_block:
            passes += 1
    return passes


def to_qcx(n, ops):
    """bra .qcx text (angles with 17 significant digits: exact round trip)."""
    lines = [f"QUBITS {n}"]
    for mnem, qubits, params in ops:
        words = [mnem] + [str(q) for q in qubits]
        words += [str(int(p)) if mnem == "U" else repr(float(p)) for p in params]
        lines.append(" ".join(words))
    return "\n".join(lines) + "\n"
