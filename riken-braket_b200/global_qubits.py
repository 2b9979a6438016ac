"""A state vector sharded over 2^g ranks by its global qubits: ket::mpi's
simple_mpi policy with one process per GPU.

Rank r holds the 2^(n-g) amplitudes whose top g physical qubits spell r
(ket/include/ket/mpi/utility/simple_mpi.hpp: global_qubit_value, rank), in an
engine state of n - g local qubits.  A layout map (ket::mpi::qubit_permutation,
qubit_permutation.hpp:40-302) sends logical qubits to physical bits; bits
0 .. n-g-1 are local, bits n-g .. n-1 are global.

Gates follow ket::mpi::gate (simple_mpi.hpp:601-782), with one difference of
B200 design: only a NON-DIAGONAL target has to be local.
  * A non-diagonal target on a global bit is first made local:
    maybe_interchange_qubits / interchange_qubits
    (mpi/utility/simple_mpi.hpp:598-690, mpi/utility/detail/interchange_qubits.hpp:29-107).
    The local qubit it trades places with is moved to the top local bit, so the
    half of the shard that changes ranks is one contiguous block.  Each rank
    sends that block to its partner and receives the partner's in one grouped
    send/receive (NCCL over NVLink, gloo on the host): 2^(n-g-1) amplitudes
    each way, the reference's volume.
  * Controls and diagonal factors on global bits need no data: they are known
    per rank.  A control on a global bit that is 0 on this rank skips the gate
    here; one that is 1 is dropped.  A phase on |1..1> of qubits that are all
    global becomes a factor on the whole shard of the ranks where they are all
    1, and EZ on a global qubit is e^{i theta} or e^{-i theta} on the whole shard.
  * SWAP of two logical qubits only exchanges their entries in the layout map.
Observables reduce per shard and sum over ranks.

The shard is any object with the small interface of `EngineShard` (the
engine's state on this rank's GPU); the communicator is `TorchComm` over
torch.distributed (NCCL for GPU tensors, gloo for host tensors).
"""
from __future__ import annotations

import cmath
import math

import numpy as np

from . import rbk

# One non-diagonal target (index into the qubit tuple), or None.
_TARGET = {"H": 0, "X": 0, "Y": 0, "U2": 0, "U3": 0, "EX": 0, "EY": 0, "CNOT": 1}
# Phase c on |1..1> of every listed qubit (ket's all-control phase gates).
_PHASE = {"Z", "CZ", "U1", "U"}


def _phase_coeff(mnem, params):
    if mnem in ("Z", "CZ"):
        return -1.0 + 0.0j
    if mnem == "U1":  # ket::gate::phase_shift: exp_i(phase)
        return cmath.exp(1j * params[0])
    k = int(params[0])  # bra's U c1 c2 k: exp_i(2 pi / 2^k), conjugated for k < 0
    c = cmath.exp(1j * (2.0 * math.pi / float(1 << abs(k))))
    return c.conjugate() if k < 0 else c


class TorchComm:
    """torch.distributed plumbing: one grouped send/receive with a partner, sums, gathers."""

    def __init__(self, group=None):
        import torch
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        # NCCL reduces device tensors, gloo host tensors
        self.device = f"cuda:{torch.cuda.current_device()}" if dist.get_backend(group) == "nccl" else "cpu"

    def exchange(self, send, recv, partner):
        d = self.dist
        ops = [d.P2POp(d.isend, send, partner, self.group), d.P2POp(d.irecv, recv, partner, self.group)]
        for req in d.batch_isend_irecv(ops):
            req.wait()

    def sum(self, value):
        import torch

        t = torch.tensor([value], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())

    def gather(self, array):
        import torch

        t = torch.as_tensor(np.ascontiguousarray(array).view(np.uint8)).to(self.device)
        out = [torch.empty_like(t) for _ in range(self.size)]
        self.dist.all_gather(out, t, group=self.group)
        return [o.cpu().numpy().view(array.dtype) for o in out]


class _DeviceBytes:
    """A device range as a __cuda_array_interface__ object (zero-copy torch view)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


class EngineShard:
    """This rank's shard: an rbk.State of the local qubits on one GPU."""

    def __init__(self, num_local_qubits, precision=rbk.C128, device=0):
        import torch

        self.torch = torch
        self.device = device
        self.n = num_local_qubits
        self.precision = precision
        self.amp_bytes = 16 if precision == rbk.C128 else 8
        self.state = rbk.State(num_local_qubits, precision, device=device)
        self._recv = None

    def apply(self, ops):
        self.state.apply(ops)

    def phase(self, coeff, qubits):
        if qubits:
            self.state.phase_shift_coeff(coeff, *qubits)
        else:
            self.state.apply_diagonal2(coeff, coeff, 0)

    def diagonal(self, d0, d1, target):
        self.state.apply_diagonal2(d0, d1, target)

    def reset(self, index):
        """|index> of the local qubits, or the zero vector for index None."""
        self.state.reset(0 if index is None else index)
        if index is None:
            self.state.apply_diagonal2(0.0, 0.0, 0)

    def half(self, upper):
        """Zero-copy device view of the amplitudes whose top local bit is `upper`
        (the engine's layout made canonical first)."""
        self.state.canonicalize()
        self.state.synchronize()
        half_bytes = (self.amp_bytes << self.n) // 2
        ptr = self.state.device_pointer() + (half_bytes if upper else 0)
        with self.torch.cuda.device(self.device):
            return self.torch.as_tensor(_DeviceBytes(ptr, half_bytes), device=f"cuda:{self.device}")

    def recv_buffer(self, like):
        if self._recv is None or self._recv.numel() != like.numel():
            self._recv = self.torch.empty_like(like)
        return self._recv

    def store(self, view, data):
        view.copy_(data)
        self.torch.cuda.current_stream(self.device).synchronize()

    def norm2(self):
        return self.state.norm2()

    def amplitudes(self):
        self.state.canonicalize()
        return self.state.amplitudes()

    def close(self):
        self.state.close()


class DistributedState:
    """n logical qubits over comm.size ranks (a power of two): ket::mpi::state
    with the simple_mpi policy.  `shard` holds this rank's n - g local qubits."""

    def __init__(self, num_qubits, comm, shard=None, precision=rbk.C128, device=0, initial_index=0):
        size = comm.size
        if size < 1 or size & (size - 1):
            raise ValueError("the number of ranks must be a power of two")
        self.comm = comm
        self.n = num_qubits
        self.g = size.bit_length() - 1
        self.nl = num_qubits - self.g
        if self.nl < 2:
            raise ValueError("each rank needs at least two local qubits")
        self.shard = shard if shard is not None else EngineShard(self.nl, precision, device)
        self.perm = list(range(num_qubits))  # logical -> physical
        self.inv = list(range(num_qubits))   # physical -> logical
        self.exchanges = 0
        self.reset(initial_index)

    # ---- layout -------------------------------------------------------------
    def _global_bit(self, physical):
        """This rank's value of a global physical bit."""
        return (self.comm.rank >> (physical - self.nl)) & 1

    def _is_local(self, q):
        return self.perm[q] < self.nl

    def _make_local(self, q, keep):
        """interchange_qubits: trade the global qubit q for a local one that is
        not in `keep` (moved to the top local bit first)."""
        pg = self.perm[q]
        used = {self.perm[k] for k in keep if self._is_local(k)}
        top = self.nl - 1
        pl = next(p for p in range(top, -1, -1) if p not in used)
        if pl != top:  # bring the chosen local qubit to the top local bit (a layout swap inside the shard)
            self.shard.apply([("SWAP", (pl, top), ())])
            a, b = self.inv[pl], self.inv[top]
            self.perm[a], self.perm[b] = top, pl
            self.inv[pl], self.inv[top] = b, a
        bit = self._global_bit(pg)
        partner = self.comm.rank ^ (1 << (pg - self.nl))
        # the half whose top local bit differs from this rank's global bit changes ranks
        view = self.shard.half(upper=1 - bit)
        recv = self.shard.recv_buffer(view)
        self.comm.exchange(view, recv, partner)
        self.shard.store(view, recv)
        moved = self.inv[top]
        self.perm[q], self.perm[moved] = top, pg
        self.inv[top], self.inv[pg] = q, moved
        self.exchanges += 1

    # ---- gates --------------------------------------------------------------
    def reset(self, index=0):
        """|index> in logical qubits (the layout map returns to the identity)."""
        self.perm = list(range(self.n))
        self.inv = list(range(self.n))
        local, owner = index & ((1 << self.nl) - 1), index >> self.nl
        self.shard.reset(local if owner == self.comm.rank else None)

    def apply(self, ops):
        """Applies bra instruction tuples (see circuits.py) in logical qubits."""
        for mnem, q, p in ops:
            if mnem in ("BEGIN FUSION", "END FUSION"):
                continue  # the engine fuses queued gates by itself
            if mnem == "SWAP":
                a, b = q
                pa, pb = self.perm[a], self.perm[b]
                self.perm[a], self.perm[b] = pb, pa
                self.inv[pa], self.inv[pb] = b, a
                continue
            if mnem in _PHASE:
                self._phase(_phase_coeff(mnem, p), q)
                continue
            if mnem == "EZ" and not self._is_local(q[0]):
                if self._global_bit(self.perm[q[0]]):
                    self.shard.phase(cmath.exp(-1j * p[0]), [])
                else:
                    self.shard.phase(cmath.exp(1j * p[0]), [])
                continue
            if mnem == "EZ":
                self.shard.apply([(mnem, (self.perm[q[0]],), p)])
                continue
            if mnem not in _TARGET:
                raise ValueError(f"unsupported instruction {mnem}")
            t = q[_TARGET[mnem]]
            if not self._is_local(t):
                self._make_local(t, q)
            if mnem == "CNOT":
                c = q[0]
                if not self._is_local(c):
                    if self._global_bit(self.perm[c]):
                        self.shard.apply([("X", (self.perm[t],), ())])
                    continue
                self.shard.apply([("CNOT", (self.perm[c], self.perm[t]), ())])
                continue
            self.shard.apply([(mnem, (self.perm[t],), p)])

    def _phase(self, coeff, qubits):
        local = []
        for q in qubits:
            if self._is_local(q):
                local.append(self.perm[q])
            elif not self._global_bit(self.perm[q]):
                return  # a global control is 0 on this rank
        self.shard.phase(coeff, local)

    # ---- observables ----------------------------------------------------------
    def norm2(self):
        return self.comm.sum(self.shard.norm2())

    def amplitudes(self):
        """All 2^n amplitudes in logical order, on every rank (for checks at small n)."""
        parts = self.comm.gather(np.ascontiguousarray(self.shard.amplitudes()))
        phys = np.concatenate(parts)  # physical index = (rank << nl) | local index
        # axis k of the reshaped array is physical bit n-1-k; reorder to logical bits
        t = phys.reshape([2] * self.n)
        axes = [self.n - 1 - self.perm[self.n - 1 - k] for k in range(self.n)]
        return np.ascontiguousarray(np.transpose(t, axes)).reshape(-1)

    def close(self):
        self.shard.close()
