"""States sharded over ranks by global qubits (riken-braket_b200/global_qubits.py,
ket::mpi's simple_mpi policy): the distribution logic -- layout map, exchanges of
half shards, controls and phases on global qubits, gathering -- on 2 and 4 gloo
ranks on the CPU, each shard held by the oracle's C restatement; and on one GPU,
two ranks in one process (two engine shards, exchanges as device copies).
Every result must equal the whole state run by the oracle."""
import os
import socket
import sys
import threading

import numpy as np
import pytest

from conftest import ROOT

N_CPU = 8


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def random_program(n, count, seed):
    """Every instruction kind the sharded state takes, on every qubit (global ones included)."""
    rng = np.random.default_rng(seed)
    ops = [("H", (q,), ()) for q in range(n)]
    for _ in range(count):
        k = rng.integers(0, 13)
        a, b = (int(x) for x in rng.choice(n, size=2, replace=False))
        ang = tuple(float(x) for x in rng.uniform(-np.pi, np.pi, size=3))
        if k == 0:
            ops.append(("U3", (a,), ang))
        elif k == 1:
            ops.append(("CNOT", (a, b), ()))
        elif k == 2:
            ops.append(("CZ", (a, b), ()))
        elif k == 3:
            ops.append(("U1", (a,), ang[:1]))
        elif k == 4:
            ops.append(("U", (a, b), (int(rng.integers(-n, n + 1)) or 1,)))
        elif k == 5:
            ops.append(("EZ", (a,), ang[:1]))
        elif k == 6:
            ops.append(("SWAP", (a, b), ()))
        elif k == 7:
            ops.append(("EX", (a,), ang[:1]))
        elif k == 8:
            ops.append(("EY", (a,), ang[:1]))
        elif k == 9:
            ops.append(("U2", (a,), ang[:2]))
        elif k == 10:
            ops.append(("Y", (a,), ()))
        elif k == 11:
            ops.append(("Z", (a,), ()))
        else:
            ops.append(("X", (a,), ()))
    return ops


class OracleShard:
    """Test shard: the oracle's C restatement holds the local qubits (host memory)."""

    def __init__(self, nl):
        import oracle
        import torch

        self.torch = torch
        self.o = oracle.COracle(nl)
        self.n = nl
        self.buf = None

    def apply(self, ops):
        self.o.apply(ops)

    def phase(self, coeff, qubits):
        a = self.o.amplitudes()
        mask = sum(1 << q for q in qubits)
        idx = np.arange(a.size)
        a[(idx & mask) == mask] *= coeff
        self.o.set_amplitudes(a)

    def reset(self, index):
        a = np.zeros(1 << self.n, dtype=np.complex128)
        if index is not None:
            a[index] = 1.0
        self.o.set_amplitudes(a)

    def half(self, upper):
        self.buf = np.ascontiguousarray(self.o.amplitudes())
        half = self.buf.size // 2
        return self.torch.from_numpy(self.buf[half:] if upper else self.buf[:half]).view(self.torch.uint8)

    def recv_buffer(self, like):
        return self.torch.empty_like(like)

    def store(self, view, data):
        view.copy_(data)
        self.o.set_amplitudes(self.buf)

    def norm2(self):
        return float(np.vdot(self.o.amplitudes(), self.o.amplitudes()).real)

    def amplitudes(self):
        return self.o.amplitudes()

    def close(self):
        pass


def _cpu_rank(rank, world, port, n, seed, init):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime

    import torch.distributed as dist

    import oracle
    from __graft_entry__ import load_package

    gq = load_package().global_qubits
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        comm = gq.TorchComm()
        st = gq.DistributedState(n, comm, shard=OracleShard(n - (world.bit_length() - 1)), initial_index=init)
        ops = random_program(n, 120, seed)
        st.apply(ops)
        got = st.amplitudes()
        ref = oracle.COracle(n, initial_index=init)
        ref.apply(ops)
        want = ref.amplitudes()
        err = np.abs(got - want).max()
        assert err <= 1e-12, (rank, err)
        assert abs(st.norm2() - 1.0) <= 1e-12
        assert st.exchanges > 0
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("seed", [1, 2])
def test_sharded_state_on_gloo_ranks_equals_whole_state(world, seed):
    import torch.multiprocessing as mp

    mp.spawn(_cpu_rank, args=(world, free_port(), N_CPU, seed, 37 * seed), nprocs=world, join=True)


def test_layout_map_only_for_swaps():
    """SWAP never moves data: it changes the layout map only (one rank, no communication)."""
    sys.path.insert(0, ROOT)
    from __graft_entry__ import load_package

    gq = load_package().global_qubits

    class One:
        rank, size = 0, 1

        def sum(self, v):
            return v

        def gather(self, a):
            return [a]

    st = gq.DistributedState(5, One(), shard=OracleShard(5))
    st.apply([("SWAP", (0, 4), ()), ("SWAP", (1, 4), ())])
    assert st.perm == [4, 0, 2, 3, 1] and st.exchanges == 0


class LoopComm:
    """Ranks as threads of one process: exchanges and sums through a shared board."""

    def __init__(self, rank, size, board, barrier):
        self.rank, self.size, self.board, self.barrier = rank, size, board, barrier

    def exchange(self, send, recv, partner):
        self.board[self.rank] = send.clone()
        self.barrier.wait()
        recv.copy_(self.board[partner])
        self.barrier.wait()

    def sum(self, value):
        self.board[self.rank] = value
        self.barrier.wait()
        total = sum(self.board[r] for r in range(self.size))
        self.barrier.wait()
        return total

    def gather(self, array):
        self.board[self.rank] = array
        self.barrier.wait()
        out = [self.board[r] for r in range(self.size)]
        self.barrier.wait()
        return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_engine_shards_exchange_on_one_gpu(pkg, precision):
    """Two ranks on one GPU (threads of one process): engine shards, half-shard
    exchanges through device views of the engine's memory, against the oracle."""
    import oracle

    gq = pkg.global_qubits
    n, size = 14, 2
    ops = random_program(n, 200, 7 + precision)
    board, barrier = {}, threading.Barrier(size, timeout=120)
    results, errors = {}, []

    def rank_main(rank):
        try:
            st = gq.DistributedState(n, LoopComm(rank, size, board, barrier), precision=precision, initial_index=5)
            st.apply(ops)
            results[rank] = (st.amplitudes(), st.norm2(), st.exchanges)
            st.close()
        except Exception as e:  # noqa: BLE001 -- reported below
            errors.append(e)
            barrier.abort()

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(size)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    ref = oracle.COracle(n, initial_index=5)
    ref.apply(ops)
    tol = 1e-12 if precision == 0 else 2e-5
    for r in range(size):
        got, norm2, exchanges = results[r]
        assert np.abs(got.astype(np.complex128) - ref.amplitudes()).max() <= tol
        assert abs(norm2 - 1.0) <= (1e-12 if precision == 0 else 1e-4)
        assert exchanges > 0


def _bench_rank(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(dist, 0)
        assert bench.dist_max(dist, 1.5 * (rank + 1), 0) == 1.5 * world
        bench.barrier(dist, 0)
    finally:
        dist.destroy_process_group()


def test_bench_timing_is_the_max_over_gloo_ranks():
    """bench.py's N > 1 plumbing (barrier, max over ranks) on 2 gloo ranks."""
    import torch.multiprocessing as mp

    mp.spawn(_bench_rank, args=(2, free_port()), nprocs=2, join=True)
