"""Dense k-qubit unitaries (rbk_apply_unitary): the tensor-core 3xTF32 path for
complex<float> (k = 5, 6) and the CUDA-core path otherwise, against numpy in
FP64; and the tensor-core fusion mode against the FP64 state.  Tolerances:
complex<double> 1e-12; complex<float> tensor-core unitaries 2e-7 max amplitude
error and normalised fidelity >= 1 - 1e-11 (3xTF32 products carry the FP32
result); whole complex<float> circuits 2e-5 and 1 - 1e-9."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return a / np.linalg.norm(a)


def random_unitary(k, seed):
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def apply_numpy(a, u, qubits, n):
    """u[r][c] = <r|U|c>, bit i of the local index = qubits[i]."""
    k = len(qubits)
    t = a.reshape([2] * n)  # axis j <-> bit n-1-j
    axes = [n - 1 - q for q in reversed(qubits)]  # local index bit order: qubits[k-1] is the most significant
    t = np.moveaxis(t, axes, list(range(k)))
    shp = t.shape
    t = (u @ t.reshape(1 << k, -1)).reshape(shp)
    t = np.moveaxis(t, list(range(k)), axes)
    return t.reshape(-1)


@pytest.mark.parametrize("n,qubits,seed", [(13, (0, 1, 2, 3, 4), 1), (14, (3, 9, 0, 12, 5, 7), 2),
                                            (16, (15, 2, 8, 11, 4), 3), (17, (1, 0, 2, 3, 4, 5), 4)])
def test_tensor_core_unitary_c64(pkg, n, qubits, seed):
    init = random_state(n, seed)
    u = random_unitary(len(qubits), seed)
    want = apply_numpy(init, u, qubits, n)
    with pkg.State(n, pkg.C64) as s:
        s.upload(init)
        s.apply_unitary(u, qubits)
        got = s.amplitudes().astype(np.complex128)
        st = s.stats()
    # FP32 accuracy (3xTF32 products, FP32 accumulation): measured 2.5e-8 max / 5.7e-9 rms at n = 13
    assert np.abs(got - want).max() <= 2e-7
    assert abs(np.vdot(want, got)) ** 2 / np.vdot(got, got).real >= 1 - 1e-11
    assert st["kernel_launches"] >= 1


@pytest.mark.parametrize("n,qubits,precision", [(10, (2, 7, 4), 0), (13, (0, 5, 9, 12, 1), 0), (12, (3, 8), 1),
                                                 (9, (0, 1, 2, 3, 4, 5), 1)])
def test_cuda_core_unitary(pkg, n, qubits, precision):
    init = random_state(n, 7 + n)
    u = random_unitary(len(qubits), n)
    want = apply_numpy(init, u, qubits, n)
    with pkg.State(n, precision) as s:
        s.upload(init)
        s.apply_unitary(u, qubits)
        got = s.amplitudes().astype(np.complex128)
    assert np.abs(got - want).max() <= (1e-12 if precision == 0 else 2e-5)


def test_unitary_then_gates_keep_the_layout_map(pkg):
    """After the targets are moved onto the low bits, later gates and reads
    still address logical qubits."""
    n = 14
    C = pkg.circuits
    init = random_state(n, 3)
    u = random_unitary(6, 5)
    ops = C.random_circuit(n, 80, seed=9)
    ref = pkg.State(n)
    ref.upload(apply_numpy(init, u, (13, 2, 7, 9, 4, 11), n))
    ref.apply(ops)
    want = ref.amplitudes()
    ref.close()
    with pkg.State(n, pkg.C64) as s:
        s.upload(init)
        s.apply_unitary(u, (13, 2, 7, 9, 4, 11))
        s.apply(ops)
        got = s.amplitudes().astype(np.complex128)
    assert np.abs(got - want).max() <= 2e-5


@pytest.mark.parametrize("n,fuse_k", [(16, 6), (18, 5)])
def test_tensor_core_fusion_mode_vs_fp64(pkg, n, fuse_k):
    C = pkg.circuits
    ops = C.brick(n, 6, seed=n, fuse_k=fuse_k)
    with pkg.State(n) as ref:
        ref.apply(ops)
        want = ref.amplitudes()
    with pkg.State(n, pkg.C64) as s:
        s.set_fusion_mode(1)
        s.apply(ops)
        got = s.amplitudes().astype(np.complex128)
        st = s.stats()
    assert np.abs(got - want).max() <= 2e-5
    assert abs(np.vdot(want, got)) ** 2 / np.vdot(got, got).real >= 1 - 1e-9
    assert st["passes"] > 0
