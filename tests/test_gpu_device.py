"""The LightningQubit-surface device whose state stays on the GPU
(lightning_b200/device.py), against the oracle: state preparation, gates, analytic
measurements, finite-shot estimates, the adjoint Jacobian with the reference's
trainable-parameter bookkeeping (lightning_base.py:257-304, lightning_qubit.py:631-692)
and both VJP forms (lightning_qubit.py:694-808)."""
import numpy as np
import pytest

from conftest import TOL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def D():
    from lightning_b200 import device
    return device


def circuit(D):
    Op = D.Operation
    return [Op("Hadamard", ["a"]), Op("RX", ["b"], [0.3]), Op("Rot", ["c"], [0.1, 0.7, -0.4]),
            Op("CNOT", ["a", "c"]), Op("CRY", [2, "b"], [1.2]), Op("IsingXY", ["c", 2], [0.45]),
            Op("PhaseShift", ["a"], [0.8]), Op("Identity", ["b"])]


def oracle_ops(D, dev, ops):
    """The same circuit as oracle records on device wire indices (Rot decomposed as the serializer does)."""
    return dev._serialize_ops([op for op in ops if op.name != "Identity"], decompose_rot=True)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_apply_and_measure(D, dtype):
    import lq_oracle as O
    dev = D.LightningQubit(["a", "b", "c", 2], c_dtype=dtype)
    ops = circuit(D)
    dev.apply(ops)
    want = O.run_circuit(4, oracle_ops(D, dev, ops))
    tol = TOL[dtype]
    assert np.abs(dev.state - want).max() < tol
    obs = {
        "named": D.named("PauliX", ["b"]),
        "tensor": D.tensor(D.named("PauliZ", ["a"]), D.named("PauliY", [2])),
        "herm": D.hermitian(np.array([[1, 2j], [-2j, 0.5]]), ["c"]),
        "ham": D.hamiltonian([0.3, -1.1], [D.named("PauliZ", ["b"]), D.tensor(D.named("PauliX", ["a"]),
                                                                               D.named("PauliX", ["c"]))]),
    }
    for k, o in obs.items():
        terms = dev._serialize_obs(o)
        assert abs(dev.expval(o) - O.expval(want, terms)) < tol, k
        assert abs(dev.var(o) - O.var(want, terms)) < tol, k
    p = dev.probability_lightning(["c", "a"])
    assert np.abs(p - O.probs(want, [2, 0])).max() < tol
    import scipy.sparse as sp
    H = sp.random(16, 16, density=0.3, random_state=1) + 1j * sp.random(16, 16, density=0.3, random_state=2)
    H = H + H.conj().T
    so = D.sparse_hamiltonian(H)
    stol = tol if dtype == np.complex128 else tol * 10  # complex64: H entries up to ~2, values up to ~10
    assert abs(dev.expval(so) - O.sparse_expval(want, *so.csr)) < stol
    assert abs(dev.var(so) - O.sparse_var(want, *so.csr)) < stol


def test_state_preparation(D):
    import lq_oracle as O
    rng = np.random.default_rng(1)
    dev = D.LightningQubit(4)
    v = rng.normal(size=4) + 1j * rng.normal(size=4)
    v /= np.linalg.norm(v)
    dev.apply([D.Operation("QubitStateVector", [3, 1], [v]), D.Operation("RY", [0], [0.4])])
    full = np.zeros(16, dtype=complex)
    for k in range(4):  # wire 3 is the high bit of k, wire 1 the low one
        full[((k >> 1) & 1) << 0 | (k & 1) << 2] = v[k]
    want = O.run_circuit(4, [("RY", [0], False, [0.4])], state=full)
    assert np.abs(dev.state - want).max() < 1e-12
    dev.reset()
    dev.apply([D.Operation("BasisState", [0, 2], [np.array([1, 1])])])
    st = dev.state
    assert st[0b1010] == 1 and np.abs(st).sum() == 1
    with pytest.raises(D.DeviceError, match="cannot be used after other Operations"):
        dev.apply([D.Operation("RX", [0], [0.1]), D.Operation("BasisState", [0], [np.array([1])])])
    with pytest.raises(ValueError, match="must consist of 0 or 1"):
        dev.apply([D.Operation("BasisState", [0], [np.array([2])])])


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_adjoint_jacobian(D, dtype):
    import lq_oracle as O
    dev = D.LightningQubit(["a", "b", "c", 2], c_dtype=dtype)
    ops = circuit(D)
    obs = [D.named("PauliZ", ["a"]), D.hamiltonian([0.5, 2.0], [D.named("PauliX", ["c"]),
                                                                  D.tensor(D.named("PauliY", ["b"]),
                                                                           D.named("PauliZ", [2]))])]
    tape = D.Tape(ops, [D.expval(o) for o in obs], trainable_params=[0, 1, 3, 5, 6])
    jac = dev.adjoint_jacobian(tape)
    # oracle: central differences over every parameter of the tape
    flat = [(i, j) for i, op in enumerate(ops) for j in range(len(op.params))]
    tol = 1e-7 if dtype == np.complex128 else 2e-4
    assert jac.shape == (2, 5)
    for col, p in enumerate(tape.trainable_params):
        i, j = flat[p]
        fd = []
        for sgn in (1, -1):
            o2 = [D.Operation(op.name, op.wires, list(op.params)) for op in ops]
            o2[i].params[j] += sgn * 1e-5
            st = O.run_circuit(4, oracle_ops(D, dev, o2))
            fd.append([O.expval(st, dev._serialize_obs(o)) for o in obs])
        want = (np.array(fd[0]) - np.array(fd[1])) / 2e-5
        assert np.abs(jac[:, col] - want).max() < tol, p
    # use_device_state: the same numbers without re-running the circuit
    dev.reset()
    dev.apply(ops)
    assert np.abs(dev.adjoint_jacobian(tape, use_device_state=True) - jac).max() < 1e-12
    with pytest.raises(D.QuantumFunctionError, match="not supported using"):
        dev.adjoint_jacobian(D.Tape([D.Operation("CRot", [0, 1], [0.1, 0.2, 0.3])], [D.expval(obs[0])]))
    with pytest.raises(D.QuantumFunctionError, match="Use vjp method instead"):
        dev.adjoint_jacobian(D.Tape(ops, [D.state()]))


def test_state_prep_shifts_trainable_params(D):
    """lightning_base.py:281-297: parameters of a leading state preparation are not
    differentiated; the others are shifted by one."""
    import lq_oracle as O
    dev = D.LightningQubit(3)
    v = np.array([0.6, 0, 0, 0.8j, 0, 0, 0, 0])
    ops = [D.Operation("StatePrep", [0, 1, 2], [v]), D.Operation("RX", [0], [0.3]), D.Operation("RY", [2], [0.9])]
    tape = D.Tape(ops, [D.expval(D.named("PauliZ", [2]))], trainable_params=[0, 1, 2])
    jac = dev.adjoint_jacobian(tape)
    psi = O.run_circuit(3, [("RX", [0], False, [0.3]), ("RY", [2], False, [0.9])], state=v)
    want = O.adjoint_jacobian(psi, [("RX", [0], False, [0.3]), ("RY", [2], False, [0.9])],
                              [[(1.0, [("PauliZ", [2])])]], [0, 1])
    assert jac.shape == (1, 3) and jac[0, 0] == 0.0
    assert np.abs(jac[0, 1:] - want[0]).max() < 1e-12


def test_vjp_expval_and_state(D):
    import lq_oracle as O
    dev = D.LightningQubit(["a", "b", "c", 2])
    ops = circuit(D)
    ms = [D.expval(D.named("PauliZ", ["a"])), D.expval(D.named("PauliX", ["c"]))]
    tape = D.Tape(ops, ms, trainable_params=[1, 2, 4])
    dy = np.array([0.7, -1.3])
    got = dev.vjp(ms, dy)(tape)
    full = dev.adjoint_jacobian(tape)
    assert np.abs(got - dy @ full).max() < 1e-12
    rng = np.random.default_rng(5)
    gv = rng.normal(size=16) + 1j * rng.normal(size=16)
    st_tape = D.Tape(ops, [D.state()], trainable_params=[1, 2, 4])
    got_s = dev.vjp([D.state()], gv)(st_tape)
    sops = oracle_ops(D, dev, ops)
    psi = O.run_circuit(4, sops)
    want_s = O.vjp_state(psi, sops, gv, [1, 2, 4])
    assert np.abs(got_s - want_s).max() < 1e-12
    with pytest.raises(ValueError, match="length of grad_vec"):
        dev.vjp(ms, np.ones(3))
    assert np.all(dev.vjp(ms, np.zeros(2))(tape) == 0)


def test_finite_shots(D):
    import lq_oracle as O
    dev = D.LightningQubit(3, shots=200000, seed=11)
    ops = [D.Operation("RY", [0], [0.7]), D.Operation("CNOT", [0, 1]), D.Operation("RX", [2], [1.1])]
    dev.apply(ops)
    s = dev.generate_samples()
    assert s.shape == (200000, 3) and set(np.unique(s)) <= {0, 1}
    st = dev.state
    p = O.probs(st, [0, 1, 2])
    counts = np.bincount(s[:, 0] * 4 + s[:, 1] * 2 + s[:, 2], minlength=8) / 200000
    assert np.abs(counts - p).max() < 0.01
    for o in (D.named("PauliZ", [0]), D.named("PauliX", [2]),
              D.tensor(D.named("PauliY", [2]), D.named("PauliZ", [1]))):
        exact = O.expval(st, dev._serialize_obs(o))
        assert abs(dev.expval(o) - exact) < 0.01
    assert np.abs(dev.state - st).max() == 0  # estimates leave the device state alone


@pytest.mark.parametrize("kernel", ["Local", "NonZeroRandom"])
def test_mcmc_device(D, kernel):
    """lightning_qubit.py:190-221, :534-537: mcmc devices sample with Metropolis chains."""
    dev = D.LightningQubit(2, shots=1000, mcmc=True, kernel_name=kernel, num_burnin=100, seed=4)
    dev.apply([D.Operation("RX", [0], [1.5708])])
    s = dev.generate_samples()
    assert s.shape == (1000, 2) and set(np.unique(s[:, 1])) == {0}
    assert 0.4 < s[:, 0].mean() < 0.6
