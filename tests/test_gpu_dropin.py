"""The lightning_qubit_ops surface: the same Python code run against this engine's
module and against the reference's own module (compiled into oracle/_ref) must
produce the same numbers — the way pennylane_lightning/lightning_qubit/lightning_qubit.py
drives it (apply_lightning :330-369, expval :401-457, adjoint_jacobian :631-691)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenario(m, dtype):
    sfx = "C64" if dtype == np.complex64 else "C128"
    rdt = np.float32 if dtype == np.complex64 else np.float64
    n = 6
    out = {}
    st = np.zeros(1 << n, dtype=dtype)
    st[0] = 1
    sv = getattr(m, "StateVector" + sfx)(st)
    sv.Hadamard([0], False, [])
    sv.RX([1], False, [0.3])
    sv.CNOT([0, 2], False, [])
    sv.Rot([3], True, [0.1, 0.2, 0.3])
    sv.CRY([4, 5], False, [1.2])
    sv.IsingXY([2, 5], False, [0.7])
    sv.SingleExcitationPlus([1, 3], True, [0.4])
    sv.MultiRZ([0, 2, 4], False, [0.9])
    u = np.linalg.qr(np.arange(16).reshape(4, 4) + 1j * np.eye(4))[0].astype(dtype)
    sv.applyMatrix(u.reshape(-1), [5, 1], False)
    obsm = m.observables
    M = getattr(m, "Measurements" + sfx)(sv)
    out["probs"] = np.asarray(M.probs())
    out["probs_w"] = np.asarray(M.probs([4, 1, 2]))
    out["ev_name"] = M.expval("PauliZ", [3])
    named = getattr(obsm, "NamedObs" + sfx)
    x0, z1, y2 = named("PauliX", [0]), named("PauliZ", [1]), named("PauliY", [2])
    tp = getattr(obsm, "TensorProdObs" + sfx)([x0, z1, y2])
    herm = getattr(obsm, "HermitianObs" + sfx)(np.array([[1, 2j], [-2j, 0.5]], dtype=dtype).reshape(-1), [4])
    ham = getattr(obsm, "Hamiltonian" + sfx)(np.array([0.3, -0.2, 1.1], dtype=rdt), [tp, herm, named("Hadamard", [5])])
    for k, o in (("tp", tp), ("herm", herm), ("ham", ham)):
        out["ev_" + k] = M.expval(o)
        out["var_" + k] = M.var(o)
    out["var_name"] = M.var("PauliX", [2])
    # sparse Hamiltonian (ragged rows, an empty row, unsorted columns)
    rng = np.random.default_rng(4)
    rows, cols, vals = [0], [], []
    for r in range(1 << n):
        k = 0 if r == 5 else int(rng.integers(1, 9))
        cols += list(rng.choice(1 << n, size=k, replace=False))
        vals += list(rng.normal(size=k) + 1j * rng.normal(size=k))
        rows.append(len(cols))
    csr = (np.array(rows, dtype=np.uint64), np.array(cols, dtype=np.uint64), np.array(vals, dtype=dtype))
    out["ev_sparse"] = M.expval(*csr)
    out["var_sparse"] = M.var(*csr)
    ops = getattr(m.algorithms, "create_ops_list" + sfx)(
        ["RX", "CRZ", "RY", "IsingZZ", "PhaseShift"], [[0.4], [0.6], [1.3], [0.2], [0.9]],
        [[0], [0, 3], [2], [1, 4], [5]], [False, True, False, False, True], [np.zeros(0, dtype=dtype)] * 5)
    adj = getattr(m.algorithms, "AdjointJacobian" + sfx)()
    out["jac"] = np.asarray(adj(sv, [tp, ham, named("PauliZ", [0])], ops, [0, 1, 3, 4]))
    out["repr"] = repr(ham)
    del M, sv
    out["state"] = st.copy()  # the borrowed array holds the final amplitudes
    return out


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_same_script_same_numbers(dtype, ref_module):
    import lightning_b200.lightning_qubit_ops as ours
    a = scenario(ours, dtype)
    b = scenario(ref_module, dtype)
    tol = 1e-12 if dtype == np.complex128 else 1e-4
    for k in a:
        if k == "repr":
            continue
        assert np.abs(np.asarray(a[k]) - np.asarray(b[k])).max() < tol, k


def test_generate_samples_surface():
    import lightning_b200.lightning_qubit_ops as ours
    st = np.zeros(8, dtype=np.complex128)
    st[0] = 1
    sv = ours.StateVectorC128(st)
    sv.Hadamard([0], False, [])
    sv.CNOT([0, 2], False, [])
    M = ours.MeasurementsC128(sv)
    s = M.generate_samples(3, 1000)
    assert s.shape == (1000, 3) and s.dtype == np.uint64
    assert set(map(tuple, s.tolist())) <= {(0, 0, 0), (1, 0, 1)}
    u = np.linspace(0.01, 0.99, 50)
    a = M.generate_samples_from_uniforms(3, u)
    assert np.array_equal(a[:, 0], (u > 0.5).astype(np.uint64))
