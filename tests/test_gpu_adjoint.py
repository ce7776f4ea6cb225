"""Adjoint Jacobian on the B200 (plain drop-in path) vs golden values and the oracle.

Golden values: CS/algorithms/tests/Test_AdjointJacobian.cpp:123-554 (param-shift
results the reference asserts with margins 1e-7 / 1e-4).  Larger random circuits
are compared with the oracle's restatement of AdjointJacobianLQubit.hpp:212-335
(and, when built, the reference itself) and with central finite differences.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = [-np.pi / 7, np.pi / 5, 2 * np.pi / 3]


@pytest.fixture(scope="module")
def capi():
    from lightning_b200 import capi as c
    return c


def Zs(*ws):
    return [(1.0, [("PauliZ", [w])]) for w in ws]


def jac(capi, n, ops, obs, tp, dtype=np.complex128, state=None):
    sv = capi.StateVector(n, dtype)
    if state is not None:
        sv.upload(np.asarray(state, dtype=dtype))
    return sv.adjoint_jacobian(ops, obs, tp, apply_operations=True)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_golden_single_ops(capi, dtype):
    tol = 1e-7 if dtype == np.complex128 else 1e-5
    for p in np.linspace(-2 * np.pi, 2 * np.pi, 7):
        assert abs(jac(capi, 1, [("RX", [0], False, [p])], [Zs(0)], [0], dtype)[0, 0] + np.sin(p)) < tol
        assert abs(jac(capi, 1, [("RY", [0], False, [p])], [[(1.0, [("PauliX", [0])])]], [0], dtype)[0, 0]
                   - np.cos(p)) < tol
    j = jac(capi, 2, [("RX", [0], False, [P[0]])], [Zs(0), Zs(1)], [0], dtype)
    assert abs(j[0, 0] + np.sin(P[0])) < tol and abs(j[1, 0]) < tol


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_golden_three_rx(capi, dtype):
    tol = 1e-7 if dtype == np.complex128 else 1e-5
    ops = [("RX", [i], False, [P[i]]) for i in range(3)]
    j = jac(capi, 3, ops, [Zs(0), Zs(1), Zs(2)], [0, 1, 2], dtype)
    assert np.allclose(np.diag(j), -np.sin(P), atol=tol)
    j = jac(capi, 3, ops, [Zs(0), Zs(1), Zs(2)], [0, 2], dtype)
    assert abs(j[0, 0] + np.sin(P[0])) < tol and abs(j[1, 1]) < tol and abs(j[2, 1] + np.sin(P[2])) < tol
    zzz = [[(1.0, [("PauliZ", [0]), ("PauliZ", [1]), ("PauliZ", [2])])]]
    j = jac(capi, 3, ops, zzz, [0, 1, 2], dtype)
    assert np.allclose(j[0], [-0.1755096592645253, 0.26478810666384334, -0.6312451595102775], atol=tol)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_golden_mixed_xxx(capi, dtype):
    tol = 1e-7 if dtype == np.complex128 else 1e-5
    names = ["RZ", "RY", "RZ", "CNOT", "CNOT", "RZ", "RY", "RZ"]
    params = [[P[0]], [P[1]], [P[2]], [], [], [P[0]], [P[1]], [P[2]]]
    wires = [[0], [0], [0], [0, 1], [1, 2], [1], [1], [1]]
    ops = [(a, w, False, p) for a, w, p in zip(names, wires, params)]
    xxx = [[(1.0, [("PauliX", [0]), ("PauliX", [1]), ("PauliX", [2])])]]
    j = jac(capi, 3, ops, xxx, list(range(6)), dtype)
    assert np.allclose(j[0], [0.0, -0.674214427, 0.275139672, 0.275139672, -0.0129093062, 0.323846156], atol=tol)


def test_golden_decomposed_rot(capi):
    expect = [[0, -9.90819496e-01, 0], [-8.18996553e-01, 1.62526544e-01, 0], [-0.203949, 0.48593716, 0],
              [0, 1, 0], [-2.03948985e-01, 4.85937177e-01, 0], [-8.18996598e-01, 1.62526487e-01, 0],
              [0, -9.90819511e-01, 0]]
    init = [1 / np.sqrt(2), -1 / np.sqrt(2)]
    for theta, e in zip(np.linspace(-2 * np.pi, 2 * np.pi, 7), expect):
        lp = [theta, theta ** 3, np.sqrt(2) * theta]
        ops = [("RZ", [0], False, [lp[0]]), ("RY", [0], False, [lp[1]]), ("RZ", [0], False, [lp[2]])]
        j = jac(capi, 1, ops, [Zs(0)], [0, 1, 2], state=init)
        assert np.allclose(j[0], e, atol=1e-4)


def test_golden_mixed_ops_obs_tp(capi):
    lp = [0.543, 0.54, 0.1, 0.5, 1.3, -2.3, 0.5, -0.5, 0.5]
    names = ["Hadamard", "RX", "CNOT", "RZ", "RY", "RZ", "RZ", "RY", "RZ", "RZ", "RY", "CNOT"]
    params = [[], [lp[0]], [], [lp[1]], [lp[2]], [lp[3]], [lp[4]], [lp[5]], [lp[6]], [lp[7]], [lp[8]], []]
    wires = [[0], [0], [0, 1], [0], [0], [0], [0], [0], [0], [0], [1], [0, 1]]
    ops = [(a, w, False, p) for a, w, p in zip(names, wires, params)]
    obs = [[(1.0, [("PauliX", [0]), ("PauliZ", [1])])]]
    j = jac(capi, 2, ops, obs, [1, 2, 3])
    assert np.allclose(j[0], [-0.71429188, 0.04998561, -0.71904837], atol=1e-7)


def test_golden_hamiltonians(capi):
    j = jac(capi, 2, [("RX", [0], False, [P[0]])], [[(0.3, [("PauliZ", [0])]), (0.7, [("PauliZ", [1])])]], [0])
    assert abs(j[0, 0] + 0.3 * np.sin(P[0])) < 1e-7
    ops = [("RX", [i], False, [P[i]]) for i in range(3)]
    ham = [[(0.47, [("PauliZ", [0])]), (0.32, [("PauliZ", [1])]), (0.96, [("PauliZ", [2])])]]
    j = jac(capi, 3, ops, ham, [0, 2])
    assert np.allclose(j[0], [-0.47 * np.sin(P[0]), -0.96 * np.sin(P[2])], atol=1e-7)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_random_circuit_vs_oracle(capi, dtype, ref_module=None):
    import lq_oracle as O
    import ref
    rng = np.random.default_rng(17)
    n = 8
    ops = []
    for l in range(3):
        for q in range(n):
            ops.append((["RX", "RY", "RZ", "PhaseShift"][(q + l) % 4], [q], bool((q * l) % 3 == 1),
                        [float(rng.uniform(0, 2 * np.pi))]))
        for q in range(n - 1):
            ops.append(("CNOT", [q, q + 1], False, []))
        ops += [("IsingXX", [0, 5], False, [0.3]), ("IsingYY", [2, 6], True, [0.5]), ("IsingZZ", [1, 7], False, [0.2]),
                ("IsingXY", [3, 4], False, [1.3]), ("CRX", [4, 0], False, [0.9]), ("CRY", [6, 2], True, [0.4]),
                ("CRZ", [1, 3], False, [2.2]), ("ControlledPhaseShift", [5, 7], False, [0.8]),
                ("SingleExcitation", [2, 5], False, [0.6]), ("SingleExcitationMinus", [0, 1], False, [1.1]),
                ("SingleExcitationPlus", [6, 7], True, [0.35]), ("MultiRZ", [0, 3, 6], False, [0.45]),
                ("DoubleExcitation", [0, 2, 4, 6], False, [0.7]), ("DoubleExcitationMinus", [1, 3, 5, 7], False, [0.2]),
                ("DoubleExcitationPlus", [7, 5, 3, 1], True, [1.7]), ("Hadamard", [2], False, [])]
    obs = [Zs(0), [(1.0, [("PauliX", [3]), ("PauliY", [5])])],
           [(0.4, [("PauliZ", [2]), ("PauliZ", [3])]), (-1.1, [("PauliX", [7])]), (0.2, [("Hadamard", [4])])]]
    npar = sum(1 for o in ops if len(o[3]) > 0)
    tp = list(range(0, npar, 2))
    psi = O.zero_state(n)
    want = O.adjoint_jacobian(psi, ops, obs, tp, apply_operations=True)
    got = jac(capi, n, ops, obs, tp, dtype)
    tol = 1e-12 if dtype == np.complex128 else 1e-5
    assert np.abs(got - want).max() < tol
    m = ref.load()
    if m is not None and dtype == np.complex128:
        final = O.run_circuit(n, ops)
        rj = ref.adjoint_jacobian(m, final.copy(), ops, obs, tp)
        assert np.abs(got - rj).max() < 1e-12
    # matrix operations are not differentiated but must be undone exactly in the reverse sweep
    from lightning_b200.workloads import random_unitary
    ops2 = ops + [("QubitUnitary", [1, 6], False, [], random_unitary(rng, 2)), ("RY", [6], False, [0.4])]
    npar2 = npar + 1
    want2 = O.adjoint_jacobian(O.zero_state(n), ops2, obs, list(range(npar2)), apply_operations=True)
    got2 = jac(capi, n, ops2, obs, list(range(npar2)), dtype)
    assert np.abs(got2 - want2).max() < tol


def test_layered_rotations_vs_fd(capi):
    """The plain-config circuit family at 10 qubits: adjoint vs central finite differences (FP64)."""
    import lq_oracle as O
    from lightning_b200.workloads import layered_rotations
    ops, obs, tp = layered_rotations(n=6, layers=3, seed=1234)
    got = jac(capi, 6, ops, obs, tp)
    fd = O.finite_difference_jacobian(6, ops, obs, h=1e-5)
    assert np.abs(got - fd).max() < 1e-8


def test_layered_rotations_full_size_vs_reference(capi, ref_module):
    """The plain configuration at its full size: 20 qubits, 10 layers of RX RY RZ + CNOT ladder
    (790 gates), <Z0> and the 600-parameter Jacobian, complex128, against the reference's own
    AdjointJacobianC128 (AdjointJacobianLQubit.hpp:212-335) to 1e-12."""
    import ref
    from lightning_b200.workloads import layered_rotations
    ops, obs, tp = layered_rotations()
    assert len(ops) == 790 and len(tp) == 600
    sv = capi.StateVector(20, np.complex128)
    sv.apply_ops(ops)
    ez = sv.expval(obs[0])
    got = sv.adjoint_jacobian(ops, obs, tp)
    psi = ref.run_circuit(ref_module, 20, ops)
    assert abs(ez - ref.expval(ref_module, psi.copy(), obs[0])) < 1e-12
    want = ref.adjoint_jacobian(ref_module, psi, ops, obs, tp)
    assert got.shape == (1, 600)
    assert np.abs(got - want).max() < 1e-12


def test_adjoint_errors(capi):
    with pytest.raises(capi.B200Error, match="not supported using the adjoint"):
        jac(capi, 1, [("Rot", [0], False, [0.1, 0.2, 0.3])], [Zs(0)], [0])
    with pytest.raises(capi.B200Error, match="sorted"):
        jac(capi, 1, [("RX", [0], False, [0.1]), ("RY", [0], False, [0.1])], [Zs(0)], [1, 0])


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_vjp_state(capi, dtype):
    """State-return VJP (VectorJacobianProduct.hpp:60-156) vs the oracle and the reference module."""
    import lq_oracle as O
    import ref
    from lightning_b200.workloads import layered_rotations
    rng = np.random.default_rng(9)
    n = 7
    ops, _, _ = layered_rotations(n=n, layers=2, seed=4)
    ops = ops + [("CRX", [6, 1], False, [0.3]), ("SingleExcitation", [2, 5], True, [0.8]),
                 ("MultiRZ", [0, 3, 6], False, [0.2]), ("DoubleExcitationMinus", [0, 2, 4, 6], False, [0.5])]
    psi = O.run_circuit(n, ops)
    dy = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)) / 8
    npar = sum(1 for op in ops if op[3])
    tp = list(range(1, npar, 2))
    sv = capi.StateVector(n, dtype)
    sv.upload(psi.astype(dtype))
    got = sv.vjp_state(ops, dy.astype(dtype), tp)
    want = O.vjp_state(psi.astype(dtype).astype(np.complex128), ops, dy.astype(dtype).astype(np.complex128), tp)
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    assert np.abs(got - want).max() < tol
    m = ref.load()
    if m is not None and dtype == np.complex128:
        assert np.abs(got - ref.vjp_state(m, psi.copy(), ops, dy, tp)).max() < 1e-12
    import lightning_b200.lightning_qubit_ops as ours
    st = psi.astype(dtype).copy()
    svo = getattr(ours, "StateVectorC" + ("64" if dtype == np.complex64 else "128"))(st)
    sfx = "C64" if dtype == np.complex64 else "C128"
    opsd = getattr(ours.algorithms, "create_ops_list" + sfx)(
        [o[0] for o in ops], [list(o[3]) for o in ops], [list(o[1]) for o in ops], [bool(o[2]) for o in ops],
        [np.zeros(0, dtype=dtype) for _ in ops])
    res = getattr(ours.algorithms, "VectorJacobianProduct" + sfx)()(svo, opsd, dy.astype(dtype), tp)
    assert np.abs(np.asarray(res) - want).max() < tol * 10


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_adjoint_fused_sweep_every_generator(capi, dtype):
    """A 13-qubit state takes the fused reverse sweep (one observable: a Hamiltonian, the VJP
    form).  Every differentiable gate kind, constant gates and matrices on 1..4 wires, a trainable
    subset with gaps and an early exit; against the oracle's AdjointJacobianLQubit restatement,
    and against the unfused sweep of the same engine (two observables)."""
    import lq_oracle as O
    from lightning_b200.workloads import random_unitary
    rng = np.random.default_rng(1313)
    n = 13
    diff_gates = {"RX": 1, "RY": 1, "RZ": 1, "PhaseShift": 1, "CRX": 2, "CRY": 2, "CRZ": 2,
                  "ControlledPhaseShift": 2, "IsingXX": 2, "IsingYY": 2, "IsingZZ": 2, "IsingXY": 2,
                  "SingleExcitation": 2, "SingleExcitationMinus": 2, "SingleExcitationPlus": 2,
                  "DoubleExcitation": 4, "DoubleExcitationMinus": 4, "DoubleExcitationPlus": 4, "MultiRZ": 3}
    names = list(diff_gates)
    ops = [("Hadamard", [q], False, []) for q in range(n)]
    for _ in range(140):
        r = rng.random()
        if r < 0.65:
            name = names[int(rng.integers(len(names)))]
            k = diff_gates[name]
            ops.append((name, [int(w) for w in rng.choice(n, k, replace=False)], bool(rng.random() < 0.3),
                        [float(rng.uniform(0, 2 * np.pi))]))
        elif r < 0.8:
            name = ["CNOT", "CZ", "SWAP", "Toffoli"][int(rng.integers(4))]
            ops.append((name, [int(w) for w in rng.choice(n, 3 if name == "Toffoli" else 2, replace=False)],
                        False, []))
        elif r < 0.9:
            k = int(rng.integers(1, 5))
            ops.append(("QubitUnitary", [int(w) for w in rng.choice(n, k, replace=False)], False, [],
                        random_unitary(rng, k)))
        else:
            ops.append((["S", "T", "PauliY", "Hadamard"][int(rng.integers(4))], [int(rng.integers(n))], False, []))
    npar = sum(1 for op in ops if op[3])
    tp = sorted(int(x) for x in rng.choice(npar - 10, (npar - 10) // 2, replace=False))  # gaps, early exit
    ham = [[(0.7, [("PauliZ", [0]), ("PauliZ", [5])]), (-1.2, [("PauliX", [12])]), (0.4, [("PauliY", [3])])]]
    st = O.run_circuit(n, ops)
    want = O.adjoint_jacobian(st, ops, ham, tp)
    sv = capi.StateVector(n, dtype)
    sv.upload(st.astype(dtype))
    got = sv.adjoint_jacobian(ops, ham, tp)
    tol = 1e-12 if dtype == np.complex128 else 1e-5
    assert np.abs(got - want).max() < tol
    # unfused sweep of the same engine: two observables
    got2 = sv.adjoint_jacobian(ops, ham + [[(1.0, [("PauliZ", [7])])]], tp)
    assert np.abs(got2[0] - got[0]).max() < tol
    want2 = O.adjoint_jacobian(st, ops, [[(1.0, [("PauliZ", [7])])]], tp)
    assert np.abs(got2[1] - want2[0]).max() < tol
