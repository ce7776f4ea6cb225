"""Gate application on the B200 vs the FP64 oracle (GateImplementationsLM semantics).

Mirrors the reference's gate tests (LQ/gates/tests/Test_GateImplementations_*.cpp):
every gate, both directions, random states, every wire placement on small
registers, dense matrices of 1..7 wires, and generators.
"""
import itertools

import numpy as np
import pytest

from conftest import TOL, random_state

pytestmark = pytest.mark.gpu

GATES = {"Identity": (1, 0), "PauliX": (1, 0), "PauliY": (1, 0), "PauliZ": (1, 0), "Hadamard": (1, 0),
         "S": (1, 0), "T": (1, 0), "PhaseShift": (1, 1), "RX": (1, 1), "RY": (1, 1), "RZ": (1, 1),
         "Rot": (1, 3), "CNOT": (2, 0), "CY": (2, 0), "CZ": (2, 0), "SWAP": (2, 0), "IsingXX": (2, 1),
         "IsingXY": (2, 1), "IsingYY": (2, 1), "IsingZZ": (2, 1), "ControlledPhaseShift": (2, 1),
         "CRX": (2, 1), "CRY": (2, 1), "CRZ": (2, 1), "CRot": (2, 3), "SingleExcitation": (2, 1),
         "SingleExcitationMinus": (2, 1), "SingleExcitationPlus": (2, 1), "Toffoli": (3, 0),
         "CSWAP": (3, 0), "DoubleExcitation": (4, 1), "DoubleExcitationMinus": (4, 1),
         "DoubleExcitationPlus": (4, 1), "MultiRZ": (3, 1)}


@pytest.fixture(scope="module")
def capi():
    from lightning_b200 import capi as c
    if c.device_count() == 0:
        pytest.fail("no CUDA device visible to libb200sv")
    return c


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("name", list(GATES))
def test_gate_random_state(capi, name, inverse, dtype):
    import lq_oracle as O
    rng = np.random.default_rng(1000 + 2 * list(GATES).index(name) + int(inverse))
    n = 9
    k, p = GATES[name]
    for _ in range(3):
        st = random_state(rng, n, dtype)
        wires = [int(w) for w in rng.choice(n, k, replace=False)]
        params = list(rng.uniform(0, 2 * np.pi, p))
        sv = capi.StateVector(n, dtype)
        sv.upload(st)
        sv.apply(name, wires, inverse, params)
        got = sv.download()
        want = O.apply_op(st.astype(np.complex128), name, wires, inverse, params)
        assert np.abs(got - want).max() < TOL[dtype], (name, wires)


@pytest.mark.parametrize("name", ["CNOT", "CRY", "IsingXY", "SWAP", "CSWAP", "Toffoli", "DoubleExcitationPlus",
                                  "ControlledPhaseShift", "CY", "SingleExcitationMinus"])
def test_gate_every_wire_placement(capi, name):
    import lq_oracle as O
    rng = np.random.default_rng(5)
    n = 5
    k, p = GATES[name]
    st = random_state(rng, n)
    sv = capi.StateVector(n)
    for wires in itertools.permutations(range(n), k):
        params = list(rng.uniform(0, 2 * np.pi, p))
        sv.upload(st)
        sv.apply(name, list(wires), False, params)
        want = O.apply_op(st, name, list(wires), False, params)
        assert np.abs(sv.download() - want).max() < 1e-12, wires


@pytest.mark.parametrize("n", [2, 5, 20])
def test_c64_two_wire_dense_on_lowest_bits(capi, n):
    """complex64 two-wire dense steps on state bits 0 and 1 (the last two wires, either order)
    move each group with two 16-byte accesses; results against the oracle, beside the same
    matrices on other wires and with a control added."""
    import lq_oracle as O
    from lightning_b200.workloads import random_unitary
    rng = np.random.default_rng(90 + n)
    st = random_state(rng, n, np.complex64)
    sv = capi.StateVector(n, np.complex64)
    placements = [[n - 2, n - 1], [n - 1, n - 2]] + ([[0, n - 1], [1, 0]] if n > 2 else [])
    for wires in placements:
        u = random_unitary(rng, 2)
        sv.upload(st)
        sv.apply_matrix(u.astype(np.complex64), wires)
        want = O.apply_op(st.astype(np.complex128), "QubitUnitary", wires, False, [], u)
        assert np.abs(sv.download() - want).max() < TOL[np.complex64], wires
        for name in ("IsingXX", "IsingXY", "SingleExcitation"):
            sv.upload(st)
            sv.apply(name, wires, False, [0.37])
            want = O.apply_op(st.astype(np.complex128), name, wires, False, [0.37])
            assert np.abs(sv.download() - want).max() < TOL[np.complex64], (name, wires)
    if n > 2:  # controlled: the general kernel
        sv.upload(st)
        sv.apply("CRY", [0, n - 1], False, [0.7])
        want = O.apply_op(st.astype(np.complex128), "CRY", [0, n - 1], False, [0.7])
        assert np.abs(sv.download() - want).max() < TOL[np.complex64]


@pytest.mark.parametrize("n", [1, 2, 14, 21])
def test_low_and_high_wires(capi, n):
    import lq_oracle as O
    rng = np.random.default_rng(n)
    st = random_state(rng, n)
    sv = capi.StateVector(n)
    sv.upload(st)
    ops = [("RX", [0], False, [0.3]), ("RY", [n - 1], False, [1.1]), ("Hadamard", [n // 2], False, []),
           ("PauliY", [n - 1], True, []), ("RZ", [0], False, [2.0])]
    if n >= 2:
        ops += [("CNOT", [n - 1, 0], False, []), ("CRX", [0, n - 1], True, [0.7])]
    for op in ops:
        sv.apply(*op)
        st = O.apply_op(st, *op)
    assert np.abs(sv.download() - st).max() < 1e-12


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6, 7])
def test_apply_matrix(capi, k, dtype):
    import lq_oracle as O
    from lightning_b200.workloads import random_unitary
    rng = np.random.default_rng(100 + k)
    n = max(k + 2, 9)
    st = random_state(rng, n, dtype)
    for inverse in (False, True):
        u = random_unitary(rng, k)
        wires = [int(w) for w in rng.choice(n, k, replace=False)]
        sv = capi.StateVector(n, dtype)
        sv.upload(st)
        sv.apply_matrix(u.astype(dtype), wires, inverse)
        want = O.apply_matrix(st.astype(np.complex128), u.astype(dtype).astype(np.complex128), wires, inverse)
        assert np.abs(sv.download() - want).max() < TOL[dtype]


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("k", [4, 5, 6, 7, 8, 10])
def test_apply_matrix_tiled(capi, k, dtype):
    """Matrices on 4..10 wires of a state wide enough for the tiled kernel (tiles of 4096
    amplitudes), wires in the lowest, highest and scattered positions."""
    import lq_oracle as O
    from lightning_b200.workloads import random_unitary
    rng = np.random.default_rng(200 + k)
    n = 14
    st = random_state(rng, n, dtype)
    placements = [list(range(n - k, n)), list(range(k)), [int(w) for w in rng.choice(n, k, replace=False)]]
    for wires, inverse in zip(placements, (False, True, False)):
        u = random_unitary(rng, k)
        sv = capi.StateVector(n, dtype)
        sv.upload(st)
        sv.apply_matrix(u.astype(dtype), wires, inverse)
        want = O.apply_matrix(st.astype(np.complex128), u.astype(dtype).astype(np.complex128), wires, inverse)
        assert np.abs(sv.download() - want).max() < TOL[dtype]


GENS = ["PhaseShift", "RX", "RY", "RZ", "IsingXX", "IsingXY", "IsingYY", "IsingZZ", "CRX", "CRY", "CRZ",
        "ControlledPhaseShift", "SingleExcitation", "SingleExcitationMinus", "SingleExcitationPlus",
        "DoubleExcitation", "DoubleExcitationMinus", "DoubleExcitationPlus", "MultiRZ"]


@pytest.mark.parametrize("name", GENS)
def test_generators(capi, name):
    import lq_oracle as O
    rng = np.random.default_rng(7)
    n = 7
    k = {"PhaseShift": 1, "RX": 1, "RY": 1, "RZ": 1, "MultiRZ": 3}.get(name, 4 if "Double" in name else 2)
    st = random_state(rng, n)
    wires = [int(w) for w in rng.choice(n, k, replace=False)]
    sv = capi.StateVector(n)
    sv.upload(st)
    scale = sv.apply_generator(name, wires)
    want, wscale = O.apply_generator(st, name, wires)
    assert scale == wscale
    assert np.abs(sv.download() - want).max() < 1e-12


def test_generator_definition(capi):
    """i G |psi> = dU/dtheta |psi> at theta = 0 (Test_GateImplementations_Generator.cpp:30-40)."""
    import lq_oracle as O
    rng = np.random.default_rng(11)
    n = 6
    eps = 1e-6
    for name in GENS:
        k = {"PhaseShift": 1, "RX": 1, "RY": 1, "RZ": 1, "MultiRZ": 2}.get(name, 4 if "Double" in name else 2)
        wires = list(range(k))
        st = random_state(rng, n)
        sv = capi.StateVector(n)
        sv.upload(st)
        scale = sv.apply_generator(name, wires)
        g = sv.download()
        plus = O.apply_op(st, name, wires, False, [eps])
        minus = O.apply_op(st, name, wires, False, [-eps])
        deriv = (plus - minus) / (2 * eps)
        assert np.abs(1j * scale * g - deriv).max() < 1e-8, name


def test_apply_ops_sequence_and_errors(capi):
    import lq_oracle as O
    from lightning_b200.workloads import gate_sweep
    n = 10
    ops = gate_sweep(n, 60, seed=3)
    sv = capi.StateVector(n)
    sv.apply_ops(ops)
    want = O.run_circuit(n, ops)
    assert np.abs(sv.download() - want).max() < 1e-12
    with pytest.raises(capi.B200Error, match="wires must be distinct"):
        sv.apply("CNOT", [1, 1])
    with pytest.raises(capi.B200Error, match="out of range"):
        sv.apply("RX", [n], False, [0.1])
    with pytest.raises(capi.B200Error, match="expected 1 parameters"):
        sv.apply("RX", [0], False, [])
    with pytest.raises(capi.B200Error, match="expected 2 wires"):
        sv.apply("CNOT", [0])


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("n", [13, 15, 20, 22])
def test_fused_apply_matches_oracle(capi, n, dtype):
    """b200sv_apply_ops_fused (segments of gates applied per shared-memory tile) on the gate-sweep
    family plus gates the tile forms do not cover (three-wire matrices, four-wire excitations,
    Rot, wide MultiRZ), which run as their own passes in order."""
    import lq_oracle as O
    from lightning_b200.workloads import gate_sweep, random_unitary, random_state as rs
    rng = np.random.default_rng(n)
    ops = gate_sweep(n, 120, seed=n)
    extra = [("Rot", [3], False, [0.1, 0.7, -0.4]), ("DoubleExcitation", [0, 5, 9, n - 1], False, [0.3]),
             ("MultiRZ", list(range(0, n, 2)), False, [0.9]), ("QubitUnitary", [1, 7, n - 2], False, [],
                                                                  random_unitary(rng, 3)),
             ("CRot", [n - 1, 2], True, [0.2, 0.3, 0.4]), ("IsingXY", [4, n - 3], False, [1.1]),
             ("PhaseShift", [n - 1], False, [0.5]), ("S", [0], True, []), ("CSWAP", [2, 9, min(14, n - 1)], False, [])]
    for k, op in enumerate(extra):
        ops.insert(10 * k + 5, op)
    st = rs(n, seed=n, dtype=dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    sv.apply_ops_fused(ops)
    want = O.run_circuit(n, ops, state=st.astype(np.complex128))
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    assert np.abs(sv.download() - want).max() < tol


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_fused_every_gate_kind_vs_reference(capi, ref_module, dtype):
    """400 gates of every kind (inverse or not) plus applyMatrix on 1..3 wires, on random wires of
    a 21-qubit state (the narrowest that takes the fused path), applied through
    b200sv_apply_ops_fused and compared with the reference's own StateVectorC128 on the same
    complex128 start state; the per-gate path must give the same state."""
    import ref
    from lightning_b200.workloads import random_unitary, random_state as rs
    n = 21
    rng = np.random.default_rng(2121)
    names = [g for g in GATES if g != "Identity"]
    ops = []
    for _ in range(400):
        if rng.random() < 0.1:
            k = int(rng.integers(1, 4))
            ops.append(("QubitUnitary", [int(w) for w in rng.choice(n, k, replace=False)], bool(rng.random() < 0.5),
                        [], random_unitary(rng, k)))
            continue
        name = names[int(rng.integers(len(names)))]
        k, p = GATES[name]
        if name == "MultiRZ":
            k = int(rng.integers(1, 7))
        ops.append((name, [int(w) for w in rng.choice(n, k, replace=False)], bool(rng.random() < 0.5),
                    list(rng.uniform(0, 2 * np.pi, p))))
    st = rs(n, seed=5, dtype=dtype)
    want = ref.run_circuit(ref_module, n, ops, state=st.astype(np.complex128))
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    sv.apply_ops_fused(ops)
    got = sv.download()
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    assert np.abs(got - want).max() < tol
    sv.upload(st)
    sv.apply_ops(ops)
    assert np.abs(sv.download() - got).max() < tol


@pytest.mark.parametrize("k", [3, 4, 5])
@pytest.mark.parametrize("n", [12, 13, 20])
def test_apply_matrix_tensor_cores_c64(capi, k, n):
    """complex64 applyMatrix on 3..5 wires runs on the tensor cores (tcgen05 kind::tf32 with split
    operands) once the state holds a 128-group tile (n >= k + 7): lowest, highest and scattered
    wires, both directions, against the FP64 oracle at the complex64 bound."""
    import lq_oracle as O
    from lightning_b200.workloads import random_unitary
    if n < k + 7:
        pytest.skip("state narrower than one tile")
    rng = np.random.default_rng(300 + 10 * k + n)
    st = random_state(rng, n, np.complex64)
    placements = [list(range(n - k, n)), list(range(k)), [int(w) for w in rng.choice(n, k, replace=False)]]
    for wires, inverse in zip(placements, (False, True, False)):
        u = random_unitary(rng, k).astype(np.complex64)
        sv = capi.StateVector(n, np.complex64)
        sv.upload(st)
        sv.apply_matrix(u, wires, inverse)
        got = sv.download()
        sv.synchronize()
        want = O.apply_matrix(st.astype(np.complex128), u.astype(np.complex128), wires, inverse)
        assert np.abs(got - want).max() < TOL[np.complex64], (wires, inverse)
        assert abs(np.linalg.norm(got.astype(np.complex128)) - 1.0) < 1e-5
