"""Precision and sampling on the RY-layer + QFT circuit family (controlled phases
2*pi/2^(k-j+1) on every pair), against FP64 references.

* 24 qubits, both precisions: the state, probs, marginals and a Pauli-sum
  expectation value against the reference's own lightning.qubit (complex128,
  compiled from its sources; MeasurementsLQubit.hpp:79-136,248-265), and sample
  indices bit-exact against the oracle's restatement of the inverse-CDF rule
  (LK/measurements/MeasuresFunctors.hpp:70-103) on the same state and uniforms.
* 32 qubits complex128 and 33 qubits complex64 (64 GiB states, indices above
  2^31): the QFT followed by its inverse returns the RY product state, whose
  <Z_q> = cos(theta_q), marginals (products of cos^2 and sin^2 of theta_q / 2)
  and CDF have closed forms in FP64.  Every sample index must satisfy the
  rule's interval condition cdf(i) < U <= cdf(i + 1) against the closed-form CDF.

Bounds: complex128 1e-12; complex64 (FP32 amplitudes, compensated gate
arithmetic, FP64 reductions and CDF) as stated per check.
"""
import numpy as np
import pytest

@pytest.fixture(scope="module")
def capi():
    from lightning_b200 import capi as c
    return c


@pytest.fixture(scope="module")
def qft24(ref_module):
    """The reference's complex128 state of the 24-qubit circuit (computed once)."""
    import ref
    from lightning_b200.workloads import qft_circuit
    n = 24
    ops = qft_circuit(n, seed=9)
    return n, ops, ref.run_circuit(ref_module, n, ops)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_qft_family_24q_vs_reference(capi, ref_module, qft24, dtype):
    import lq_oracle as O
    import ref
    n, ops, psi = qft24
    c128 = dtype == np.complex128
    sv = capi.StateVector(n, dtype)
    sv.apply_ops_fused(ops)
    got = sv.download()
    # state: complex128 per amplitude; complex64 relative to the norm (FP32 storage per gate)
    if c128:
        assert np.abs(got - psi).max() < 1e-12
    else:
        assert np.linalg.norm(got.astype(np.complex128) - psi) < 2e-6
    # the per-gate path gives the same state
    sv2 = capi.StateVector(n, dtype)
    sv2.apply_ops(ops)
    assert np.abs(sv2.download().astype(np.complex128) - psi).max() < (1e-12 if c128 else 1e-7)
    sv2.close()
    ptol = 1e-12 if c128 else 2e-6
    p_all = sv.probs()
    assert np.abs(p_all - np.abs(psi) ** 2).max() < ptol
    for wires in (list(range(10)), list(range(n - 10, n)), [0, 7, 23, 12, 3]):
        want = ref.probs(ref_module, psi.copy(), wires)
        assert np.abs(sv.probs(wires) - want).max() < ptol, wires
    ham = [(0.7, [("PauliZ", [0]), ("PauliX", [5])]), (-1.3, [("PauliY", [23])]),
           (0.4, [("PauliX", [11]), ("PauliX", [12])]), (2.1, [("PauliZ", [17])])]
    assert abs(sv.expval(ham) - ref.expval(ref_module, psi.copy(), ham)) < (1e-12 if c128 else 2e-6)
    # sample indices: the engine's CDF and search against the oracle's restatement on this state
    rng = np.random.default_rng(24)
    u = rng.uniform(size=20000)
    want_idx = O.sample_kokkos_rule(O.cdf_fixed_order(got), u)
    assert np.array_equal(sv.sample(len(u), uniforms=u), want_idx)
    sv.close()


def _product_probs(thetas):
    """Per wire (p0, p1) of RY(theta)|0> = cos(theta/2)|0> + sin(theta/2)|1>."""
    t = np.asarray(thetas, dtype=np.float64)
    return np.stack([np.cos(t / 2) ** 2, np.sin(t / 2) ** 2], axis=1)


def _marginal(pq, wires):
    """Closed-form probs(wires) of a product state, wires[0] the most significant output bit."""
    out = np.ones(1)
    for w in wires:
        out = np.kron(out, pq[w])
    return out


def _cdf_closed(pq, idx):
    """sum_{j < idx} P(j) for a product state, MSB-first (wire 0 = bit n-1); idx may equal 2^n."""
    n = pq.shape[0]
    idx = np.asarray(idx, dtype=np.uint64)
    full = idx >= np.uint64(1 << n)
    cdf = np.zeros(idx.size)
    prefix = np.ones(idx.size)
    for q in range(n):
        bit = ((idx >> np.uint64(n - 1 - q)) & np.uint64(1)).astype(bool)
        cdf += np.where(bit, prefix * pq[q, 0], 0.0)
        prefix *= np.where(bit, pq[q, 1], pq[q, 0])
    cdf[full] = 1.0
    return cdf


def test_product_state_closed_forms_cpu():
    """The closed forms used below, against an explicit product state (CPU only)."""
    rng = np.random.default_rng(3)
    th = rng.uniform(0, 2 * np.pi, 6)
    pq = _product_probs(th)
    p = _marginal(pq, list(range(6)))
    assert abs(p.sum() - 1) < 1e-14
    idx = np.arange(65, dtype=np.uint64)
    want = np.concatenate([[0.0], np.cumsum(p)])
    assert np.abs(_cdf_closed(pq, idx) - want).max() < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("n,dtype", [(32, np.complex128), (33, np.complex64)])
def test_qft_inverse_known_answer_large(capi, n, dtype):
    """64 GiB states: RY layer, QFT, inverse QFT (fused apply), then <Z_q> for every wire,
    marginals on the highest, lowest and scattered wires, and 4096 sample indices against the
    product state's closed forms."""
    from lightning_b200.workloads import qft_circuit
    c128 = dtype == np.complex128
    ops = qft_circuit(n, seed=9)
    thetas = [op[3][0] for op in ops[:n]]
    assert all(op[0] == "RY" for op in ops[:n])
    undo = [(name, wires, not inv, params) for name, wires, inv, params in reversed(ops[n:])]
    sv = capi.StateVector(n, dtype)
    sv.apply_ops_fused(ops + undo)
    pq = _product_probs(thetas)
    tol = 1e-12 if c128 else 1e-5
    assert abs(sv.norm2() - 1.0) < (1e-12 if c128 else 1e-5)
    z, _ = sv.expval_pauli([("Z", [q]) for q in range(n)])
    assert np.abs(z - np.cos(thetas)).max() < tol
    import lq_oracle as O
    # unsorted wires come out in the reference's transpose_state_tensor order (CS/utils/Util.hpp:465-496)
    for wires in (list(range(10)), list(range(n - 10, n)), [0, n - 1, 15, 16, 30]):
        assert np.abs(sv.probs(wires) - _marginal(pq, O.probs_output_order(wires))).max() < tol, wires
    rng = np.random.default_rng(n)
    u = rng.uniform(size=4096)
    idx = sv.sample(len(u), uniforms=u)
    assert idx.max() >= np.uint64(1 << 31)
    lo, hi = _cdf_closed(pq, idx), _cdf_closed(pq, idx + np.uint64(1))
    slack = 1e-12 if c128 else 1e-5
    assert np.all(lo - slack < u) and np.all(u <= hi + slack)
    sv.close()
