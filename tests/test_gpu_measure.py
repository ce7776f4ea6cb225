"""Measurements on the B200 vs the oracle: probs, expval, var, sampling.

Golden values follow LQ/measurements/tests/Test_MeasurementsLQubit.cpp:41-197 on
the state of CS/utils/TestHelpers.hpp:380-414 (RX then RY with angles 0.7, 0.5, 0.3
on three qubits).  Sample indices are checked bit-exactly against the oracle's
restatement of the inverse-CDF rule fed the same uniforms.
"""
import numpy as np
import pytest

from conftest import TOL, random_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from lightning_b200 import capi as c
    return c


def nontrivial_state_ops():
    angles = [0.7, 0.5, 0.3]
    ops = []
    for q, a in enumerate(angles):
        ops.append(("RX", [q], False, [a]))
        ops.append(("RY", [q], False, [a]))
    return ops


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_golden_expvals(capi, dtype):
    sv = capi.StateVector(3, dtype)
    sv.apply_ops(nontrivial_state_ops())
    tol = 1e-6
    # Test_MeasurementsLQubit.cpp:56-69 (PauliX) and :76-89 (PauliY), :96-109 (PauliZ)
    x = [sv.expval([(1.0, [("PauliX", [w])])]) for w in range(3)]
    y = [sv.expval([(1.0, [("PauliY", [w])])]) for w in range(3)]
    z = [sv.expval([(1.0, [("PauliZ", [w])])]) for w in range(3)]
    assert np.allclose(x, [0.49272486, 0.42073549, 0.28232124], atol=tol)
    assert np.allclose(y, [-0.64421768, -0.47942553, -0.29552020], atol=tol)
    assert np.allclose(z, [0.58498357, 0.77015115, 0.91266780], atol=tol)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_probs(capi, dtype):
    import lq_oracle as O
    rng = np.random.default_rng(2)
    n = 11
    st = random_state(rng, n, dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    tol = 1e-14 if dtype == np.complex128 else 1e-7
    assert np.abs(sv.probs() - O.probs(st)).max() < tol
    for wires in ([0], [n - 1], [3, 1], [1, 3], [2, 7, 5], list(range(n))[::-1], [0, 1, 2, 3, 4, 5, 6, 8, 9, 10],
                  list(range(1, n))):
        assert np.abs(sv.probs(wires) - O.probs(st, wires)).max() < tol * 10, wires


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_pauli_sums_and_hamiltonians(capi, dtype):
    import lq_oracle as O
    rng = np.random.default_rng(4)
    n = 10
    st = random_state(rng, n, dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    st64 = st.astype(np.complex128)
    words = [("Z", [0]), ("X", [3]), ("Y", [9]), ("ZZ", [1, 2]), ("XY", [0, 9]), ("YYZ", [4, 2, 6]),
             ("XX", [5, 8]), ("IZ", [3, 4]), ("ZXZ", [0, 5, 9])]
    coeffs = rng.normal(size=len(words))
    per, tot = sv.expval_pauli(words, coeffs)
    want = [O.pauli_expval(st64, wd, ws) for wd, ws in words]
    tol = 1e-12 if dtype == np.complex128 else 1e-6
    assert np.abs(per - want).max() < tol
    assert abs(tot - float(np.dot(coeffs, want))) < tol * 10
    ham = [(float(c), [({"X": "PauliX", "Y": "PauliY", "Z": "PauliZ", "I": "Identity"}[ch], [w])
                       for ch, w in zip(wd, ws)]) for c, (wd, ws) in zip(coeffs, words)]
    assert abs(sv.expval(ham) - O.expval(st64, ham)) < tol * 10
    assert abs(sv.var(ham) - O.var(st64, ham)) < tol * 20
    # non-Pauli named observables and Hermitian matrices
    herm = rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))
    herm = herm + herm.conj().T
    for terms in ([(1.0, [("Hadamard", [2])])], [(1.0, [("Hermitian", [1, 7], herm)])],
                  [(1.0, [("PauliX", [0]), ("Hermitian", [1, 7], herm)])],
                  [(0.5, [("Hadamard", [3])]), (-2.0, [("Hermitian", [1, 7], herm)])],
                  [(1.0, [("PauliZ", [4])])]):
        assert abs(sv.expval(terms) - O.expval(st64, terms)) < tol * 100
        assert abs(sv.var(terms) - O.var(st64, terms)) < tol * 100


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_pauli_passes_near_and_far(capi, dtype):
    """Pauli sums at 20 qubits, where X masks on the two highest wires (state bits 19, 18) lie
    beyond the shared passes' 4 MiB reach and get pair passes: 70 words (several passes of
    each kind, more than 8 X masks), and single-word variances on an unnormalised state
    (the norm comes from the same pass)."""
    import lq_oracle as O
    rng = np.random.default_rng(21)
    n = 20
    st = (random_state(rng, n, dtype) * 1.3).astype(dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    st64 = st.astype(np.complex128)
    letters = "XYZ"
    words = [("ZZ", [q, (q + 1) % n]) for q in range(n)] + [("X", [q]) for q in range(n)]
    for _ in range(30):
        k = int(rng.integers(1, 4))
        ws = [int(w) for w in rng.choice(n, k, replace=False)]
        words.append(("".join(letters[int(rng.integers(3))] for _ in ws), ws))
    coeffs = rng.normal(size=len(words))
    per, tot = sv.expval_pauli(words, coeffs)
    want = [O.pauli_expval(st64, wd, ws) for wd, ws in words]
    tol = 1e-11 if dtype == np.complex128 else 1e-5
    assert np.abs(per - want).max() < tol
    assert abs(tot - float(np.dot(coeffs, want))) < tol * 10
    names = {"X": "PauliX", "Y": "PauliY", "Z": "PauliZ"}
    for wd, ws in (("X", [0]), ("Y", [1]), ("Z", [5]), ("XY", [0, 19]), ("Y", [19])):
        terms = [(0.7, [(names[c], [w]) for c, w in zip(wd, ws)])]
        assert abs(sv.var(terms) - O.var(st64, terms)) < tol * 10


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("n", [12, 13, 20, 22])
def test_pauli_tiled_passes(capi, dtype, n):
    """Words with X factors packed into tiled passes (12 or 13 tile bits: the words' X bits and the
    lowest state bits, one state read for up to 32 words): one-wire X/Y words on every wire,
    Jordan-Wigner strings, 8 words on one 4-wire X mask (runs of 4 sharing the partner reads),
    40 words on one mask (chunks of 32), masks whose highest bit is a thread bit, a register bit
    or outside the tile's low bits, and words whose masks do not fit a tile with others (multi
    and pair passes), on one tile (12 qubits) and up; per word against the oracle."""
    import lq_oracle as O
    rng = np.random.default_rng(60 + n)
    st = random_state(rng, n, dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    st64 = st.astype(np.complex128)
    words = [("X", [q]) for q in range(n)] + [("YZ", [q, (q + 3) % n]) for q in range(n)]
    from lightning_b200.workloads import jordan_wigner_words
    words += jordan_wigner_words(rng, n, 60)
    quad = [0, 3, n // 2, n - 1]
    words += [("".join(p), quad) for p in ("XXXX", "XXYY", "XYXY", "XYYX", "YXXY", "YXYX", "YYXX", "YYYY")]
    words += [("XXZ", [1, n - 3, 5 + q % 4]) for q in range(40)]
    wide = sorted(int(w) for w in rng.choice(n, 10, replace=False))
    words += [("XXXXXXXX", list(range(n - 8, n))), ("YXYXYXYXYX", wide), ("ZZ", [0, n - 1]), ("Z", [4])]
    coeffs = rng.normal(size=len(words))
    per, tot = sv.expval_pauli(words, coeffs)
    want = np.array([O.pauli_expval(st64, wd, ws) for wd, ws in words])
    tol = TOL[dtype] * (1 if dtype == np.complex128 else 10)
    err = np.abs(per - want)
    assert err.max() < tol, (int(err.argmax()), words[int(err.argmax())], err.max())
    assert abs(tot - float(np.dot(coeffs, want))) < tol * 20


@pytest.mark.parametrize("n", [12, 13, 15])
def test_diagonal_pauli_words_one_pass(capi, n):
    """Many diagonal words (Z and I factors, masks on low, high and both halves of the
    4096-amplitude tiles) in the Walsh-Hadamard pass, from one tile (12 qubits) up."""
    import lq_oracle as O
    rng = np.random.default_rng(40 + n)
    st = random_state(rng, n)
    sv = capi.StateVector(n)
    sv.upload(st)
    words = []
    for _ in range(300):
        k = int(rng.integers(1, 5))
        ws = [int(w) for w in rng.choice(n, k, replace=False)]
        words.append(("".join("Z" if rng.random() < 0.8 else "I" for _ in ws), ws))
    per, _ = sv.expval_pauli(words)
    want = [O.pauli_expval(st, wd, ws) for wd, ws in words]
    assert np.abs(per - want).max() < 1e-12


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_apply_observable_in_place(capi, dtype):
    """psi <- O psi (Observable::applyInPlace): named, tensor, Hermitian and Hamiltonian."""
    import lq_oracle as O
    rng = np.random.default_rng(8)
    n = 9
    st = random_state(rng, n, dtype)
    herm = rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))
    herm = herm + herm.conj().T
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    for terms in ([(1.0, [("PauliY", [4])])], [(1.0, [("PauliX", [0]), ("PauliZ", [8])])],
                  [(1.0, [("Hermitian", [2, 6], herm)])],
                  [(0.5, [("PauliZ", [1]), ("PauliZ", [2])]), (-1.5, [("PauliX", [3])]),
                   (2.0, [("Hermitian", [2, 6], herm)])]):
        sv = capi.StateVector(n, dtype)
        sv.upload(st)
        sv.apply_observable(terms)
        want = O.apply_observable(st.astype(np.complex128), terms)
        assert np.abs(sv.download() - want).max() < tol * (1 + np.abs(want).max())


def test_inner_product_norm(capi):
    rng = np.random.default_rng(6)
    n = 12
    a, b = random_state(rng, n), random_state(rng, n)
    sa, sb = capi.StateVector(n), capi.StateVector(n)
    sa.upload(a)
    sb.upload(b)
    assert abs(sa.inner(sb) - np.vdot(a, b)) < 1e-13
    assert abs(sa.norm2() - 1.0) < 1e-13


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("n", [1, 3, 5, 6, 10, 16])
def test_sampling_bit_exact(capi, n, dtype):
    import lq_oracle as O
    rng = np.random.default_rng(30 + n)
    st = random_state(rng, n, dtype)
    # make some probabilities exactly zero (the rule's edge cases)
    st[rng.choice(st.size, st.size // 4, replace=False)] = 0
    st /= np.linalg.norm(st.astype(np.complex128))
    st = st.astype(dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    u = rng.uniform(size=20000)
    u[:4] = [0.0, 1e-300, np.nextafter(1.0, 0), 0.5]
    cdf = O.cdf_fixed_order(st)
    want = O.sample_kokkos_rule(cdf, u)
    got = sv.sample(len(u), uniforms=u)
    assert np.array_equal(got, want)
    bits = sv.sample_bits(len(u), uniforms=u)
    assert np.array_equal(bits, O.indices_to_bits(want, n))
    # device Philox draws == oracle Philox draws
    got_p = sv.sample(5000, seed=1234567)
    want_p = O.sample_kokkos_rule(cdf, O.philox_uniforms(5000, 1234567))
    assert np.array_equal(got_p, want_p)


def test_sampling_distribution(capi):
    """Histogram of 10^5 shots vs probabilities, margin 0.05 (Test_MeasurementsBase.cpp:364-424)."""
    sv = capi.StateVector(3)
    sv.apply_ops(nontrivial_state_ops())
    p = sv.probs()
    idx = sv.sample(100000, seed=99)
    hist = np.bincount(idx.astype(np.int64), minlength=8) / 1e5
    assert np.allclose(hist, p, atol=0.05)
    assert np.allclose(p, [0.67078706, 0.03062806, 0.0870997, 0.00397696, 0.17564072, 0.00801973,
                           0.02280642, 0.00104134], atol=1e-6)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_sparse_golden(capi, dtype):
    """LQ/measurements/tests/Test_MeasurementsLQubitSparse.cpp:41-78."""
    import lq_oracle as O
    sv = capi.StateVector(3, dtype)
    sv.apply_ops(nontrivial_state_ops())
    csr = O.tridiagonal_periodic_csr(8)
    assert abs(sv.expval_sparse(*csr) - 0.5930885) < 1e-6
    assert abs(sv.var_sparse(*csr) - 2.4624654) < 1e-6
    with pytest.raises(capi.B200Error, match="Statevector and Hamiltonian have incompatible sizes."):
        sv.expval_sparse(*O.tridiagonal_periodic_csr(16))


@pytest.mark.parametrize("n,density", [(1, 1.0), (5, 0.3), (8, 0.03), (10, 0.04), (12, 0.0005), (14, 0.00002)])
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_sparse_vs_oracle(capi, n, density, dtype):
    """Ragged rows (lane widths 1..32 are all reached over the sizes), empty rows,
    unsorted and repeated columns, a row_map that does not start at zero."""
    import scipy.sparse as sp
    import lq_oracle as O
    rng = np.random.default_rng(n)
    N = 1 << n
    A = sp.random(N, N, density=density, format="csr", random_state=n, dtype=np.float64)
    A = (A + 1j * sp.random(N, N, density=density, format="csr", random_state=n + 1)).tocsr()
    A.data[::5] = 0  # explicit zeros stay in the structure
    indptr = A.indptr.astype(np.uint64) + 7
    indices = A.indices.astype(np.uint64)
    perm = np.concatenate([rng.permutation(np.arange(a, b)) for a, b in zip(A.indptr[:-1], A.indptr[1:])]
                          or [np.zeros(0, int)]).astype(np.int64)
    indices, data = indices[perm], A.data[perm].astype(dtype)
    if len(indices) > 1:
        indices[1] = indices[0]  # a repeated column inside a row is summed as given
    st = random_state(rng, n, dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    want_e = O.sparse_expval(st, indptr - 7, indices, data)
    want_v = O.sparse_var(st, indptr - 7, indices, data)
    tol = 1e-10 if dtype == np.complex128 else 1e-4
    scale = max(1.0, abs(want_v))
    assert abs(sv.expval_sparse(indptr, indices, data) - want_e) < tol * scale
    assert abs(sv.var_sparse(indptr, indices, data) - want_v) < tol * scale


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_sparse_device_arrays(capi, dtype):
    """The CSR arrays in device memory give the host-array results; bad arrays are rejected
    with the same messages (checked on the device)."""
    import torch
    import lq_oracle as O
    rng = np.random.default_rng(31)
    n = 9
    st = random_state(rng, n, dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    indptr, indices, data = O.tridiagonal_periodic_csr(1 << n)
    data = (data * rng.normal(size=data.size)).astype(dtype)
    tdt = torch.complex64 if dtype == np.complex64 else torch.complex128
    dp = torch.tensor(indptr.astype(np.int64), device="cuda")
    di = torch.tensor(indices.astype(np.int64), device="cuda")
    dv = torch.tensor(data, dtype=tdt, device="cuda")
    got = sv.expval_sparse_device(dp.data_ptr(), di.data_ptr(), dv.data_ptr(), data.size)
    assert got == sv.expval_sparse(indptr, indices, data)
    gv = sv.var_sparse_device(dp.data_ptr(), di.data_ptr(), dv.data_ptr(), data.size)
    assert gv == sv.var_sparse(indptr, indices, data)
    tol = 1e-12 if dtype == np.complex128 else 1e-5
    assert abs(got - O.sparse_expval(st.astype(np.complex128), indptr, indices, data.astype(np.complex128))) < tol
    bad = di.clone()
    bad[7] = 1 << n
    with pytest.raises(capi.B200Error, match="column index out of range"):
        sv.expval_sparse_device(dp.data_ptr(), bad.data_ptr(), dv.data_ptr(), data.size)
    with pytest.raises(capi.B200Error, match="more non-zeros"):
        sv.expval_sparse_device(dp.data_ptr(), di.data_ptr(), dv.data_ptr(), data.size - 3)
    rows = dp.clone()
    rows[5], rows[6] = dp[6], dp[5]
    with pytest.raises(capi.B200Error, match="non-decreasing"):
        sv.expval_sparse_device(rows.data_ptr(), di.data_ptr(), dv.data_ptr(), data.size)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_sparse_host_arrays_staged(capi, dtype):
    """Host CSR arrays above the staging threshold (20 qubits, 16 non-zeros a row: 134 MB of
    column indices and 134-268 MB of values, several 64 MiB staging chunks each) give exactly
    the device-array result, twice in a row (the staging halves are reused), from pageable and
    from pinned host memory, and agree with scipy's CSR product."""
    import scipy.sparse as sp
    import torch
    rng = np.random.default_rng(77)
    n, per_row = 20, 16
    N = 1 << n
    st = random_state(rng, n, dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    indptr = np.arange(0, N * per_row + 1, per_row, dtype=np.uint64)
    indices = rng.integers(0, N, size=N * per_row, dtype=np.uint64)
    data = (rng.normal(size=N * per_row) + 1j * rng.normal(size=N * per_row)).astype(dtype)
    tdt = torch.complex64 if dtype == np.complex64 else torch.complex128
    dp = torch.tensor(indptr.astype(np.int64), device="cuda")
    di = torch.tensor(indices.astype(np.int64), device="cuda")
    dv = torch.tensor(data, dtype=tdt, device="cuda")
    want = sv.expval_sparse_device(dp.data_ptr(), di.data_ptr(), dv.data_ptr(), data.size)
    assert sv.expval_sparse(indptr, indices, data) == want
    assert sv.expval_sparse(indptr, indices, data) == want
    assert sv.var_sparse(indptr, indices, data) == sv.var_sparse_device(dp.data_ptr(), di.data_ptr(),
                                                                       dv.data_ptr(), data.size)
    pinned_cols = torch.from_numpy(indices.view(np.int64)).pin_memory()
    pinned_vals = torch.from_numpy(data).pin_memory()
    assert sv.expval_sparse(indptr, pinned_cols.numpy().view(np.uint64), pinned_vals.numpy()) == want
    H = sp.csr_matrix((data.astype(np.complex128), indices.astype(np.int64), indptr.astype(np.int64)), shape=(N, N))
    psi = st.astype(np.complex128)
    ref = float(np.real(np.vdot(psi, H @ psi)))
    tol = 1e-10 if dtype == np.complex128 else 1e-3
    assert abs(want - ref) < tol * max(1.0, abs(ref))


def test_sparse_rejects_bad_csr(capi):
    sv = capi.StateVector(2)
    rows = np.array([0, 1, 2, 3, 4], dtype=np.uint64)
    with pytest.raises(capi.B200Error, match="column index out of range"):
        sv.expval_sparse(rows, np.array([0, 1, 2, 4], dtype=np.uint64), np.ones(4))
    with pytest.raises(capi.B200Error, match="non-decreasing"):
        sv.expval_sparse(np.array([0, 2, 1, 3, 4], dtype=np.uint64), np.zeros(4, dtype=np.uint64), np.ones(4))
    with pytest.raises(capi.B200Error, match="more non-zeros"):
        sv.expval_sparse(rows, np.zeros(3, dtype=np.uint64), np.ones(3))
    assert sv.expval_sparse(np.zeros(5, dtype=np.uint64), np.zeros(0, dtype=np.uint64), np.zeros(0)) == 0.0


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("proposal", [0, 1])
@pytest.mark.parametrize("n,burnin,shots,chains", [(1, 0, 50, 1), (3, 13, 640, 7), (8, 50, 3000, 64),
                                                   (11, 5, 5000, 4096)])
def test_mcmc_bit_exact(capi, dtype, proposal, n, burnin, shots, chains):
    """Metropolis chains: the same indices as the oracle's restatement for the same seed."""
    import lq_oracle as O
    rng = np.random.default_rng(n + 10 * proposal)
    st = random_state(rng, n, np.complex128)
    st[rng.integers(0, 1 << n, size=max(1, (1 << n) // 4))] = 0  # zero-probability states
    st /= np.linalg.norm(st)
    st = st.astype(dtype)
    sv = capi.StateVector(n, dtype)
    sv.upload(st)
    got = sv.sample_mcmc(proposal, burnin, shots, chains, seed=1234 + n)
    want = O.mcmc_chains(st, proposal, burnin, shots, chains, seed=1234 + n)
    assert np.array_equal(got, want)


def test_mcmc_distribution_and_errors(capi):
    import lq_oracle as O
    rng = np.random.default_rng(2)
    n = 10
    st = random_state(rng, n)
    sv = capi.StateVector(n)
    sv.upload(st)
    p = O.probs(st)
    for proposal in (0, 1):
        # one sample per chain after burn-in: independent draws, so chi^2 needs no
        # correction for the correlation between consecutive steps of a chain
        idx = sv.sample_mcmc(proposal, 300, 200000, 200000, seed=5)
        counts = np.bincount(idx.astype(np.int64), minlength=1 << n)
        # coarse bins over the top 5 qubits: chi^2 per degree of freedom near 1
        c5 = counts.reshape(32, -1).sum(1)
        p5 = p.reshape(32, -1).sum(1) * len(idx)
        chi2 = ((c5 - p5) ** 2 / p5).sum() / 31
        assert chi2 < 3.0, (proposal, chi2)
    z = capi.StateVector(3)
    z.upload(np.zeros(8))
    with pytest.raises(capi.B200Error, match="no basis state has a non-zero amplitude"):
        z.sample_mcmc(1, 10, 100)
    with pytest.raises(capi.B200Error, match="chains must be positive"):
        sv.sample_mcmc(0, 10, 100, 0)


@pytest.mark.parametrize("kernel", ["Local", "NonZeroRandom"])
def test_mcmc_reference_golden(kernel):
    """Test_MeasurementsLQubit.cpp:199-320 through the module surface
    (generate_mcmc_samples(num_wires, kernelname, num_burnin, num_shots))."""
    import lightning_b200.lightning_qubit_ops as m
    st = np.zeros(8, dtype=np.complex128)
    st[0] = 1
    sv = m.StateVectorC128(st)
    for op in nontrivial_state_ops():
        getattr(sv, op[0])(op[1], False, op[3])
    bits = np.asarray(m.MeasurementsC128(sv).generate_mcmc_samples(3, kernel, 1000, 100000))
    assert bits.shape == (100000, 3)
    idx = bits[:, 0] * 4 + bits[:, 1] * 2 + bits[:, 2]
    got = np.bincount(idx, minlength=8) / 100000
    want = [0.67078706, 0.03062806, 0.0870997, 0.00397696, 0.17564072, 0.00801973, 0.02280642, 0.00104134]
    assert np.abs(got - want).max() < 0.05
