"""Pins the CPU oracle (oracle/lq_oracle.py) before it is trusted as the checker.

* golden values asserted by the reference's own C++ tests (cited per case);
* outputs of the reference itself, committed as fixtures by tests/golden/make_golden.py;
* live comparison with the reference module when oracle/_ref is built;
* published Philox4x32-10 known-answer vectors (Random123 kat_vectors);
* the inverse-CDF rule against a literal scalar restatement of
  LK/measurements/MeasuresFunctors.hpp:70-103.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import lq_oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
P = [-np.pi / 7, np.pi / 5, 2 * np.pi / 3]


def nontrivial_state():
    """CS/utils/TestHelpers.hpp:380-414: RX then RY with angles 0.7, 0.5, 0.3."""
    ops = []
    for q, a in enumerate([0.7, 0.5, 0.3]):
        ops += [("RX", [q], False, [a]), ("RY", [q], False, [a])]
    return O.run_circuit(3, ops)


def test_measurement_golden_values():
    st = nontrivial_state()
    # LQ/measurements/tests/Test_MeasurementsLQubit.cpp:56-116
    x = [O.expval(st, [(1.0, [("PauliX", [w])])]) for w in range(3)]
    y = [O.expval(st, [(1.0, [("PauliY", [w])])]) for w in range(3)]
    z = [O.expval(st, [(1.0, [("PauliZ", [w])])]) for w in range(3)]
    assert np.allclose(x, [0.49272486, 0.42073549, 0.28232124], atol=1e-6)
    assert np.allclose(y, [-0.64421768, -0.47942553, -0.29552020], atol=1e-6)
    assert np.allclose(z, [0.58498357, 0.77015115, 0.91266780], atol=1e-6)


def test_probs_golden_permutations():
    """CS/measurements/tests/Test_MeasurementsBase.cpp:96-118."""
    st = nontrivial_state()
    cases = {(0, 1, 2): [0.67078706, 0.03062806, 0.0870997, 0.00397696, 0.17564072, 0.00801973, 0.02280642, 0.00104134],
             (0, 2, 1): [0.67078706, 0.0870997, 0.03062806, 0.00397696, 0.17564072, 0.02280642, 0.00801973, 0.00104134],
             (1, 0, 2): [0.67078706, 0.03062806, 0.17564072, 0.00801973, 0.0870997, 0.00397696, 0.02280642, 0.00104134],
             (1, 2, 0): [0.67078706, 0.0870997, 0.17564072, 0.02280642, 0.03062806, 0.00397696, 0.00801973, 0.00104134]}
    for wires, want in cases.items():
        assert np.allclose(O.probs(st, list(wires)), want, atol=1e-6), wires


def test_adjoint_golden_values():
    """CS/algorithms/tests/Test_AdjointJacobian.cpp:283-418, :486-554."""
    def jac(n, ops, obs, tp, init=None):
        psi = O.zero_state(n) if init is None else np.asarray(init, dtype=complex)
        return O.adjoint_jacobian(psi, ops, obs, tp, apply_operations=True)
    ops = [("RX", [i], False, [P[i]]) for i in range(3)]
    zzz = [[(1.0, [("PauliZ", [0]), ("PauliZ", [1]), ("PauliZ", [2])])]]
    assert np.allclose(jac(3, ops, zzz, [0, 1, 2])[0], [-0.1755096592645253, 0.26478810666384334,
                                                        -0.6312451595102775], atol=1e-7)
    names = ["RZ", "RY", "RZ", "CNOT", "CNOT", "RZ", "RY", "RZ"]
    params = [[P[0]], [P[1]], [P[2]], [], [], [P[0]], [P[1]], [P[2]]]
    wires = [[0], [0], [0], [0, 1], [1, 2], [1], [1], [1]]
    xxx = [[(1.0, [("PauliX", [0]), ("PauliX", [1]), ("PauliX", [2])])]]
    got = jac(3, [(a, w, False, p) for a, w, p in zip(names, wires, params)], xxx, list(range(6)))
    assert np.allclose(got[0], [0, -0.674214427, 0.275139672, 0.275139672, -0.0129093062, 0.323846156], atol=1e-7)
    theta = np.linspace(-2 * np.pi, 2 * np.pi, 7)[1]
    lp = [theta, theta ** 3, np.sqrt(2) * theta]
    rot = [("RZ", [0], False, [lp[0]]), ("RY", [0], False, [lp[1]]), ("RZ", [0], False, [lp[2]])]
    got = jac(1, rot, [[(1.0, [("PauliZ", [0])])]], [0, 1, 2], init=[1 / np.sqrt(2), -1 / np.sqrt(2)])
    assert np.allclose(got[0], [-8.18996553e-01, 1.62526544e-01, 0], atol=1e-4)
    ham = [[(0.47, [("PauliZ", [0])]), (0.32, [("PauliZ", [1])]), (0.96, [("PauliZ", [2])])]]
    assert np.allclose(jac(3, ops, ham, [0, 2])[0], [-0.47 * np.sin(P[0]), -0.96 * np.sin(P[2])], atol=1e-7)


def test_generator_definition():
    """i G |psi> = dU/dtheta |psi> at theta = 0 (LQ/gates/tests/Test_GateImplementations_Generator.cpp:30-40)."""
    rng = np.random.default_rng(1)
    st = rng.normal(size=32) + 1j * rng.normal(size=32)
    for name in O.GEN_OF_GATE:
        k = {"PhaseShift": 1, "RX": 1, "RY": 1, "RZ": 1, "MultiRZ": 3}.get(name, 4 if "Double" in name else 2)
        g, s = O.apply_generator(st, name, list(range(k)))
        eps = 1e-6
        d = (O.apply_op(st, name, list(range(k)), False, [eps]) - O.apply_op(st, name, list(range(k)), False, [-eps]))
        assert np.abs(1j * s * g - d / (2 * eps)).max() < 1e-8, name


def test_oracle_matches_reference_fixtures():
    data = np.load(GOLDEN / "reference_outputs.npz")
    meta = json.loads((GOLDEN / "reference_outputs.json").read_text())
    st = data["gate_input"]
    for i, (name, wires, inv, params) in enumerate(meta["gates"]):
        want = data[f"gate{i}_c128"]
        assert np.abs(O.apply_op(st, name, wires, inv, params) - want).max() < 1e-14, name
        # complex64: the reference rounds in float; agreement to float precision
        got64 = O.apply_op(st.astype(np.complex64).astype(np.complex128), name, wires, inv, params)
        assert np.abs(got64 - data[f"gate{i}_c64"]).max() < 5e-7, name
    import sys
    sys.path.insert(0, str(GOLDEN))
    from make_golden import obs_cases, adjoint_cases
    s6 = data["meas_input"]
    assert np.abs(O.probs(s6) - data["probs_all"]).max() < 1e-15
    assert np.abs(O.probs(s6, [4, 1, 3]) - data["probs_413"]).max() < 1e-15
    for k, terms in obs_cases().items():
        assert abs(O.expval(s6, terms) - data[f"ev_{k}"]) < 1e-14, k
        assert abs(O.var(s6, terms) - data[f"var_{k}"]) < 1e-13, k
    for j, (n, ops, obs, tp) in enumerate(adjoint_cases()):
        got = O.adjoint_jacobian(O.run_circuit(n, ops), ops, obs, tp)
        assert np.abs(got - data[f"adj{j}"]).max() < 1e-14, j


def test_oracle_matches_live_reference(ref_module):
    import ref
    rng = np.random.default_rng(3)
    from lightning_b200.workloads import gate_sweep
    ops = gate_sweep(7, 80, seed=11)
    a = O.run_circuit(7, ops)
    b = ref.run_circuit(ref_module, 7, ops)
    assert np.abs(a - b).max() < 1e-13
    st = rng.normal(size=128) + 1j * rng.normal(size=128)
    st /= np.linalg.norm(st)
    for w in ([0], [6, 2], [3, 5, 1, 0]):
        assert np.abs(O.probs(st, w) - ref.probs(ref_module, st, w)).max() < 1e-15


def test_philox_known_answers():
    """Random123 kat_vectors, philox4x32 with 10 rounds."""
    z = np.zeros(1, np.uint64)
    f = np.full(1, 0xFFFFFFFF, np.uint64)
    a = lambda v: np.full(1, v, np.uint64)  # noqa: E731
    cases = [((z, z, z, z, 0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
             ((f, f, f, f, 0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
             ((a(0x243F6A88), a(0x85A308D3), a(0x13198A2E), a(0x03707344), 0xA4093822, 0x299F31D0),
              (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for args, want in cases:
        got = tuple(int(x[0]) for x in O.philox4x32_10(*args))
        assert got == want
    u = O.philox_uniforms(100000, 42)
    assert u.min() >= 0 and u.max() < 1 and abs(u.mean() - 0.5) < 0.005


def _kokkos_scalar(cdf, U):
    """Literal restatement of Sampler::operator() (MeasuresFunctors.hpp:70-103)."""
    length = len(cdf)
    if U <= cdf[1]:
        return 0
    low, high = 1, length
    while high - low > 1:
        mid = high - ((high - low) >> 1)
        cdf_t = 1.0 if mid == length else cdf[mid]
        if cdf_t < U:
            low = mid
        else:
            high = mid
    return high - 1


@pytest.mark.parametrize("n", [1, 2, 5, 6, 11])
def test_cdf_and_sampling_rule(n):
    rng = np.random.default_rng(n)
    st = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    st[rng.choice(st.size, st.size // 3, replace=False)] = 0
    st /= np.linalg.norm(st)
    cdf = O.cdf_fixed_order(st)
    p = np.abs(st) ** 2
    assert cdf[0] == 0.0
    assert np.abs(cdf - np.concatenate([[0], np.cumsum(p)[:-1]])).max() < 1e-14
    u = np.concatenate([rng.uniform(size=500), [0.0, 1e-300, np.nextafter(1.0, 0.0), cdf[1], cdf[-1]]])
    got = O.sample_kokkos_rule(cdf, u)
    want = [_kokkos_scalar(cdf, x) for x in u]
    assert np.array_equal(got, np.array(want, dtype=np.uint64))
    # a sample never lands on a zero-probability index unless U sits exactly on a CDF step
    assert np.all(p[got.astype(int)[:500]] > 0)


def test_cdf_association_order_is_hierarchical():
    """The fixed order differs from a flat running sum in the last bits for long inputs:
    the oracle must reproduce the engine's order, not numpy's cumsum."""
    rng = np.random.default_rng(0)
    st = (rng.uniform(size=1 << 16) + 1j * rng.uniform(size=1 << 16))
    st /= np.linalg.norm(st)
    cdf = O.cdf_fixed_order(st)
    flat = np.concatenate([[0.0], np.cumsum(np.abs(st) ** 2)[:-1]])
    assert np.abs(cdf - flat).max() < 1e-12
    assert not np.array_equal(cdf, flat)


def test_finite_difference_agrees_with_adjoint():
    from lightning_b200.workloads import layered_rotations
    ops, obs, tp = layered_rotations(n=4, layers=2, seed=3)
    adj = O.adjoint_jacobian(O.run_circuit(4, ops), ops, obs, tp)
    fd = O.finite_difference_jacobian(4, ops, obs, h=1e-5)
    assert np.abs(adj - fd).max() < 1e-8


def test_vjp_state_matches_live_reference(ref_module):
    import ref
    from lightning_b200.workloads import layered_rotations
    rng = np.random.default_rng(8)
    ops, _, _ = layered_rotations(n=5, layers=2, seed=21)
    ops = ops + [("CRY", [0, 3], True, [0.7]), ("IsingXY", [1, 4], False, [0.4]), ("PhaseShift", [2], True, [1.2])]
    psi = O.run_circuit(5, ops)
    dy = rng.normal(size=32) + 1j * rng.normal(size=32)
    npar = sum(1 for op in ops if op[3])
    tp = list(range(0, npar, 3))
    a = O.vjp_state(psi, ops, dy, tp)
    b = ref.vjp_state(ref_module, psi.copy(), ops, dy, tp)
    assert np.abs(a - b).max() < 1e-13


def test_sparse_golden_values():
    """LQ/utils/tests/Test_SparseLinAlg.cpp:33-70 (CSR product) and
    LQ/measurements/tests/Test_MeasurementsLQubitSparse.cpp:41-61 (expval, var) on the
    periodic tridiagonal matrix of CS/utils/TestHelpers.hpp:430-470."""
    indptr, indices, data = O.tridiagonal_periodic_csr(8)
    v1 = np.array([0.33160916, 0.90944626, 0.81097291, 0.46112135, 0.42801563, 0.38077181, 0.23550137, 0.57416324])
    r1 = [-1.15200034, -0.23313581, -0.5595947, -0.7778672, -0.41387753, -0.28274519, -0.71943368, 0.00705271]
    v2 = np.array([0.26752544 + 0.00484225j, 0.49189265 + 0.21231633j, 0.28691029 + 0.87552205j,
                   0.13499786 + 0.63862517j, 0.31748372 + 0.25701515j, 0.96968437 + 0.69821151j,
                   0.53674213 + 0.58564544j, 0.02213429 + 0.3050882j])
    r2 = np.array([-0.24650151 - 0.51256229j, -0.06254307 - 0.66804797j, -0.33998022 + 0.02458055j,
                   -0.46939616 - 0.49391203j, -0.7871985 - 1.07982153j, 0.11545852 - 0.14444908j,
                   -0.45507653 - 0.41765428j, -0.78213328 - 0.28539948j])
    assert np.allclose(O.sparse_matvec(v1, indptr, indices, data), r1, atol=1e-6)
    assert np.allclose(O.sparse_matvec(v2, indptr, indices, data), r2, atol=1e-6)
    st = nontrivial_state()
    assert abs(O.sparse_expval(st, indptr, indices, data) - 0.5930885) < 1e-6
    assert abs(O.sparse_var(st, indptr, indices, data) - 2.4624654) < 1e-6
    with pytest.raises(ValueError, match="incompatible sizes"):
        O.sparse_expval(st, *O.tridiagonal_periodic_csr(16))


def random_csr(n, rng, density=0.3, empty_rows=True):
    """Random complex CSR matrix with ragged rows (some empty) and unsorted columns."""
    N = 1 << n
    rows, cols, vals = [0], [], []
    for r in range(N):
        k = 0 if (empty_rows and r % 7 == 3) else int(rng.integers(0, max(2, int(density * N)) + 1))
        c = rng.choice(N, size=k, replace=False)
        cols += list(c)
        vals += list(rng.normal(size=k) + 1j * rng.normal(size=k))
        rows.append(len(cols))
    return (np.array(rows, dtype=np.uint64), np.array(cols, dtype=np.uint64), np.array(vals, dtype=np.complex128))


def test_sparse_matches_live_reference(ref_module):
    import ref
    rng = np.random.default_rng(17)
    for n in (1, 3, 6):
        st = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        st /= np.linalg.norm(st)
        csr = random_csr(n, rng)
        assert abs(O.sparse_expval(st, *csr) - ref.sparse_expval(ref_module, st, *csr)) < 1e-12
        assert abs(O.sparse_var(st, *csr) - ref.sparse_var(ref_module, st, *csr)) < 1e-12


@pytest.mark.parametrize("proposal", [O.MCMC_LOCAL, O.MCMC_NONZERO])
def test_mcmc_chains_match_reference_histogram(proposal):
    """LQ/measurements/tests/Test_MeasurementsLQubit.cpp:199-320: 10^5 Metropolis samples
    after 1000 burn-in steps on the non-trivial state reproduce its probabilities within 0.05."""
    st = nontrivial_state()
    want = [0.67078706, 0.03062806, 0.0870997, 0.00397696, 0.17564072, 0.00801973, 0.02280642, 0.00104134]
    idx = O.mcmc_chains(st, proposal, 1000, 100000, 256, seed=3)
    got = np.bincount(idx.astype(np.int64), minlength=8) / 100000
    assert np.abs(got - want).max() < 0.05
    assert np.abs(got - O.probs(st)).max() < 0.01


def test_mcmc_kernel_name_binding():
    """kernel_factory (TransitionKernels.hpp:147-159) builds the non-zero kernel for the name
    "Local" and the local kernel for "NonZeroRandom"."""
    assert O.mcmc_kernel_for_name("Local") == O.MCMC_NONZERO
    assert O.mcmc_kernel_for_name("NonZeroRandom") == O.MCMC_LOCAL
    assert O.mcmc_kernel_for_name("anything") == O.MCMC_NONZERO


def test_mcmc_local_chain_stays_in_support():
    """From |0...0>, local moves to zero-probability states are never accepted (p_t = 0 < U p_i)."""
    st = np.zeros(16, dtype=np.complex128)
    st[0] = st[5] = 1 / np.sqrt(2)
    idx = O.mcmc_chains(st, O.MCMC_LOCAL, 10, 500, 5, seed=9)
    assert set(idx.tolist()) <= {0}
    idx = O.mcmc_chains(st, O.MCMC_NONZERO, 10, 2000, 5, seed=9)
    assert set(idx.tolist()) == {0, 5}


def test_mcmc_reference_module_histogram(ref_module):
    """The reference's own generate_mcmc_samples (unseeded) gives the same distribution."""
    st = nontrivial_state()
    for name in ("Local", "NonZeroRandom"):
        sv = ref_module.StateVectorC128(st.copy())
        bits = np.asarray(ref_module.MeasurementsC128(sv).generate_mcmc_samples(3, name, 1000, 50000))
        idx = bits[:, 0] * 4 + bits[:, 1] * 2 + bits[:, 2]
        got = np.bincount(idx, minlength=8) / 50000
        assert np.abs(got - O.probs(st)).max() < 0.02, name
