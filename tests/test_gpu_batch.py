"""Batched engine on the B200 vs the FP64 oracle: forward expectation values,
vector-Jacobian products through torch.autograd and full per-circuit Jacobians.

Circuit widths straddle the on-chip threshold so both the shared-memory-resident
path and the tiled HBM path run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Gradient bounds against the FP64 oracle: 1e-12 for complex128, 1e-5 for complex64 (FP32
# amplitudes, compensated gate arithmetic, FP64 inner products).
GRAD_TOL = {np.complex128: 1e-12, np.complex64: 1e-5}


def small_hea(dtype, seed=3):
    from lightning_b200.workloads import hea_batch
    return hea_batch(ncirc=24, nmin=3, nmax=15 if dtype == np.complex64 else 14, dmin=1, dmax=3, seed=seed)


def mixed_batch(seed=8):
    """Circuits using every gate kind the batch supports, with shared and constant parameters."""
    rng = np.random.default_rng(seed)
    circuits, params = [], list(rng.uniform(0, 2 * np.pi, 6))
    kinds1 = ["RX", "RY", "RZ", "PhaseShift"]
    kinds2 = ["CRX", "CRY", "CRZ", "ControlledPhaseShift", "IsingXX", "IsingYY", "IsingZZ", "IsingXY",
              "SingleExcitation", "SingleExcitationMinus", "SingleExcitationPlus"]
    const = ["Hadamard", "PauliX", "PauliY", "PauliZ", "S", "T", "Identity"]
    for c in range(10):
        n = [3, 5, 9, 13, 14, 15][c % 6]
        ops, pidx = [], []
        for _ in range(30):
            r = rng.random()
            if r < 0.3:
                ops.append((kinds1[rng.integers(4)], [int(rng.integers(n))], bool(rng.random() < 0.3), []))
                pidx.append(len(params))
                params.append(float(rng.uniform(0, 2 * np.pi)))
            elif r < 0.55:
                w = [int(x) for x in rng.choice(n, 2, replace=False)]
                ops.append((kinds2[rng.integers(len(kinds2))], w, bool(rng.random() < 0.3), []))
                pidx.append(len(params))
                params.append(float(rng.uniform(0, 2 * np.pi)))
            elif r < 0.65:  # shared parameter slot
                ops.append(("RY", [int(rng.integers(n))], False, []))
                pidx.append(int(rng.integers(6)))
            elif r < 0.75:
                ops.append(("RX", [int(rng.integers(n))], False, [float(rng.uniform(0, 6))]))  # constant angle
                pidx.append(-1)
            elif r < 0.85:
                ops.append((const[rng.integers(len(const))], [int(rng.integers(n))], False, []))
                pidx.append(-1)
            else:
                k = 3 if n >= 3 and rng.random() < 0.3 else 2
                name = {2: ["CNOT", "CZ", "SWAP", "CY"][rng.integers(4)], 3: ["Toffoli", "CSWAP"][rng.integers(2)]}[k]
                ops.append((name, [int(x) for x in rng.choice(n, k, replace=False)], False, []))
                pidx.append(-1)
        ops.append(("MultiRZ", [0, n - 1], False, []))
        pidx.append(len(params))
        params.append(0.77)
        obs = [[(0.5, "Z", [0]), (-1.5, "XZ", [n - 1, 1 % n])], [(1.0, "Y", [n // 2])], [(0.3, "ZZ", [0, n - 1])]]
        circuits.append({"num_qubits": n, "ops": ops, "param_index": pidx, "observables": obs})
    return circuits, np.array(params)


def oracle_outputs(circuits, params):
    import lq_oracle as O
    from lightning_b200.workloads import bind, obs_terms
    out = []
    for c in circuits:
        st = O.run_circuit(c["num_qubits"], bind(c, params))
        out += [O.expval(st, obs_terms(ob)) for ob in c["observables"]]
    return np.array(out)


def oracle_vjp(circuits, params, dy):
    import lq_oracle as O
    from lightning_b200.workloads import bind, obs_terms
    grad = np.zeros(len(params))
    k = 0
    for c in circuits:
        ops = bind(c, params)
        n = c["num_qubits"]
        obs = [obs_terms(ob) for ob in c["observables"]]
        slots = [p for p in c["param_index"] if p >= 0]
        tp = list(range(len(slots)))
        psi = O.run_circuit(n, ops)
        # only ops with a slot are trainable; constant-angle ops are parametric but not trainable
        pops = [i for i, op in enumerate(ops) if len(op[3]) > 0]
        trainable = [j for j, i in enumerate(pops) if c["param_index"][i] >= 0]
        j = O.adjoint_jacobian(psi, ops, obs, trainable)
        for oi in range(len(obs)):
            for col, i in enumerate([pops[t] for t in trainable]):
                grad[c["param_index"][i]] += dy[k + oi] * j[oi, col]
        k += len(obs)
        del tp
    return grad


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("maker", ["hea", "mixed"])
def test_batch_forward_and_vjp(dtype, maker):
    import torch
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.autograd import batched_expval
    circuits, params = small_hea(dtype) if maker == "hea" else mixed_batch()
    eng = BatchedCircuits(circuits, len(params), dtype=dtype, use_graphs=False)
    p = torch.tensor(params, dtype=torch.float64, device="cuda", requires_grad=True)
    out = batched_expval(p, eng)
    want = oracle_outputs(circuits, params)
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    assert np.abs(out.detach().cpu().numpy() - want).max() < tol
    rng = np.random.default_rng(1)
    dy = rng.normal(size=out.numel())
    (out * torch.tensor(dy, device="cuda")).sum().backward()
    gwant = oracle_vjp(circuits, params, dy)
    assert np.abs(p.grad.cpu().numpy() - gwant).max() < GRAD_TOL[dtype]


def wide_gate_batch(seed=31):
    """Circuits with the four-wire double excitations (trainable, shared-slot and constant
    angles, inverted) and constant matrices on 3 and 4 wires, between layers of rotations and
    CNOTs; widths on both sides of the on-chip threshold."""
    from lightning_b200.workloads import random_unitary
    rng = np.random.default_rng(seed)
    circuits, params = [], list(rng.uniform(0, 2 * np.pi, 4))
    de = ["DoubleExcitation", "DoubleExcitationMinus", "DoubleExcitationPlus"]
    for c in range(9):
        n = [4, 6, 9, 12, 13, 14, 15, 5, 11][c]
        ops, pidx = [], []
        for layer in range(3):
            for q in range(n):
                ops.append((["RX", "RY"][(q + layer) % 2], [q], False, []))
                pidx.append(len(params))
                params.append(float(rng.uniform(0, 2 * np.pi)))
            for _ in range(3):
                w = [int(x) for x in rng.choice(n, 4, replace=False)]
                r = rng.random()
                if r < 0.5:
                    ops.append((de[int(rng.integers(3))], w, bool(rng.random() < 0.3), []))
                    pidx.append(len(params))
                    params.append(float(rng.uniform(0, 2 * np.pi)))
                elif r < 0.65:
                    ops.append((de[int(rng.integers(3))], w, False, []))
                    pidx.append(int(rng.integers(4)))  # shared slot
                elif r < 0.8:
                    ops.append((de[int(rng.integers(3))], w, bool(rng.random() < 0.5), [float(rng.uniform(0, 6))]))
                    pidx.append(-1)  # constant angle
                else:
                    k = 3 if rng.random() < 0.5 else 4
                    ops.append(("QubitUnitary", w[:k], bool(rng.random() < 0.5), [], random_unitary(rng, k)))
                    pidx.append(-1)
            for q in range(0, n - 1, 2):
                ops.append(("CNOT", [q, q + 1], False, []))
                pidx.append(-1)
        obs = [[(1.0, "Z", [0])], [(0.7, "XY", [n - 1, 1]), (-0.4, "ZZ", [2, n - 1])], [(1.0, "Y", [n // 2])]]
        circuits.append({"num_qubits": n, "ops": ops, "param_index": pidx, "observables": obs})
    return circuits, np.array(params)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_batch_double_excitations_and_wide_matrices(dtype):
    """Four-wire double excitations (their generators in the VJP) and 3-/4-wire matrices in the
    batched engine: forward outputs, the VJP and the full Jacobian against the FP64 oracle."""
    import torch
    from lightning_b200.batch import BatchedCircuits
    circuits, params = wide_gate_batch()
    eng = BatchedCircuits(circuits, len(params), dtype=dtype, use_graphs=False)
    p = torch.tensor(params, dtype=torch.float64, device="cuda")
    out = eng.forward(p).cpu().numpy()
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    assert np.abs(out - oracle_outputs(circuits, params)).max() < tol
    rng = np.random.default_rng(2)
    dy = rng.normal(size=out.size)
    g = eng.vjp(p, torch.tensor(dy, device="cuda")).cpu().numpy()
    assert np.abs(g - oracle_vjp(circuits, params, dy)).max() < GRAD_TOL[dtype]
    # Jacobian blocks [nobs x trainable ops] per circuit against the oracle's adjoint Jacobian
    import lq_oracle as O
    from lightning_b200.workloads import bind, obs_terms
    jac = eng.jacobian(p).cpu().numpy()
    k = 0
    for c in circuits:
        ops = bind(c, params)
        pops = [i for i, op in enumerate(ops) if len(op[3]) > 0]
        trainable = [j for j, i in enumerate(pops) if c["param_index"][i] >= 0]
        want = O.adjoint_jacobian(O.run_circuit(c["num_qubits"], ops), ops,
                                  [obs_terms(ob) for ob in c["observables"]], trainable)
        got = jac[k:k + want.size].reshape(want.shape)
        k += want.size
        assert np.abs(got - want).max() < GRAD_TOL[dtype]


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_batch_graphs_and_autotune_repeatable(dtype):
    import torch
    from lightning_b200.batch import BatchedCircuits
    circuits, params = small_hea(dtype, seed=9)
    eng = BatchedCircuits(circuits, len(params), dtype=dtype, use_graphs=True)
    p = torch.tensor(params, dtype=torch.float64, device="cuda")
    a = eng.forward(p)
    b = eng.forward(p)  # graph replay
    assert torch.equal(a, b)
    dy = torch.ones_like(a)
    g1 = eng.vjp(p, dy)
    eng.autotune(p)
    g2 = eng.vjp(p, dy)
    c = eng.forward(p)
    assert np.abs(a.cpu().numpy() - oracle_outputs(circuits, params)).max() < (1e-12 if dtype == np.complex128 else 2e-5)
    assert torch.allclose(a, c, atol=1e-12 if dtype == np.complex128 else 1e-5, rtol=0)
    assert torch.allclose(g1, g2, atol=GRAD_TOL[dtype], rtol=0)


def test_batch_jacobian_rot_ring():
    import torch
    import lq_oracle as O
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.workloads import rot_ring_batch, bind, obs_terms
    circuits, params = rot_ring_batch(ncirc=3, n=6, layers=2, seed=4)
    eng = BatchedCircuits(circuits, len(params), dtype=np.complex128, use_graphs=False)
    p = torch.tensor(params, dtype=torch.float64, device="cuda")
    jac = eng.jacobian(p).cpu().numpy()
    off = 0
    for c in circuits:
        ops = bind(c, params)
        obs = [obs_terms(o) for o in c["observables"]]
        npo = sum(1 for q in c["param_index"] if q >= 0)
        want = O.adjoint_jacobian(O.run_circuit(6, ops), ops, obs, list(range(npo)))
        got = jac[off:off + len(obs) * npo].reshape(len(obs), npo)
        assert np.abs(got - want).max() < 1e-12
        off += len(obs) * npo


def test_batch_rejects_bad_input():
    from lightning_b200 import capi
    from lightning_b200.batch import BatchedCircuits
    with pytest.raises(capi.B200Error, match="decomposed"):
        BatchedCircuits([{"num_qubits": 2, "ops": [("Rot", [0], False, [])], "param_index": [0],
                          "observables": [[(1.0, "Z", [0])]]}], 1)
    with pytest.raises(capi.B200Error, match="out of range"):
        BatchedCircuits([{"num_qubits": 2, "ops": [("RX", [0], False, [])], "param_index": [5],
                          "observables": [[(1.0, "Z", [0])]]}], 1)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_batch_vjp_tiled_rot_ring(dtype):
    """The benchmark's circuit family at 16 qubits: wider than a tile, so every circuit runs the
    segmented HBM path with CNOT rings crossing tile bits; forward, VJP (which reuses the forward's
    states) and a second VJP (which must recompute them) against the FP64 oracle."""
    import torch
    import lq_oracle as O
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.autograd import batched_expval
    from lightning_b200.workloads import rot_ring_batch, bind, obs_terms
    circuits, params = rot_ring_batch(ncirc=3, n=16, layers=3, seed=12)
    eng = BatchedCircuits(circuits, len(params), dtype=dtype, use_graphs=True)
    p = torch.tensor(params, dtype=torch.float64, device="cuda", requires_grad=True)
    out = batched_expval(p, eng)
    dy = np.random.default_rng(2).normal(size=out.numel())
    (g,) = torch.autograd.grad(out, p, torch.tensor(dy, device="cuda"))
    g2 = eng.vjp(p.detach(), torch.tensor(dy, device="cuda"))
    want_out, want_g = [], np.zeros(len(params))
    for ci, c in enumerate(circuits):
        ops = bind(c, params)
        obs = [obs_terms(o) for o in c["observables"]]
        psi = O.run_circuit(16, ops)
        want_out += [O.expval(psi, o) for o in obs]
        npo = sum(1 for q in c["param_index"] if q >= 0)
        ham = [[(float(dy[ci * 16 + q]), [("PauliZ", [q])]) for q in range(16)]]
        jac = O.adjoint_jacobian(psi, ops, ham, list(range(npo)))[0]
        slots = [q for q in c["param_index"] if q >= 0]
        want_g[slots] = jac
    tol_out, tol_g = (1e-12, GRAD_TOL[dtype]) if dtype == np.complex128 else (2e-5, GRAD_TOL[dtype])
    assert np.abs(out.detach().cpu().numpy() - want_out).max() < tol_out
    assert np.abs(g.cpu().numpy() - want_g).max() < tol_g
    assert np.abs(g2.cpu().numpy() - want_g).max() < tol_g


def edge_batch(seed=21):
    """Edge shapes: an empty circuit, one-qubit circuits, a circuit without parameters, and
    circuits longer than one staged segment (160 ops) both on-chip (10 qubits) and tiled
    (15 qubits complex64 / 14 complex128)."""
    rng = np.random.default_rng(seed)
    params = []
    circuits = []

    def obs_for(n):
        return [[(1.0, "Z", [0])], [(0.7, "X", [n - 1])]]

    circuits.append({"num_qubits": 2, "ops": [], "param_index": [], "observables": obs_for(2)})
    for name in ("RX", "RY", "PhaseShift"):
        circuits.append({"num_qubits": 1, "ops": [("Hadamard", [0], False, []), (name, [0], True, [])],
                         "param_index": [-1, len(params)], "observables": [[(1.0, "Z", [0])], [(1.0, "Y", [0])]]})
        params.append(float(rng.uniform(0, 6)))
    circuits.append({"num_qubits": 3, "ops": [("Hadamard", [0], False, []), ("CNOT", [0, 2], False, []),
                                              ("S", [2], False, [])], "param_index": [-1, -1, -1],
                     "observables": obs_for(3)})
    for n in (10, 15):
        ops, pidx = [], []
        for layer in range(12):
            for q in range(n):
                for g in ("RZ", "RY", "RZ"):
                    ops.append((g, [q], False, []))
                    pidx.append(len(params))
                    params.append(float(rng.uniform(0, 2 * np.pi)))
            for q in range(n):
                ops.append(("CNOT", [q, (q + 1 + layer % (n - 1)) % n], False, []))
                pidx.append(-1)
        circuits.append({"num_qubits": n, "ops": ops, "param_index": pidx, "observables": obs_for(n)})
    return circuits, np.array(params)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_batch_edge_shapes(dtype):
    import torch
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.autograd import batched_expval
    circuits, params = edge_batch()
    if dtype == np.complex128:
        circuits[-1] = dict(circuits[-1], num_qubits=14,
                            ops=[op for op in circuits[-1]["ops"] if max(op[1]) < 14],
                            param_index=[p for op, p in zip(circuits[-1]["ops"], circuits[-1]["param_index"])
                                         if max(op[1]) < 14],
                            observables=[[(1.0, "Z", [0])], [(0.7, "X", [13])]])
        used = sorted({p for c in circuits for p in c["param_index"] if p >= 0})
        remap = {p: i for i, p in enumerate(used)}
        for c in circuits:
            c["param_index"] = [remap[p] if p >= 0 else -1 for p in c["param_index"]]
        params = params[used]
    assert max(len(c["ops"]) for c in circuits) > 160
    eng = BatchedCircuits(circuits, len(params), dtype=dtype, use_graphs=False)
    p = torch.tensor(params, dtype=torch.float64, device="cuda", requires_grad=True)
    out = batched_expval(p, eng)
    want = oracle_outputs(circuits, params)
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    assert np.abs(out.detach().cpu().numpy() - want).max() < tol
    rng = np.random.default_rng(2)
    dy = rng.normal(size=out.numel())
    (out * torch.tensor(dy, device="cuda")).sum().backward()
    gwant = oracle_vjp(circuits, params, dy)
    assert np.abs(p.grad.cpu().numpy() - gwant).max() < GRAD_TOL[dtype]


def _z_expvals(state, n):
    """<Z_q> for every wire q of an n-qubit state (wire 0 = most significant bit), FP64."""
    p = (np.abs(np.asarray(state, dtype=np.complex128)) ** 2).reshape([2] * n)
    return np.array([p.take(0, axis=q).sum() - p.take(1, axis=q).sum() for q in range(n)])


def test_batch_c64_rot_ring_full_shape_vs_reference_and_fd(ref_module):
    """The batched-adjoint configuration's circuit shape on 4 circuits: 16 qubits, 8 layers of
    Rot (serialised RZ RY RZ) on every qubit plus a CNOT ring of range (l mod 15) + 1,
    384 parameters, PauliZ on every qubit, complex64 with FP64 reductions.

    (a) The full 16 x 384 Jacobian of every circuit against the reference's own
        AdjointJacobianC128 (AdjointJacobianLQubit.hpp:212-335), within 1e-5.
    (b) Central finite differences, h = 1e-4, from FP64 forward passes of the reference's
        StateVectorC128 (the check of tests/test_adjoint_jacobian.py in the reference), on 48
        seeded parameters per circuit (the first three, the last three and 42 in between),
        within 1e-5.
    (c) The dy-weighted VJP through torch.autograd against dy . J_reference, within 1e-5."""
    import torch
    import ref
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.autograd import batched_expval
    from lightning_b200.workloads import rot_ring_batch, bind
    n, layers = 16, 8
    circuits, params = rot_ring_batch(ncirc=4, n=n, layers=layers, seed=31)
    eng = BatchedCircuits(circuits, len(params), dtype=np.complex64, use_graphs=True)
    p = torch.tensor(params, dtype=torch.float64, device="cuda", requires_grad=True)
    jac = eng.jacobian(p.detach()).cpu().numpy()
    rng = np.random.default_rng(77)
    dy = rng.normal(size=eng.total_obs)
    out = batched_expval(p, eng)
    (g,) = torch.autograd.grad(out, p, torch.tensor(dy, device="cuda"))
    g = g.cpu().numpy()
    out = out.detach().cpu().numpy()
    obs = [[(1.0, [("PauliZ", [q])])] for q in range(n)]
    npo = 3 * n * layers
    assert npo == 384
    off = 0
    for ci, c in enumerate(circuits):
        ops = bind(c, params)
        slots = [q for q in c["param_index"] if q >= 0]
        psi = ref.run_circuit(ref_module, n, ops)
        assert np.abs(out[ci * n:(ci + 1) * n] - _z_expvals(psi, n)).max() < 2e-6
        want = ref.adjoint_jacobian(ref_module, psi, ops, obs, list(range(npo)))
        got = jac[off:off + n * npo].reshape(n, npo)
        off += n * npo
        assert np.abs(got - want).max() < 1e-5, ci
        assert np.abs(g[slots] - dy[ci * n:(ci + 1) * n] @ want).max() < 1e-5, ci
        pick = np.concatenate([[0, 1, 2], np.sort(rng.choice(np.arange(3, npo - 3), 42, replace=False)),
                               [npo - 3, npo - 2, npo - 1]])
        h = 1e-4
        for col in pick:
            s = slots[col]
            shifted = []
            for sgn in (1.0, -1.0):
                pp = params.copy()
                pp[s] += sgn * h
                shifted.append(_z_expvals(ref.run_circuit(ref_module, n, bind(c, pp)), n))
            fd = (shifted[0] - shifted[1]) / (2 * h)
            assert np.abs(got[:, col] - fd).max() < 1e-5, (ci, col)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_hea_batch_wide_vs_reference(ref_module, dtype):
    """The batched hardware-efficient ansatz at the configuration's upper widths (16..20 qubits,
    RY RZ layers + CZ ring, 3n-term ZZ/X Hamiltonian with N(0, 1) coefficients): forward values
    against the reference's own StateVectorC128 + Hamiltonian expval (ObservablesLQubit.hpp:156-305,
    MeasurementsLQubit.hpp:248-265), and the VJP against the reference's AdjointJacobianC128."""
    import torch
    import ref
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.autograd import batched_expval
    from lightning_b200.workloads import hea_batch, bind, obs_terms
    circuits, params = hea_batch(ncirc=5, nmin=16, nmax=20, dmin=2, dmax=4, seed=61)
    circuits[0] = hea_batch(ncirc=1, nmin=20, nmax=20, dmin=3, dmax=3, seed=62)[0][0]
    circuits[0]["param_index"] = [p if p < 0 else p % len(params) for p in circuits[0]["param_index"]]
    eng = BatchedCircuits(circuits, len(params), dtype=dtype, use_graphs=True)
    p = torch.tensor(params, dtype=torch.float64, device="cuda", requires_grad=True)
    out = batched_expval(p, eng)
    dy = np.random.default_rng(5).normal(size=out.numel())
    (g,) = torch.autograd.grad(out, p, torch.tensor(dy, device="cuda"))
    out = out.detach().cpu().numpy()
    want_g = np.zeros(len(params))
    for ci, c in enumerate(circuits):
        ops = bind(c, params)
        terms = obs_terms(c["observables"][0])
        psi = ref.run_circuit(ref_module, c["num_qubits"], ops)
        want = ref.expval(ref_module, psi.copy(), terms)
        assert abs(out[ci] - want) < (1e-12 if dtype == np.complex128 else 2e-5) * max(1.0, abs(want)), ci
        pops = [i for i, op in enumerate(ops) if len(op[3]) > 0]
        jac = ref.adjoint_jacobian(ref_module, psi, ops, [terms], list(range(len(pops))))[0]
        for col, i in enumerate(pops):
            want_g[c["param_index"][i]] += dy[ci] * jac[col]
    assert np.abs(g.cpu().numpy() - want_g).max() < GRAD_TOL[dtype]


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_batch_many_observables(dtype):
    """Circuits with more observables than one forward pass accumulates (16): 37 and 5 Pauli sums,
    forward values and the VJP against the oracle."""
    import torch
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.autograd import batched_expval
    circuits, params = hea_batch_small_many_obs()
    eng = BatchedCircuits(circuits, len(params), dtype=dtype, use_graphs=False)
    p = torch.tensor(params, dtype=torch.float64, device="cuda", requires_grad=True)
    out = batched_expval(p, eng)
    assert out.numel() == 37 + 5
    want = oracle_outputs(circuits, params)
    assert np.abs(out.detach().cpu().numpy() - want).max() < (1e-12 if dtype == np.complex128 else 2e-5)
    dy = np.random.default_rng(4).normal(size=out.numel())
    (out * torch.tensor(dy, device="cuda")).sum().backward()
    assert np.abs(p.grad.cpu().numpy() - oracle_vjp(circuits, params, dy)).max() < GRAD_TOL[dtype]


def hea_batch_small_many_obs():
    from lightning_b200.workloads import hea_batch
    circuits, params = hea_batch(ncirc=2, nmin=9, nmax=14, dmin=2, dmax=2, seed=44)
    n0, n1 = circuits[0]["num_qubits"], circuits[1]["num_qubits"]
    obs0 = [[(1.0, "Z", [q])] for q in range(n0)] + [[(0.5, "ZZ", [q, (q + 1) % n0])] for q in range(n0)]
    obs0 += [[(0.3, "X", [q]), (-0.2, "Y", [(q + 2) % n0])] for q in range(37 - len(obs0))]
    circuits[0] = dict(circuits[0], observables=obs0[:37])
    circuits[1] = dict(circuits[1], observables=[[(1.0, "Z", [q])] for q in range(5)])
    return circuits, params
