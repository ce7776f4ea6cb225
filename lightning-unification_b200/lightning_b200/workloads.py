"""Seeded synthetic circuit families used by the benchmark and the tests.

Every generator returns plain Python data (op tuples ``(name, wires, inverse,
params)``), so the same circuits can be fed to this engine and to the
reference.  ``Rot`` is serialised as RZ(phi), RY(theta), RZ(omega) exactly as
the reference's Python layer does before adjoint differentiation
(pennylane_lightning/core/_serialize.py:212-213).
"""
from __future__ import annotations

import numpy as np


def layered_rotations(n: int = 20, layers: int = 10, seed: int = 1234):
    """n qubits, `layers` x (RX, RY, RZ on every qubit, then a CNOT ladder q -> q+1).

    Returns (ops, observables, trainable): <Z0> and all 3*n*layers parameters."""
    rng = np.random.default_rng(seed)
    ops = []
    for _ in range(layers):
        for q in range(n):
            for g in ("RX", "RY", "RZ"):
                ops.append((g, [q], False, [float(rng.uniform(0, 2 * np.pi))]))
        for q in range(n - 1):
            ops.append(("CNOT", [q, q + 1], False, []))
    obs = [[(1.0, [("PauliZ", [0])])]]
    return ops, obs, list(range(3 * n * layers))


def random_unitary(rng, k: int) -> np.ndarray:
    """QR of a complex Gaussian matrix with the phases of R's diagonal removed (Haar)."""
    d = 1 << k
    z = (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    ph = np.diag(r) / np.abs(np.diag(r))
    return q * ph


SWEEP_KINDS = ("Hadamard", "RX", "RY", "RZ", "CNOT", "CZ", "SWAP", "Toffoli", "U2", "U3")


def gate_sweep(n: int, ngates: int = 200, seed: int = 7):
    """`ngates` gates drawn uniformly from SWEEP_KINDS on uniformly drawn distinct wires."""
    rng = np.random.default_rng(seed)
    ops = []
    for _ in range(ngates):
        kind = SWEEP_KINDS[rng.integers(len(SWEEP_KINDS))]
        nw = {"CNOT": 2, "CZ": 2, "SWAP": 2, "Toffoli": 3, "U2": 2, "U3": 3}.get(kind, 1)
        wires = [int(w) for w in rng.choice(n, nw, replace=False)]
        if kind in ("U2", "U3"):
            ops.append(("QubitUnitary", wires, False, [], random_unitary(rng, nw)))
        elif kind in ("RX", "RY", "RZ"):
            ops.append((kind, wires, False, [float(rng.uniform(0, 2 * np.pi))]))
        else:
            ops.append((kind, wires, False, []))
    return ops


def random_state(n: int, seed: int = 3, dtype=np.complex128) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = rng.uniform(-1, 1, size=1 << n) + 1j * rng.uniform(-1, 1, size=1 << n)
    s /= np.linalg.norm(s)
    return s.astype(dtype)


def hea_batch(ncirc: int = 4096, nmin: int = 10, nmax: int = 20, dmin: int = 4, dmax: int = 16, seed: int = 11):
    """Hardware-efficient ansatz batch: per circuit n ~ U[nmin, nmax], depth ~ U[dmin, dmax];
    each layer RY, RZ on every qubit then a CZ ring; observable: 3n-term Hamiltonian of
    Z_i Z_{i+1}, Z_i Z_{i+2} and X_i with N(0,1) coefficients.  Parameters are
    numbered consecutively over the whole batch."""
    rng = np.random.default_rng(seed)
    circuits, params = [], []
    for _ in range(ncirc):
        n = int(rng.integers(nmin, nmax + 1))
        d = int(rng.integers(dmin, dmax + 1))
        ops, pidx = [], []
        for _ in range(d):
            for q in range(n):
                for g in ("RY", "RZ"):
                    ops.append((g, [q], False, []))
                    pidx.append(len(params))
                    params.append(float(rng.uniform(0, 2 * np.pi)))
            for q in range(n):
                ops.append(("CZ", [q, (q + 1) % n], False, []))
                pidx.append(-1)
        terms = []
        for q in range(n):
            terms.append((float(rng.normal()), "ZZ", [q, (q + 1) % n]))
        for q in range(n):
            terms.append((float(rng.normal()), "ZZ", [q, (q + 2) % n]))
        for q in range(n):
            terms.append((float(rng.normal()), "X", [q]))
        circuits.append({"num_qubits": n, "ops": ops, "param_index": pidx, "observables": [terms]})
    return circuits, np.array(params)


def rot_ring_batch(ncirc: int = 1024, n: int = 16, layers: int = 8, seed: int = 5):
    """Batched-adjoint workload: per layer a general Rot(phi, theta, omega) on every qubit,
    serialised as RZ(phi) RY(theta) RZ(omega), then CNOT(q, (q + r_l) mod n) with
    r_l = (l mod (n-1)) + 1; observables Z_q on every qubit.  3*n*layers parameters per
    circuit, uniform in [0, 2*pi)."""
    rng = np.random.default_rng(seed)
    circuits, params = [], []
    for _ in range(ncirc):
        ops, pidx = [], []
        for l in range(layers):
            for q in range(n):
                for g in ("RZ", "RY", "RZ"):
                    ops.append((g, [q], False, []))
                    pidx.append(len(params))
                    params.append(float(rng.uniform(0, 2 * np.pi)))
            r = (l % (n - 1)) + 1
            for q in range(n):
                ops.append(("CNOT", [q, (q + r) % n], False, []))
                pidx.append(-1)
        obs = [[(1.0, "Z", [q])] for q in range(n)]
        circuits.append({"num_qubits": n, "ops": ops, "param_index": pidx, "observables": obs})
    return circuits, np.array(params)


def jordan_wigner_words(rng, n: int, count: int):
    """Pauli words shaped like Jordan-Wigner fermion terms: X/Y on 1, 2 or 4 wires with Z
    strings between the paired wires, as ("XZZY", [wires]) in ascending wire order."""
    words = []
    for _ in range(count):
        k = int(rng.choice([1, 2, 2, 4]))
        ws = sorted(int(w) for w in rng.choice(n, k, replace=False))
        letters = {w: "XY"[int(rng.integers(2))] for w in ws}
        for lo, hi in zip(ws[0::2], ws[1::2]):
            for w in range(lo + 1, hi):
                letters[w] = "Z"
        wires = sorted(letters)
        words.append(("".join(letters[w] for w in wires), wires))
    return words


def bind(circuit, params):
    """Materialise a batch circuit's op list with concrete parameter values."""
    out = []
    for op, pi in zip(circuit["ops"], circuit["param_index"]):
        name, wires, inv, p = op[:4]
        out.append((name, wires, inv, [float(params[pi])] if pi >= 0 else list(p)) + tuple(op[4:]))
    return out


def obs_terms(observable):
    """Batch observable [(coeff, 'ZZ', wires)] -> oracle terms [(coeff, [(name, [w])...])]."""
    names = {"X": "PauliX", "Y": "PauliY", "Z": "PauliZ", "I": "Identity"}
    return [(c, [(names[ch], [w]) for ch, w in zip(word, wires)]) for c, word, wires in observable]


def qft_circuit(n: int, seed: int = 9):
    """RY(theta_q) on every qubit, then for j: H(j) and ControlledPhaseShift(2*pi/2^(k-j+1)) on (k, j), k > j."""
    rng = np.random.default_rng(seed)
    ops = [("RY", [q], False, [float(rng.uniform(0, 2 * np.pi))]) for q in range(n)]
    for j in range(n):
        ops.append(("Hadamard", [j], False, []))
        for k in range(j + 1, n):
            ops.append(("ControlledPhaseShift", [k, j], False, [2 * np.pi / 2 ** (k - j + 1)]))
    return ops
