"""Generate golden fixtures from the reference itself.

Runs the reference's lightning_qubit_ops (compiled from its own sources into
oracle/_ref by oracle/Makefile) on seeded inputs and stores the outputs in
tests/golden/reference_outputs.npz:

  * every gate, both directions, on a seeded random 5-qubit state (complex128
    and complex64);
  * probabilities, expectation values and variances of Named, TensorProd,
    Hermitian and Hamiltonian observables on a seeded 6-qubit state;
  * adjoint Jacobians of two seeded circuits.

The tests compare the NumPy oracle and the B200 engine against these arrays,
so parity is pinned even where the reference cannot be built.

Usage: python tests/golden/make_golden.py   (needs oracle/_ref; run make -C oracle)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT / "oracle"), str(ROOT / "lightning-unification_b200")]

GATES = {"Identity": (1, 0), "PauliX": (1, 0), "PauliY": (1, 0), "PauliZ": (1, 0), "Hadamard": (1, 0),
         "S": (1, 0), "T": (1, 0), "PhaseShift": (1, 1), "RX": (1, 1), "RY": (1, 1), "RZ": (1, 1),
         "Rot": (1, 3), "CNOT": (2, 0), "CY": (2, 0), "CZ": (2, 0), "SWAP": (2, 0), "IsingXX": (2, 1),
         "IsingXY": (2, 1), "IsingYY": (2, 1), "IsingZZ": (2, 1), "ControlledPhaseShift": (2, 1),
         "CRX": (2, 1), "CRY": (2, 1), "CRZ": (2, 1), "CRot": (2, 3), "SingleExcitation": (2, 1),
         "SingleExcitationMinus": (2, 1), "SingleExcitationPlus": (2, 1), "Toffoli": (3, 0),
         "CSWAP": (3, 0), "DoubleExcitation": (4, 1), "DoubleExcitationMinus": (4, 1),
         "DoubleExcitationPlus": (4, 1), "MultiRZ": (3, 1)}


def gate_cases(seed=2024, n=5):
    rng = np.random.default_rng(seed)
    st = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    st /= np.linalg.norm(st)
    cases = []
    for name, (k, p) in GATES.items():
        for inv in (False, True):
            wires = [int(w) for w in rng.choice(n, k, replace=False)]
            params = [float(x) for x in rng.uniform(0, 2 * np.pi, p)]
            cases.append((name, wires, inv, params))
    return st, cases


def obs_cases():
    herm = np.array([[1.0, 0.5 - 0.25j], [0.5 + 0.25j, -0.3]])
    return {
        "z3": [(1.0, [("PauliZ", [3])])],
        "h5": [(1.0, [("Hadamard", [5])])],
        "xzy": [(1.0, [("PauliX", [0]), ("PauliZ", [2]), ("PauliY", [4])])],
        "herm": [(1.0, [("Hermitian", [1], herm)])],
        "ham": [(0.4, [("PauliX", [1]), ("PauliX", [2])]), (-1.3, [("PauliZ", [0])]),
                (0.7, [("Hermitian", [5], herm)])],
    }


def adjoint_cases():
    from lightning_b200.workloads import layered_rotations
    ops1, obs1, tp1 = layered_rotations(n=5, layers=2, seed=77)
    ops2 = [("RX", [0], False, [0.3]), ("CNOT", [0, 1], False, []), ("IsingXY", [1, 2], False, [0.8]),
            ("CRY", [2, 0], True, [1.1]), ("RZ", [1], False, [-0.4]), ("SingleExcitation", [0, 2], False, [0.6]),
            ("MultiRZ", [0, 1, 2], False, [0.25]), ("PhaseShift", [2], True, [1.7])]
    obs2 = [[(1.0, [("PauliZ", [0])])], [(0.5, [("PauliX", [1]), ("PauliY", [2])]), (0.2, [("PauliZ", [2])])]]
    return [(5, ops1, obs1, tp1), (3, ops2, obs2, [0, 1, 3, 4, 5, 6])]


def main():
    import lq_oracle as O
    import ref
    m = ref.load()
    if m is None:
        sys.exit("oracle/_ref is not built: run make -C oracle first")
    out = {}
    meta = {"gates": [], "obs": list(obs_cases().keys())}
    st, cases = gate_cases()
    out["gate_input"] = st
    for i, (name, wires, inv, params) in enumerate(cases):
        meta["gates"].append([name, wires, inv, params])
        out[f"gate{i}_c128"] = ref.run_circuit(m, 5, [(name, wires, inv, params)], np.complex128, state=st)
        out[f"gate{i}_c64"] = ref.run_circuit(m, 5, [(name, wires, inv, params)], np.complex64,
                                              state=st.astype(np.complex64))
    rng = np.random.default_rng(99)
    s6 = rng.normal(size=64) + 1j * rng.normal(size=64)
    s6 /= np.linalg.norm(s6)
    out["meas_input"] = s6
    out["probs_all"] = ref.probs(m, s6)
    out["probs_413"] = ref.probs(m, s6, [4, 1, 3])
    for k, terms in obs_cases().items():
        out[f"ev_{k}"] = np.array(ref.expval(m, s6, terms))
        out[f"var_{k}"] = np.array(ref.var(m, s6, terms))
    for j, (n, ops, obs, tp) in enumerate(adjoint_cases()):
        final = O.run_circuit(n, ops)
        out[f"adj{j}"] = ref.adjoint_jacobian(m, final.copy(), ops, obs, tp)
    np.savez_compressed(HERE / "reference_outputs.npz", **out)
    (HERE / "reference_outputs.json").write_text(json.dumps(meta))
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
