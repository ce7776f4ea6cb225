"""The C++ host API as a C++ caller uses it: tests/cpp/host_api_check.cpp is compiled with
g++ against include/ and csrc/host/, linked to libb200sv.so, run, and its printed results are
checked against the FP64 oracle (complex128, 1e-12) and the reference's known values
(Test_AdjointJacobian.cpp:123-176: d<Z>/dp of RX(p) = -sin p)."""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "lightning-unification_b200"

OPS = [("Hadamard", [0], False, []), ("RX", [1], False, [0.3]), ("CNOT", [0, 2], False, []),
       ("RY", [2], True, [0.7]), ("CRZ", [1, 0], False, [-1.1])]
HAM = [(0.5, [("PauliZ", [0]), ("PauliX", [2])]), (-1.25, [("PauliY", [1])])]
ZX = [(1.0, [("PauliZ", [0]), ("PauliX", [2])])]


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    from lightning_b200 import capi
    capi.lib()  # the library is built and loads
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("host") / "host_api_check"
    libdir = PKG / "lightning_b200"
    cmd = [gxx, "-std=c++20", "-O1", f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc' / 'host'}",
           str(ROOT / "tests" / "cpp" / "host_api_check.cpp"), f"-L{libdir}", "-lb200sv",
           f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=300).stdout
    return {d["label"]: d for d in (json.loads(line) for line in out.splitlines() if line.strip())}


def state_of(r):
    return np.array(r["re"]) + 1j * np.array(r["im"])


def test_gates_matrix_generator(results):
    import lq_oracle as O
    psi = O.run_circuit(3, OPS)
    assert np.abs(state_of(results["after_ops"]) - psi).max() < 1e-12
    u = np.array([[0.6, 0.8j], [0.8j, 0.6]])
    psi = O.apply_matrix(psi, u, [1])
    assert np.abs(state_of(results["after_matrix"]) - psi).max() < 1e-12
    g, scale = O.apply_generator(psi, "RX", [2])
    assert results["generator_scale"]["values"][0] == scale
    assert np.abs(state_of(results["after_generator"]) - g).max() < 1e-12


def test_measurements(results):
    import lq_oracle as O
    psi = O.apply_matrix(O.run_circuit(3, OPS), np.array([[0.6, 0.8j], [0.8j, 0.6]]), [1])
    assert np.abs(np.array(results["probs"]["values"]) - O.probs(psi)).max() < 1e-12
    assert np.abs(np.array(results["probs_20"]["values"]) - O.probs(psi, [2, 0])).max() < 1e-12
    assert abs(results["expval_z1"]["values"][0] - O.expval(psi, [(1.0, [("PauliZ", [1])])])) < 1e-12
    assert abs(results["var_x0"]["values"][0] - O.var(psi, [(1.0, [("PauliX", [0])])])) < 1e-12
    assert abs(results["expval_ham"]["values"][0] - O.expval(psi, HAM)) < 1e-12
    assert abs(results["var_ham"]["values"][0] - O.var(psi, HAM)) < 1e-12


def test_apply_in_place(results):
    import lq_oracle as O
    psi = O.apply_matrix(O.run_circuit(3, OPS), np.array([[0.6, 0.8j], [0.8j, 0.6]]), [1])
    assert np.abs(state_of(results["ham_applied"]) - O.apply_observable(psi, HAM)).max() < 1e-12
    assert np.abs(state_of(results["zx_applied"]) - O.apply_observable(psi, ZX)).max() < 1e-12


def test_adjoint(results):
    import lq_oracle as O
    got = np.array(results["adjoint_rx_z"]["values"])
    assert np.abs(got + np.sin([-1.2, 0.4, 2.5])).max() < 1e-12
    psi = O.run_circuit(3, OPS)
    want = O.adjoint_jacobian(psi, OPS, [HAM, [(1.0, [("PauliZ", [0])])]], [0, 1, 2])
    assert np.abs(np.array(results["adjoint_circuit"]["values"]) - np.asarray(want).reshape(-1)).max() < 1e-12


def test_error_message(results):
    assert "Cannot find a registered kernel for a given gate: NotAGate" in results["unknown_gate_message"]["text"]
