"""CPU-side checks of the boundary: the C-ABI library loads and exports every
entry point include/b200sv.h declares, the pybind11 module carries the
reference's Python surface, gate tables agree with the reference enum order,
and host-side helpers (operation packing, workloads) behave.  No compute call
needs a GPU here; without one the library must refuse cleanly instead of
falling back to the CPU."""
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared():
    text = (ROOT / "include" / "b200sv.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b200sv_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes
    lib = ctypes.CDLL(str(ROOT / "lightning-unification_b200" / "lightning_b200" / "libb200sv.so"))
    names = declared()
    assert len(names) >= 37
    for n in names:
        assert hasattr(lib, n), n
    from lightning_b200 import capi
    assert sorted(capi.declared_symbols()) == names


def test_gate_ids_follow_reference_enum():
    """CS/gates/GateOperation.hpp:27-70: ids in declaration order."""
    from lightning_b200 import capi
    expected = ["Identity", "PauliX", "PauliY", "PauliZ", "Hadamard", "S", "T", "PhaseShift", "RX", "RY", "RZ",
                "Rot", "CNOT", "CY", "CZ", "SWAP", "IsingXX", "IsingXY", "IsingYY", "IsingZZ",
                "ControlledPhaseShift", "CRX", "CRY", "CRZ", "CRot", "SingleExcitation", "SingleExcitationMinus",
                "SingleExcitationPlus", "Toffoli", "CSWAP", "DoubleExcitation", "DoubleExcitationMinus",
                "DoubleExcitationPlus", "MultiRZ"]
    assert [capi.GATE_NAMES[i] for i in range(len(expected))] == expected
    hdr = (ROOT / "include" / "b200sv.h").read_text()
    body = hdr[hdr.index("enum b200sv_gate {"):hdr.index("B200SV_GATE_END")]
    hdr_names = [x.replace("B200SV_", "") for x in re.findall(r"B200SV_(\w+)", body)]
    assert hdr_names == expected


def test_module_surface_matches_reference_names():
    import lightning_b200.lightning_qubit_ops as m
    for name in ("StateVectorC64", "StateVectorC128", "MeasurementsC64", "MeasurementsC128", "compile_info",
                 "runtime_info", "backend_info", "allocate_aligned_array", "get_alignment", "best_alignment"):
        assert hasattr(m, name), name
    for name in ("NamedObsC64", "NamedObsC128", "HermitianObsC128", "TensorProdObsC128", "HamiltonianC128"):
        assert hasattr(m.observables, name), name
    for name in ("AdjointJacobianC64", "AdjointJacobianC128", "create_ops_listC64", "create_ops_listC128",
                 "OpsStructC128"):
        assert hasattr(m.algorithms, name), name
    from lightning_b200 import capi
    for g in capi.GATE_IDS:
        assert hasattr(m.StateVectorC128, g), g


def test_same_names_as_built_reference(ref_module):
    import lightning_b200.lightning_qubit_ops as ours
    ours_names = {n for n in dir(ours) if not n.startswith("_")}
    ref_names = {n for n in dir(ref_module) if not n.startswith("_")}
    assert ref_names <= ours_names
    ref_sv = {n for n in dir(ref_module.StateVectorC128) if not n.startswith("_")}
    ours_sv = {n for n in dir(ours.StateVectorC128) if not n.startswith("_")}
    assert ref_sv <= ours_sv
    missing_alg = {n for n in dir(ref_module.algorithms) if not n.startswith("_")} - \
        {n for n in dir(ours.algorithms) if not n.startswith("_")}
    assert not missing_alg


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lightning_b200 import capi
    assert capi.device_count() == 0
    with pytest.raises(capi.B200Error, match="no CUDA device"):
        capi.StateVector(3)
    import lightning_b200.lightning_qubit_ops as m
    with pytest.raises(Exception, match="no CUDA device"):
        m.StateVectorC128(np.zeros(8, np.complex128))


def test_device_shim_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lightning_b200 import capi, device
    with pytest.raises(capi.B200Error, match="no CUDA device"):
        device.LightningQubit(3)
    with pytest.raises(NotImplementedError, match="only 'Local' and 'NonZeroRandom'"):
        device.LightningQubit(3, shots=1000, mcmc=True, kernel_name="Global")
    with pytest.raises(ValueError, match="Shots should be greater than num_burnin"):
        device.LightningQubit(3, shots=10, mcmc=True, num_burnin=100)
    tape = device.Tape([device.Operation("RX", [0], [0.1]), device.Operation("Rot", [1], [1, 2, 3]),
                        device.Operation("CNOT", [0, 1])], trainable_params=[3, 1])
    assert tape.num_params == 4
    assert tape.get_operation(0)[0].name == "Rot" and tape.get_operation(0)[2] == 0
    assert tape.get_operation(1)[0].name == "Rot" and tape.get_operation(1)[2] == 2


def test_oplist_packing():
    from lightning_b200 import capi
    ops = [("RX", [0], False, [0.5]), ("CNOT", [1, 2], True, []),
           ("QubitUnitary", [0, 1], False, [], np.eye(4)), ("BasisState", [0], False, [])]
    ol = capi.OpList(ops)
    assert ol.n == 4
    assert ol.arr[0].gate == capi.GATE_IDS["RX"] and ol.arr[0].nparams == 1 and ol.arr[0].params[0] == 0.5
    assert ol.arr[1].inverse == 1 and list(ol.arr[1].wires[i] for i in range(2)) == [1, 2]
    assert ol.arr[2].gate == capi.OP_MATRIX and ol.arr[2].matrix
    assert ol.arr[3].gate == capi.OP_SKIP


def test_workload_shapes():
    from lightning_b200.workloads import rot_ring_batch, hea_batch, layered_rotations, gate_sweep, qft_circuit
    circuits, params = rot_ring_batch(ncirc=4, n=16, layers=8, seed=5)
    assert len(params) == 4 * 384
    assert all(sum(1 for p in c["param_index"] if p >= 0) == 384 for c in circuits)
    assert all(len(c["observables"]) == 16 for c in circuits)
    # CNOT ring range (l mod 15) + 1
    c0 = circuits[0]["ops"]
    cn = [op for op in c0 if op[0] == "CNOT"]
    assert cn[0][1] == [0, 1] and cn[16][1] == [0, 2] and cn[16 * 7][1] == [0, 8]
    ops, obs, tp = layered_rotations()
    assert len(ops) == 790 and len(tp) == 600
    hc, hp = hea_batch(ncirc=50, seed=1)
    for c in hc:
        n = c["num_qubits"]
        assert 10 <= n <= 20 and len(c["observables"][0]) == 3 * n
    assert len(gate_sweep(10, 200)) == 200
    assert len(qft_circuit(6)) == 6 + 6 + 15
