"""A device object with the surface of lightning.qubit's ``LightningQubit`` whose state
stays on the GPU between calls.

The reference device (pennylane_lightning/lightning_qubit/lightning_qubit.py:153-808,
core/lightning_base.py) keeps its state in a NumPy array and wraps that array in a
fresh ``StateVectorC*`` for every call (``apply_lightning`` :330-369, ``expval`` :401-457,
``generate_samples`` :518-540).  Here one device handle owns the amplitudes in HBM for
the device's lifetime: ``apply`` launches gates on it, measurements read it in place,
``adjoint_jacobian`` and ``vjp`` start from it, and the host sees the amplitudes only
when ``state`` is read.

PennyLane itself is not a dependency.  Operations, observables, measurements and tapes
are small records carrying what the reference's serializer extracts from PennyLane
objects (core/_serialize.py): operation name, wires, parameters, optional matrix;
observables as sums of products of named or Hermitian factors, or a CSR sparse matrix.
Method names, argument meaning, the order of checks and the error messages follow the
reference device.
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import capi

STATE_PREPS = ("QubitStateVector", "StatePrep", "BasisState")


class DeviceError(RuntimeError):
    """Invalid use of the device (pennylane.DeviceError in the reference)."""


class QuantumFunctionError(RuntimeError):
    """Unsupported differentiation request (pennylane.QuantumFunctionError in the reference)."""


# ---- records standing in for PennyLane objects -------------------------------------
@dataclass
class Operation:
    """One gate: a name of the reference's gate set, wire labels, parameters, and a
    matrix for gates without a kernel (applied through ``applyMatrix``)."""
    name: str
    wires: Sequence
    params: Sequence = ()
    matrix: Optional[np.ndarray] = None

    @property
    def num_params(self) -> int:
        return len(self.params)


@dataclass
class Observable:
    """Sum of coefficient x product-of-factors terms; a factor is (name, wires) or
    ("Hermitian", wires, matrix).  ``name`` is the reference observable's name
    ("PauliZ", "Hermitian", "Hamiltonian", "Tensor", "SparseHamiltonian", "Identity",
    "Projector").  A SparseHamiltonian carries ``csr = (indptr, indices, data)`` over the
    device's wire order instead of terms."""
    name: str
    terms: list = field(default_factory=list)
    csr: Optional[tuple] = None

    @property
    def wires(self):
        seen = []
        for _, factors in self.terms:
            for f in factors:
                for w in f[1]:
                    if w not in seen:
                        seen.append(w)
        return seen


def named(name: str, wires) -> Observable:
    wires = list(wires) if isinstance(wires, (list, tuple)) else [wires]
    return Observable(name, [(1.0, [(name, wires)])])


def hermitian(matrix, wires) -> Observable:
    wires = list(wires) if isinstance(wires, (list, tuple)) else [wires]
    return Observable("Hermitian", [(1.0, [("Hermitian", wires, np.asarray(matrix))])])


def tensor(*obs: Observable) -> Observable:
    factors = []
    for o in obs:
        if len(o.terms) != 1 or o.terms[0][0] != 1.0:
            raise ValueError("tensor factors must be single named or Hermitian observables")
        factors += o.terms[0][1]
    return Observable("Tensor", [(1.0, factors)])


def hamiltonian(coeffs, obs: Sequence[Observable]) -> Observable:
    terms = []
    for c, o in zip(coeffs, obs):
        for c2, f in o.terms:
            terms.append((float(c) * c2, f))
    return Observable("Hamiltonian", terms)


def sparse_hamiltonian(matrix) -> Observable:
    """A scipy sparse matrix (any format) over all device wires."""
    m = matrix.tocsr()
    return Observable("SparseHamiltonian", csr=(m.indptr, m.indices, m.data))


@dataclass
class Measurement:
    """("expval" | "var", observable), ("probs", wires), ("sample", None) or ("state", None)."""
    return_type: str
    obs: Optional[Observable] = None
    wires: Optional[Sequence] = None


def expval(obs: Observable) -> Measurement:
    return Measurement("expval", obs)


def var(obs: Observable) -> Measurement:
    return Measurement("var", obs)


def state() -> Measurement:
    return Measurement("state")


def probs(wires=None) -> Measurement:
    return Measurement("probs", wires=wires)


@dataclass
class Tape:
    """Operations, measurements and trainable parameter indices.  Parameters are numbered
    over the operations in order, every parameter of every operation (a Rot has three,
    a state preparation one), as PennyLane numbers tape parameters."""
    operations: List[Operation]
    measurements: List[Measurement] = field(default_factory=list)
    trainable_params: Optional[List[int]] = None

    def __post_init__(self):
        if self.trainable_params is None:
            self.trainable_params = list(range(self.num_params))

    @property
    def num_params(self) -> int:
        return sum(len(op.params) for op in self.operations)

    def get_operation(self, idx: int):
        """(operation, index of the operation, index of the parameter inside it) of the
        idx-th trainable parameter, as QuantumTape.get_operation."""
        p = sorted(self.trainable_params)[idx]
        k = 0
        for i, op in enumerate(self.operations):
            if p < k + len(op.params):
                return op, i, p - k
            k += len(op.params)
        raise IndexError(idx)

    @property
    def observables(self):
        return [m.obs for m in self.measurements]


# ---- the device -------------------------------------------------------------------------
class LightningQubit:
    """lightning.qubit device surface on a B200 state vector (lightning_qubit.py:153-808)."""

    name = "Lightning Qubit B200 plugin"
    short_name = "lightning.qubit"

    def __init__(self, wires, *, c_dtype=np.complex128, shots=None, mcmc=False, kernel_name="Local",
                 num_burnin=100, batch_obs=False, seed=None):
        if c_dtype not in (np.complex64, np.complex128):
            raise TypeError(f"Unsupported complex Type: {c_dtype}")  # lightning_base.py:80-85
        self.wires = list(range(wires)) if isinstance(wires, int) else list(wires)
        self.num_wires = len(self.wires)
        self.wire_map = {w: i for i, w in enumerate(self.wires)}
        self.C_DTYPE = np.dtype(c_dtype)
        self.use_csingle = self.C_DTYPE == np.complex64
        self.shots = shots
        self._batch_obs = batch_obs
        self._seed = seed
        self._draws = 0
        self._mcmc = mcmc
        if self._mcmc:  # lightning_qubit.py:208-221
            if kernel_name not in ["Local", "NonZeroRandom"]:
                raise NotImplementedError(
                    f"The {kernel_name} is not supported and currently "
                    "only 'Local' and 'NonZeroRandom' kernels are supported.")
            if shots is None or num_burnin >= shots:
                raise ValueError("Shots should be greater than num_burnin.")
            self._kernel_name = kernel_name
            self._num_burnin = num_burnin
        self._sv = capi.StateVector(self.num_wires, self.C_DTYPE)  # pre-rotated state
        self._rot = None                                            # rotated copy, when rotations ran
        self.reset()

    # -- helpers --
    def map_wires(self, wires):
        try:
            return [self.wire_map[w] for w in wires]
        except KeyError as e:
            raise DeviceError(f"Did not find some of the wires {tuple(wires)} on device with wires "
                              f"{tuple(self.wires)}.") from e

    def _serialize_ops(self, operations, decompose_rot=False):
        """(name, device wires, inverse, params[, matrix]) records (core/_serialize.py:184-232):
        Rot becomes RZ(phi) RY(theta) RZ(omega) when ``decompose_rot``; gates without a
        kernel go through their matrix."""
        out = []
        for op in operations:
            w = self.map_wires(op.wires)
            if decompose_rot and op.name == "Rot":
                phi, theta, omega = op.params
                out += [("RZ", w, False, [float(phi)]), ("RY", w, False, [float(theta)]),
                        ("RZ", w, False, [float(omega)])]
            elif op.name in capi.GATE_IDS and op.matrix is None:
                out.append((op.name, w, False, [float(p) for p in op.params]))
            else:
                if op.matrix is None:
                    raise DeviceError(f"Gate {op.name} not supported on device {self.short_name}")
                out.append((op.name, w, False, [], np.asarray(op.matrix, dtype=self.C_DTYPE)))
        return out

    def _serialize_obs(self, obs: Observable):
        if obs.name == "SparseHamiltonian":
            raise QuantumFunctionError("SparseHamiltonian is not supported as an adjoint observable")
        terms = []
        for c, factors in obs.terms:
            fs = []
            for f in factors:
                if f[0] == "Hermitian":
                    fs.append(("Hermitian", self.map_wires(f[1]), np.asarray(f[2], dtype=self.C_DTYPE)))
                elif f[0] == "Projector":
                    raise QuantumFunctionError("Adjoint differentiation method does not support the "
                                               "Projector observable")
                else:
                    fs.append((f[0], self.map_wires(f[1])))
            terms.append((float(c), fs))
        return terms

    # -- state --
    def reset(self):
        """|0...0> (lightning_qubit.py:257-264)."""
        self._sv.set_basis_state(0)
        if self._rot is not None:
            self._rot.close()
        self._rot = None

    @property
    def state(self) -> np.ndarray:
        """The pre-rotated state, copied to the host (lightning_qubit.py:283-287)."""
        return self._sv.download()

    def _measured(self) -> capi.StateVector:
        return self._rot if self._rot is not None else self._sv

    def _apply_state_vector(self, vec, device_wires):
        """lightning_qubit.py:294-314 with lightning_base.py:195-226."""
        vec = np.asarray(vec, dtype=self.C_DTYPE).reshape(-1)
        dw = self.map_wires(device_wires)
        if len(dw) == self.num_wires and sorted(dw) == dw:
            if vec.size != 1 << self.num_wires:
                raise ValueError("State vector must have shape (2**wires,) or (batch_size, 2**wires).")
            self._sv.upload(vec)
            return
        full = np.zeros(1 << self.num_wires, dtype=self.C_DTYPE)
        for k in range(1 << len(dw)):
            idx = 0
            for j, w in enumerate(dw):
                if (k >> (len(dw) - 1 - j)) & 1:
                    idx |= 1 << (self.num_wires - 1 - w)
            full[idx] = vec[k]
        self._sv.upload(full)

    def _apply_basis_state(self, bits, wires):
        """lightning_qubit.py:316-328 with lightning_base.py:228-255."""
        bits = np.asarray(bits)
        dw = self.map_wires(wires)
        if not set(bits.tolist()).issubset({0, 1}):
            raise ValueError("BasisState parameter must consist of 0 or 1 integers.")
        if len(bits) != len(dw):
            raise ValueError("BasisState parameter and wires must be of equal length.")
        index = int(sum(int(b) << (self.num_wires - 1 - w) for b, w in zip(bits, dw)))
        self._sv.set_basis_state(index)

    def apply(self, operations: List[Operation], rotations: Optional[List[Operation]] = None, **kwargs):
        """lightning_qubit.py:371-399: an optional state preparation first, then the gates
        on the device state; rotations act on a device-side copy."""
        operations = list(operations)
        if operations:
            if operations[0].name in ("QubitStateVector", "StatePrep"):
                self._apply_state_vector(np.array(operations[0].params[0], copy=True), operations[0].wires)
                del operations[0]
            elif operations[0].name == "BasisState":
                self._apply_basis_state(operations[0].params[0], operations[0].wires)
                del operations[0]
        for op in operations:
            if op.name in STATE_PREPS:
                raise DeviceError(f"Operation {op.name} cannot be used after other "
                                  f"Operations have already been applied on a {self.short_name} device.")
        ops = [op for op in operations if op.name != "Identity"]
        # the fused apply: one pass over the state per run of gates that fit a shared-memory
        # tile on wide states, one launch per gate on narrow ones (same results to rounding)
        if ops:
            self._sv.apply_ops_fused(self._serialize_ops(ops))
        if rotations:
            if self._rot is None:
                self._rot = capi.StateVector(self.num_wires, self.C_DTYPE)
            self._rot.copy_from(self._sv)
            self._rot.apply_ops_fused(self._serialize_ops(rotations))
        else:
            if self._rot is not None:
                self._rot.close()
            self._rot = None

    def execute(self, tape: Tape):
        """reset, apply the tape's operations, evaluate its measurements (one result each)."""
        self.reset()
        self.apply(tape.operations)
        out = []
        for m in tape.measurements:
            if m.return_type == "expval":
                out.append(self.expval(m.obs))
            elif m.return_type == "var":
                out.append(self.var(m.obs))
            elif m.return_type == "probs":
                out.append(self.probability_lightning(self.wires if m.wires is None else m.wires))
            elif m.return_type == "state":
                out.append(self.state)
            elif m.return_type == "sample":
                out.append(self.generate_samples())
            else:
                raise DeviceError(f"Unsupported return type {m.return_type}")
        return out

    # -- measurements --
    def _pauli_rotations(self, obs: Observable):
        """Diagonalising gates of a product of Pauli factors: X -> H, Y -> Z S H."""
        if len(obs.terms) != 1:
            raise DeviceError(f"Finite-shot estimates support products of Pauli observables, not {obs.name}")
        rots, diag = [], []
        for f in obs.terms[0][1]:
            if f[0] not in ("PauliX", "PauliY", "PauliZ", "Identity"):
                raise DeviceError(f"Finite-shot estimates support products of Pauli observables, not {f[0]}")
            if f[0] == "PauliX":
                rots.append(Operation("Hadamard", f[1]))
            elif f[0] == "PauliY":
                rots += [Operation("PauliZ", f[1]), Operation("S", f[1]), Operation("Hadamard", f[1])]
            if f[0] != "Identity":
                diag += list(f[1])
        return rots, diag

    def _eigen_samples(self, obs: Observable):
        rots, diag = self._pauli_rotations(obs)
        saved = self._rot
        self._rot = None
        if rots:
            self.apply([], rotations=rots)
        bits = self.generate_samples()
        if self._rot is not None:
            self._rot.close()
        self._rot = saved
        cols = self.map_wires(diag)
        parity = bits[:, cols].sum(axis=1) % 2 if cols else np.zeros(bits.shape[0], dtype=int)
        return obs.terms[0][0] * (1 - 2 * parity)

    def expval(self, observable: Observable, shot_range=None, bin_size=None):
        """lightning_qubit.py:401-457."""
        if observable.name == "Projector":
            raise DeviceError("Projector observables are not supported by this device")
        if self.shots is not None:
            return float(np.mean(self._eigen_samples(observable)))
        if observable.name == "SparseHamiltonian":
            return self._sv.expval_sparse(*observable.csr)
        if observable.name == "Identity":
            return 1.0
        return self._sv.expval(self._serialize_obs(observable))

    def var(self, observable: Observable, shot_range=None, bin_size=None):
        """lightning_qubit.py:459-516."""
        if observable.name == "Projector":
            raise DeviceError("Projector observables are not supported by this device")
        if self.shots is not None:
            return float(np.var(self._eigen_samples(observable)))
        if observable.name == "SparseHamiltonian":
            return self._sv.var_sparse(*observable.csr)
        if observable.name == "Identity":
            return 0.0
        return self._sv.var(self._serialize_obs(observable))

    def probability_lightning(self, wires):
        """lightning_qubit.py:542-558 (marginal order as MeasurementsLQubit::probs(wires))."""
        return self._measured().probs(self.map_wires(wires))

    def generate_samples(self):
        """(shots, num_wires) array of bits, wire 0 first (lightning_qubit.py:518-540): inverse-CDF
        draws, or Metropolis chains when the device was created with ``mcmc=True``."""
        if self.shots is None:
            raise DeviceError("The number of shots has to be explicitly set on the device "
                              "when using sample-based measurements.")
        if self._seed is None:
            seed = int(np.random.SeedSequence().generate_state(1, dtype=np.uint64)[0])
        else:
            seed = int(self._seed) * 0x10001 + self._draws
        self._draws += 1
        sv = self._measured()
        if self._mcmc:
            return sv.sample_mcmc_bits(self._kernel_name, self._num_burnin, self.shots, seed=seed).astype(int)
        return sv.sample_bits(self.shots, seed=seed).astype(int)

    # -- differentiation --
    @staticmethod
    def _check_adjdiff_supported_measurements(measurements: List[Measurement]):
        """lightning_qubit.py:560-596."""
        if not measurements:
            return None
        if len(measurements) == 1 and measurements[0].return_type == "state":
            return "state"
        if any(m.return_type != "expval" for m in measurements):
            raise QuantumFunctionError("Adjoint differentiation method does not support expectation return type "
                                       "mixed with other return types")
        for m in measurements:
            if m.obs.name == "Projector" or any(f[0] == "Projector" for _, fs in m.obs.terms for f in fs):
                raise QuantumFunctionError("Adjoint differentiation method does not support the Projector "
                                           "observable")
        return "expval"

    @staticmethod
    def _check_adjdiff_supported_operations(operations):
        """lightning_qubit.py:598-612."""
        for op in operations:
            if op.num_params > 1 and op.name != "Rot":
                raise QuantumFunctionError(f"The {op.name} operation is not supported using "
                                           'the "adjoint" differentiation method')

    def _init_process_jacobian_tape(self, tape, starting_state, use_device_state):
        """lightning_qubit.py:614-629: the state the adjoint sweep starts from, on the device."""
        if starting_state is not None:
            starting_state = np.asarray(starting_state)
            if starting_state.size != 2 ** len(self.wires):
                raise QuantumFunctionError("The number of qubits of starting_state must be the same as "
                                           "that of the device.")
            sv = capi.StateVector(self.num_wires, self.C_DTYPE)
            sv.upload(starting_state.reshape(-1))
            return sv
        if not use_device_state:
            self.reset()
            self.apply(tape.operations)
        sv = capi.StateVector(self.num_wires, self.C_DTYPE)
        sv.copy_from(self._sv)
        return sv

    def _process_jacobian_tape(self, tape, starting_state, use_device_state):
        """lightning_base.py:257-304: serialized operations without state preparations, the
        trainable parameters shifted past a leading state preparation, and the rows of the
        full Jacobian they fill."""
        sv = self._init_process_jacobian_tape(tape, starting_state, use_device_state)
        use_sp = any(op.name in STATE_PREPS for op in tape.operations)
        ops = self._serialize_ops([op for op in tape.operations if op.name not in STATE_PREPS],
                                  decompose_rot=True)
        trainable = sorted(tape.trainable_params)
        if not trainable:
            sv.close()
            return None
        tp_shift, record_tp_rows, all_params = [], [], 0
        for op_idx, p in enumerate(trainable):
            op, _, _ = tape.get_operation(op_idx)
            if op.name not in STATE_PREPS:
                tp_shift.append(p)
                record_tp_rows.append(all_params)
            all_params += 1
        if use_sp:
            tp_shift = [i - 1 for i in tp_shift]
        return {"state_vector": sv, "ops_serialized": ops, "tp_shift": tp_shift,
                "record_tp_rows": record_tp_rows, "all_params": all_params}

    def adjoint_jacobian(self, tape: Tape, starting_state=None, use_device_state=False):
        """lightning_qubit.py:631-692: Jacobian [observable][trainable parameter]."""
        if self.shots is not None:
            warnings.warn("Requested adjoint differentiation to be computed with finite shots. "
                          "The derivative is always exact when using the adjoint "
                          "differentiation method.", UserWarning)
        rtype = self._check_adjdiff_supported_measurements(tape.measurements)
        if not rtype:
            return np.array([], dtype=self.C_DTYPE)
        if rtype == "state":
            raise QuantumFunctionError("This method does not support statevector return type. "
                                       "Use vjp method instead for this purpose.")
        self._check_adjdiff_supported_operations(tape.operations)
        obs = [self._serialize_obs(o) for o in tape.observables]
        data = self._process_jacobian_tape(tape, starting_state, use_device_state)
        if not data:
            return np.array([], dtype=self.C_DTYPE)
        try:
            jac = data["state_vector"].adjoint_jacobian(data["ops_serialized"], obs, data["tp_shift"])
        finally:
            data["state_vector"].close()
        jac = np.asarray(jac).reshape(-1, len(data["tp_shift"]))
        jac_r = np.zeros((jac.shape[0], data["all_params"]))
        jac_r[:, data["record_tp_rows"]] = jac
        return jac_r

    def vjp(self, measurements: List[Measurement], grad_vec, starting_state=None,
            use_device_state=False) -> Callable[[Tape], np.ndarray]:
        """lightning_qubit.py:694-808: a function of a tape returning the vector-Jacobian
        product, through one Hamiltonian adjoint pass for expectation values or through
        VectorJacobianProduct for a state return."""
        if self.shots is not None:
            warnings.warn("Requested adjoint differentiation to be computed with finite shots. "
                          "The derivative is always exact when using the adjoint differentiation "
                          "method.", UserWarning)
        rtype = self._check_adjdiff_supported_measurements(measurements)
        grad_vec = np.asarray(grad_vec)
        if np.allclose(grad_vec, 0) or rtype is None:
            return lambda tape: np.zeros(len(tape.trainable_params))
        if rtype == "expval":
            if len(grad_vec) != len(measurements):
                raise ValueError("Number of observables in the tape must be the same as the "
                                 "length of grad_vec in the vjp method")
            if np.iscomplexobj(grad_vec):
                raise ValueError("The vjp method only works with a real-valued grad_vec when the "
                                 "tape is returning an expectation value")
            ham = hamiltonian(grad_vec, [m.obs for m in measurements])

            def processing_fn_expval(tape):
                if len(tape.trainable_params) == 0:
                    return np.array([], dtype=self.C_DTYPE)
                new_tape = Tape(tape.operations, [expval(ham)], list(tape.trainable_params))
                return self.adjoint_jacobian(new_tape, starting_state, use_device_state)
            return processing_fn_expval

        if len(grad_vec) != 2 ** len(self.wires):
            raise ValueError("Size of the provided vector grad_vec must be the same as "
                             "the size of the statevector")
        if np.isrealobj(grad_vec):
            warnings.warn("The vjp method only works with complex-valued grad_vec when "
                          "the tape is returning a statevector. Upcasting grad_vec.")
        gv = grad_vec.astype(self.C_DTYPE)

        def processing_fn_state(tape):
            data = self._process_jacobian_tape(tape, starting_state, use_device_state)
            if not data:
                return np.array([], dtype=self.C_DTYPE)
            try:
                return data["state_vector"].vjp_state(data["ops_serialized"], gv, data["tp_shift"])
            finally:
                data["state_vector"].close()
        return processing_fn_state
