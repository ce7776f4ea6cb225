"""ctypes view of the C ABI in include/b200sv.h (libb200sv.so).

This is the Python binding a maintainer would add on the reference side for the
batched and autograd paths; the lightning.qubit class surface itself is the
pybind11 module ``lightning_qubit_ops``.  Loading fails loudly when the shared
library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "libb200sv.so"

B200SV_OK = 0
B200SV_C64 = 0
B200SV_C128 = 1
OP_MATRIX = 1000
OP_SKIP = 1001
FACTOR_NAMED = 0
FACTOR_MATRIX = 1

# CS/gates/GateOperation.hpp:27-70 (the enum values of the reference)
GATE_IDS = {
    name: i for i, name in enumerate([
        "Identity", "PauliX", "PauliY", "PauliZ", "Hadamard", "S", "T", "PhaseShift", "RX", "RY", "RZ",
        "Rot", "CNOT", "CY", "CZ", "SWAP", "IsingXX", "IsingXY", "IsingYY", "IsingZZ",
        "ControlledPhaseShift", "CRX", "CRY", "CRZ", "CRot", "SingleExcitation", "SingleExcitationMinus",
        "SingleExcitationPlus", "Toffoli", "CSWAP", "DoubleExcitation", "DoubleExcitationMinus",
        "DoubleExcitationPlus", "MultiRZ"])
}
GATE_NAMES = {v: k for k, v in GATE_IDS.items()}
# CS/gates/GateOperation.hpp:75-98
GENERATOR_IDS = {
    name: i for i, name in enumerate([
        "PhaseShift", "RX", "RY", "RZ", "IsingXX", "IsingXY", "IsingYY", "IsingZZ", "CRX", "CRY", "CRZ",
        "ControlledPhaseShift", "SingleExcitation", "SingleExcitationMinus", "SingleExcitationPlus",
        "DoubleExcitation", "DoubleExcitationMinus", "DoubleExcitationPlus", "MultiRZ"])
}


MCMC_LOCAL, MCMC_NONZERO = 0, 1


def mcmc_proposal_for_name(kernel_name: str) -> int:
    """The proposal the reference runs for a transition-kernel name: generate_samples_metropolis
    (LQ/measurements/MeasurementsLQubit.hpp:387-400) maps "NonZeroRandom" to
    TransitionKernelType::NonZeroRandom and every other name to ::Local, and kernel_factory
    (TransitionKernels.hpp:147-159) builds the non-zero kernel for ::Local and the local
    kernel for ::NonZeroRandom."""
    return MCMC_LOCAL if kernel_name == "NonZeroRandom" else MCMC_NONZERO


class B200Error(RuntimeError):
    """Raised when a libb200sv call returns a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class Op(C.Structure):
    _fields_ = [("gate", C.c_uint32), ("nwires", C.c_uint32), ("wires", C.POINTER(C.c_uint32)),
                ("inverse", C.c_int32), ("nparams", C.c_uint32), ("params", C.POINTER(C.c_double)),
                ("matrix", C.c_void_p)]


class Factor(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("gate", C.c_uint32), ("nwires", C.c_uint32),
                ("wires", C.POINTER(C.c_uint32)), ("matrix", C.c_void_p)]


class Term(C.Structure):
    _fields_ = [("coeff", C.c_double), ("nfactors", C.c_uint32), ("factors", C.POINTER(Factor))]


class Observable(C.Structure):
    _fields_ = [("nterms", C.c_uint32), ("terms", C.POINTER(Term))]


# numpy view of b200sv_op (same layout as the ctypes structure above)
_OP_DTYPE = np.dtype({"names": ["gate", "nwires", "wires", "inverse", "nparams", "params", "matrix"],
                      "formats": ["<u4", "<u4", "<u8", "<i4", "<u4", "<u8", "<u8"],
                      "offsets": [0, 4, 8, 16, 20, 24, 32], "itemsize": 40})
assert C.sizeof(Op) == 40 and Op.wires.offset == 8 and Op.params.offset == 24 and Op.matrix.offset == 32


class BatchCircuit(C.Structure):
    _fields_ = [("num_qubits", C.c_uint32), ("nops", C.c_uint32), ("ops", C.POINTER(Op)),
                ("param_index", C.POINTER(C.c_int64)), ("nobs", C.c_uint32),
                ("obs_nterms", C.POINTER(C.c_uint32)), ("obs_coeffs", C.POINTER(C.c_double)),
                ("obs_offsets", C.POINTER(C.c_uint32)), ("obs_wires", C.POINTER(C.c_uint32)),
                ("obs_paulis", C.c_char_p)]


_SIGS = {
    "b200sv_last_error": ([], C.c_char_p),
    "b200sv_version": ([], C.c_int),
    "b200sv_device_count": ([C.POINTER(C.c_int)], C.c_int),
    "b200sv_create": ([C.c_uint32, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "b200sv_destroy": ([C.c_void_p], C.c_int),
    "b200sv_num_qubits": ([C.c_void_p, C.POINTER(C.c_uint32)], C.c_int),
    "b200sv_dtype": ([C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "b200sv_set_stream": ([C.c_void_p, C.c_void_p], C.c_int),
    "b200sv_synchronize": ([C.c_void_p], C.c_int),
    "b200sv_device_ptr": ([C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "b200sv_upload": ([C.c_void_p, C.c_void_p, C.c_uint64], C.c_int),
    "b200sv_download": ([C.c_void_p, C.c_void_p, C.c_uint64], C.c_int),
    "b200sv_copy": ([C.c_void_p, C.c_void_p], C.c_int),
    "b200sv_set_basis_state": ([C.c_void_p, C.c_uint64], C.c_int),
    "b200sv_apply_gate": ([C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32, C.c_int,
                           C.POINTER(C.c_double), C.c_uint32], C.c_int),
    "b200sv_apply_matrix": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32, C.c_int], C.c_int),
    "b200sv_apply_ops": ([C.c_void_p, C.POINTER(Op), C.c_uint32], C.c_int),
    "b200sv_apply_ops_fused": ([C.c_void_p, C.POINTER(Op), C.c_uint32], C.c_int),
    "b200sv_apply_generator": ([C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32, C.c_int,
                                C.POINTER(C.c_double)], C.c_int),
    "b200sv_probs": ([C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(C.c_double)], C.c_int),
    "b200sv_probs_device": ([C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32, C.c_void_p], C.c_int),
    "b200sv_apply_observable": ([C.c_void_p, C.POINTER(Observable)], C.c_int),
    "b200sv_expval": ([C.c_void_p, C.POINTER(Observable), C.POINTER(C.c_double)], C.c_int),
    "b200sv_var": ([C.c_void_p, C.POINTER(Observable), C.POINTER(C.c_double)], C.c_int),
    "b200sv_expval_pauli": ([C.c_void_p, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                             C.POINTER(C.c_uint32), C.c_char_p, C.POINTER(C.c_double),
                             C.POINTER(C.c_double)], C.c_int),
    "b200sv_inner_product": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "b200sv_norm2": ([C.c_void_p, C.POINTER(C.c_double)], C.c_int),
    "b200sv_sample_mcmc": ([C.c_void_p, C.c_int, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint64,
                            C.POINTER(C.c_uint64)], C.c_int),
    "b200sv_expval_sparse_device": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                     C.POINTER(C.c_double)], C.c_int),
    "b200sv_var_sparse_device": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                  C.POINTER(C.c_double)], C.c_int),
    "b200sv_expval_sparse": ([C.c_void_p, C.POINTER(C.c_uint64), C.c_uint64, C.POINTER(C.c_uint64), C.c_void_p,
                              C.c_uint64, C.POINTER(C.c_double)], C.c_int),
    "b200sv_var_sparse": ([C.c_void_p, C.POINTER(C.c_uint64), C.c_uint64, C.POINTER(C.c_uint64), C.c_void_p,
                           C.c_uint64, C.POINTER(C.c_double)], C.c_int),
    "b200sv_sample": ([C.c_void_p, C.c_uint64, C.POINTER(C.c_double), C.c_uint64,
                       C.POINTER(C.c_uint64)], C.c_int),
    "b200sv_sample_bits": ([C.c_void_p, C.c_uint64, C.POINTER(C.c_double), C.c_uint64,
                            C.POINTER(C.c_uint64)], C.c_int),
    "b200sv_expval_pauli_noalloc": ([C.c_void_p, C.c_uint32, C.c_int, C.c_uint32, C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_uint32), C.c_char_p, C.c_void_p, C.c_void_p], C.c_int),
    "b200sv_adjoint_jacobian": ([C.c_void_p, C.POINTER(Op), C.c_uint32, C.POINTER(Observable), C.c_uint32,
                                 C.POINTER(C.c_uint64), C.c_uint32, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "b200sv_vjp_state": ([C.c_void_p, C.POINTER(Op), C.c_uint32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                          C.c_uint32, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "b200sv_batch_create": ([C.c_int, C.POINTER(BatchCircuit), C.c_uint32, C.c_uint64,
                             C.POINTER(C.c_void_p)], C.c_int),
    "b200sv_batch_destroy": ([C.c_void_p], C.c_int),
    "b200sv_batch_set_stream": ([C.c_void_p, C.c_void_p], C.c_int),
    "b200sv_batch_forward": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "b200sv_batch_vjp": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "b200sv_batch_jacobian": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "b200sv_batch_use_graphs": ([C.c_void_p, C.c_int], C.c_int),
    "b200sv_batch_autotune": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "b200sv_batch_last_launches": ([C.c_void_p, C.POINTER(C.c_uint32)], C.c_int),
}

_lib = None


def lib() -> C.CDLL:
    """Load libb200sv.so (once).  Raises if the library was not built."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(f"libb200sv.so not found at {_LIB_PATH}; run __graft_entry__.build() "
                              "(the CUDA extension is required, there is no CPU path)")
        L = C.CDLL(str(_LIB_PATH))
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def declared_symbols():
    return list(_SIGS)


def check(status: int) -> None:
    if status != B200SV_OK:
        msg = lib().b200sv_last_error().decode(errors="replace")
        raise B200Error(status, msg)


def device_count() -> int:
    n = C.c_int(0)
    check(lib().b200sv_device_count(C.byref(n)))
    return n.value


def _u32(seq):
    a = np.ascontiguousarray(np.asarray(seq, dtype=np.uint32))
    return a, a.ctypes.data_as(C.POINTER(C.c_uint32))


def _f64(seq):
    a = np.ascontiguousarray(np.asarray(seq, dtype=np.float64))
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


class OpList:
    """Packs a list of (name_or_id, wires, inverse, params[, matrix]) into b200sv_op records.

    All wires and parameters go into two contiguous arrays, and each record points into
    them, so packing costs a few hundred nanoseconds per op.  The object keeps every
    backing array alive for its lifetime."""

    def __init__(self, ops, complex_dtype=np.complex128):
        n = len(ops)
        self.n = n
        self._keep = []
        gids = np.empty(n, dtype=np.uint32)
        nw = np.empty(n, dtype=np.uint32)
        npar = np.empty(n, dtype=np.uint32)
        inv = np.empty(n, dtype=np.int32)
        wires, params = [], []
        mats = {}
        for i, op in enumerate(ops):
            name, w, inverse, p = op[:4]
            if isinstance(name, (int, np.integer)):
                gid = int(name)
            elif name in ("QubitUnitary", "Matrix"):
                gid = OP_MATRIX
            elif name in ("QubitStateVector", "BasisState", "StatePrep"):
                gid = OP_SKIP
            else:
                gid = GATE_IDS[name]
            gids[i] = gid
            nw[i] = len(w)
            wires.extend(w)
            p = () if p is None else p
            npar[i] = len(p)
            params.extend(p)
            inv[i] = 1 if inverse else 0
            if len(op) > 4 and op[4] is not None:
                mats[i] = np.ascontiguousarray(np.asarray(op[4], dtype=complex_dtype))
        W = np.ascontiguousarray(np.asarray(wires if wires else [0], dtype=np.uint32))
        P = np.ascontiguousarray(np.asarray(params if params else [0.0], dtype=np.float64))
        woff = np.concatenate([[0], np.cumsum(nw, dtype=np.uint64)[:-1]]).astype(np.uint64)
        poff = np.concatenate([[0], np.cumsum(npar, dtype=np.uint64)[:-1]]).astype(np.uint64)
        rec = np.zeros(max(1, n), dtype=_OP_DTYPE)
        if n:
            rec["gate"][:n] = gids
            rec["nwires"][:n] = nw
            rec["wires"][:n] = np.uint64(W.ctypes.data) + np.uint64(4) * woff[:n]
            rec["inverse"][:n] = inv
            rec["nparams"][:n] = npar
            rec["params"][:n] = np.uint64(P.ctypes.data) + np.uint64(8) * poff[:n]
            for i, m in mats.items():
                rec["matrix"][i] = m.ctypes.data
        self._keep += [W, P, list(mats.values()), rec]
        self.arr = C.cast(rec.ctypes.data, C.POINTER(Op))

    @property
    def ptr(self):
        return self.arr


class ObservableBuilder:
    """Builds b200sv_observable records.

    An observable is a list of terms ``(coeff, [factor, ...])``; a factor is
    ``(name, wires)`` for a named operator or ``("Hermitian", wires, matrix)``."""

    def __init__(self, terms, complex_dtype=np.complex128):
        self._keep = []
        self.terms = (Term * max(1, len(terms)))()
        for t, (coeff, factors) in enumerate(terms):
            fa = (Factor * max(1, len(factors)))()
            self._keep.append(fa)
            for j, f in enumerate(factors):
                w, wp = _u32(f[1])
                self._keep.append(w)
                fa[j].nwires = len(w)
                fa[j].wires = wp
                if f[0] == "Hermitian":
                    m = np.ascontiguousarray(np.asarray(f[2], dtype=complex_dtype))
                    self._keep.append(m)
                    fa[j].kind = FACTOR_MATRIX
                    fa[j].gate = 0
                    fa[j].matrix = m.ctypes.data
                else:
                    fa[j].kind = FACTOR_NAMED
                    fa[j].gate = GATE_IDS[f[0]]
                    fa[j].matrix = None
            self.terms[t].coeff = float(coeff)
            self.terms[t].nfactors = len(factors)
            self.terms[t].factors = fa
        self.obs = Observable(len(terms), self.terms)


class StateVector:
    """Device state vector handle (b200sv_create / b200sv_destroy)."""

    def __init__(self, num_qubits: int, dtype=np.complex128):
        self.num_qubits = int(num_qubits)
        self.np_dtype = np.dtype(dtype)
        self.code = B200SV_C64 if self.np_dtype == np.complex64 else B200SV_C128
        h = C.c_void_p()
        check(lib().b200sv_create(self.num_qubits, self.code, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().b200sv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # data movement
    def upload(self, data):
        a = np.ascontiguousarray(np.asarray(data, dtype=self.np_dtype))
        check(lib().b200sv_upload(self.h, a.ctypes.data, a.size))

    def download(self):
        a = np.empty(1 << self.num_qubits, dtype=self.np_dtype)
        check(lib().b200sv_download(self.h, a.ctypes.data, a.size))
        return a

    def copy_from(self, src: "StateVector"):
        """Device-to-device copy of another handle's amplitudes (same width and dtype)."""
        check(lib().b200sv_copy(self.h, src.h))

    def set_basis_state(self, index: int):
        check(lib().b200sv_set_basis_state(self.h, int(index)))

    def device_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().b200sv_device_ptr(self.h, C.byref(p)))
        return p.value

    def synchronize(self):
        check(lib().b200sv_synchronize(self.h))

    def set_stream(self, stream_handle: int | None):
        check(lib().b200sv_set_stream(self.h, C.c_void_p(stream_handle or 0)))

    # gates
    def apply(self, name, wires, inverse=False, params=()):
        gid = name if isinstance(name, int) else GATE_IDS[name]
        w, wp = _u32(wires)
        p, pp = _f64(params)
        check(lib().b200sv_apply_gate(self.h, gid, wp, len(w), 1 if inverse else 0, pp, len(p)))

    def apply_matrix(self, matrix, wires, inverse=False):
        m = np.ascontiguousarray(np.asarray(matrix, dtype=self.np_dtype))
        w, wp = _u32(wires)
        check(lib().b200sv_apply_matrix(self.h, m.ctypes.data, wp, len(w), 1 if inverse else 0))

    def _oplist(self, ops):
        return ops if isinstance(ops, OpList) else OpList(ops, self.np_dtype)

    def apply_ops(self, ops):
        ol = self._oplist(ops)
        check(lib().b200sv_apply_ops(self.h, ol.ptr, ol.n))

    def apply_ops_fused(self, ops):
        ol = self._oplist(ops)
        check(lib().b200sv_apply_ops_fused(self.h, ol.ptr, ol.n))

    def apply_generator(self, name, wires, adj=False) -> float:
        gid = name if isinstance(name, int) else GENERATOR_IDS[name]
        w, wp = _u32(wires)
        s = C.c_double()
        check(lib().b200sv_apply_generator(self.h, gid, wp, len(w), 1 if adj else 0, C.byref(s)))
        return s.value

    # measurements
    def probs(self, wires=None):
        wires = [] if wires is None else list(wires)
        k = len(wires) if wires else self.num_qubits
        out = np.empty(1 << k, dtype=np.float64)
        w, wp = _u32(wires)
        check(lib().b200sv_probs(self.h, wp, len(w), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def apply_observable(self, terms):
        """psi <- O psi (Observable::applyInPlace); terms as for expval."""
        ob = ObservableBuilder(terms, self.np_dtype)
        check(lib().b200sv_apply_observable(self.h, C.byref(ob.obs)))

    def expval(self, terms) -> float:
        ob = ObservableBuilder(terms, self.np_dtype)
        r = C.c_double()
        check(lib().b200sv_expval(self.h, C.byref(ob.obs), C.byref(r)))
        return r.value

    def var(self, terms) -> float:
        ob = ObservableBuilder(terms, self.np_dtype)
        r = C.c_double()
        check(lib().b200sv_var(self.h, C.byref(ob.obs), C.byref(r)))
        return r.value

    def _sparse(self, fn, indptr, indices, data) -> float:
        rows = np.ascontiguousarray(indptr, dtype=np.uint64)
        cols = np.ascontiguousarray(indices, dtype=np.uint64)
        vals = np.ascontiguousarray(data, dtype=self.np_dtype)
        r = C.c_double()
        check(fn(self.h, rows.ctypes.data_as(C.POINTER(C.c_uint64)), rows.size,
                 cols.ctypes.data_as(C.POINTER(C.c_uint64)), vals.ctypes.data_as(C.c_void_p), vals.size,
                 C.byref(r)))
        return r.value

    def expval_sparse(self, indptr, indices, data) -> float:
        """Re<psi|H psi> for H in CSR form (scipy's indptr, indices, data)."""
        return self._sparse(lib().b200sv_expval_sparse, indptr, indices, data)

    def var_sparse(self, indptr, indices, data) -> float:
        return self._sparse(lib().b200sv_var_sparse, indptr, indices, data)

    def expval_sparse_device(self, indptr_ptr: int, indices_ptr: int, data_ptr: int, nnz: int) -> float:
        """expval_sparse with the CSR arrays in device memory (uint64, uint64, the state's dtype)."""
        r = C.c_double()
        check(lib().b200sv_expval_sparse_device(self.h, C.c_void_p(indptr_ptr), C.c_void_p(indices_ptr),
                                                C.c_void_p(data_ptr), int(nnz), C.byref(r)))
        return r.value

    def var_sparse_device(self, indptr_ptr: int, indices_ptr: int, data_ptr: int, nnz: int) -> float:
        r = C.c_double()
        check(lib().b200sv_var_sparse_device(self.h, C.c_void_p(indptr_ptr), C.c_void_p(indices_ptr),
                                             C.c_void_p(data_ptr), int(nnz), C.byref(r)))
        return r.value

    def expval_pauli(self, words, coeffs=None):
        """words: list of (pauli_string, wires); returns (per-term values, weighted sum)."""
        coeffs = np.ones(len(words)) if coeffs is None else np.asarray(coeffs, dtype=np.float64)
        offs = [0]
        wires, letters = [], []
        for s, w in words:
            assert len(s) == len(w)
            wires += list(w)
            letters += list(s)
            offs.append(len(wires))
        o, op_ = _u32(offs)
        w, wp = _u32(wires)
        c, cp = _f64(coeffs)
        pl = "".join(letters).encode() + b"\0"
        out = np.empty(max(1, len(words)))
        tot = C.c_double()
        check(lib().b200sv_expval_pauli(self.h, len(words), cp, op_, wp, pl,
                                        out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(tot)))
        return out[:len(words)], tot.value

    def inner(self, ket: "StateVector") -> complex:
        re, im = C.c_double(), C.c_double()
        check(lib().b200sv_inner_product(self.h, ket.h, C.byref(re), C.byref(im)))
        return complex(re.value, im.value)

    def probs_device(self, out_ptr: int, wires=None):
        """probs(wires) into a caller-owned device buffer of 2^len(wires) doubles (all wires when None)."""
        w, wp = _u32([] if wires is None else wires)
        check(lib().b200sv_probs_device(self.h, wp, len(w), C.c_void_p(out_ptr)))

    def norm2(self) -> float:
        r = C.c_double()
        check(lib().b200sv_norm2(self.h, C.byref(r)))
        return r.value

    def sample(self, nshots: int, uniforms=None, seed: int = 0):
        out = np.empty(max(1, nshots), dtype=np.uint64)
        up = None
        if uniforms is not None:
            u, up = _f64(uniforms)
            assert len(u) == nshots
        check(lib().b200sv_sample(self.h, nshots, up, seed, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out[:nshots]

    def sample_bits(self, nshots: int, uniforms=None, seed: int = 0):
        out = np.empty(max(1, nshots * self.num_qubits), dtype=np.uint64)
        up = None
        if uniforms is not None:
            u, up = _f64(uniforms)
        check(lib().b200sv_sample_bits(self.h, nshots, up, seed, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out[:nshots * self.num_qubits].reshape(nshots, self.num_qubits)

    def sample_mcmc(self, proposal: int, num_burnin: int, nshots: int, nchains: int = 4096, seed: int = 0):
        """Basis indices from Metropolis chains (proposal MCMC_LOCAL or MCMC_NONZERO)."""
        out = np.empty(max(1, nshots), dtype=np.uint64)
        check(lib().b200sv_sample_mcmc(self.h, int(proposal), int(num_burnin), int(nshots), int(nchains), int(seed),
                                       out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out[:nshots]

    def sample_mcmc_bits(self, kernel_name: str, num_burnin: int, nshots: int, nchains: int = 4096, seed: int = 0):
        """generate_mcmc_samples: (nshots, n) bits, wire 0 first, with the reference's
        kernel-name binding (its "Local" name runs the non-zero proposal)."""
        idx = self.sample_mcmc(mcmc_proposal_for_name(kernel_name), num_burnin, nshots, nchains, seed)
        n = self.num_qubits
        shifts = np.arange(n - 1, -1, -1, dtype=np.uint64)
        return ((idx[:, None] >> shifts[None, :]) & np.uint64(1)).astype(np.uint64)

    def vjp_state(self, ops, dy, trainable, apply_operations=False):
        ol = OpList(ops, self.np_dtype)
        d = np.ascontiguousarray(np.asarray(dy, dtype=self.np_dtype))
        tp = np.ascontiguousarray(np.asarray(trainable, dtype=np.uint64))
        out = np.zeros(2 * max(1, len(tp)), dtype=np.float64)
        check(lib().b200sv_vjp_state(self.h, ol.ptr, ol.n, d.ctypes.data, d.size,
                                     tp.ctypes.data_as(C.POINTER(C.c_uint64)), len(tp), 1 if apply_operations else 0,
                                     out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[0:2 * len(tp):2] + 1j * out[1:2 * len(tp):2]

    def adjoint_jacobian(self, ops, observables, trainable, apply_operations=False):
        ol = OpList(ops, self.np_dtype)
        builders = [ObservableBuilder(t, self.np_dtype) for t in observables]
        arr = (Observable * max(1, len(builders)))(*[b.obs for b in builders])
        tp = np.ascontiguousarray(np.asarray(trainable, dtype=np.uint64))
        jac = np.zeros(max(1, len(builders) * len(tp)), dtype=np.float64)
        check(lib().b200sv_adjoint_jacobian(self.h, ol.ptr, ol.n, arr, len(builders),
                                            tp.ctypes.data_as(C.POINTER(C.c_uint64)), len(tp),
                                            1 if apply_operations else 0,
                                            jac.ctypes.data_as(C.POINTER(C.c_double))))
        return jac[:len(builders) * len(tp)].reshape(len(builders), len(tp))
