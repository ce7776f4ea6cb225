"""The reference itself as an oracle — TEST INFRASTRUCTURE ONLY.

Loads the reference's lightning.qubit pybind11 module compiled from its own
sources by oracle/Makefile into oracle/_ref/lq_reference, and drives it through
its public Python surface (StateVectorC64/C128, MeasurementsC*, observables.*,
algorithms.AdjointJacobianC*).  Returns None from ``load()`` when the module was
not built, so callers can skip.
"""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np

_REF_DIR = Path(__file__).resolve().parent / "_ref"


def load():
    if not (_REF_DIR / "lq_reference").exists():
        return None
    if str(_REF_DIR) not in sys.path:
        sys.path.insert(0, str(_REF_DIR))
    try:
        return importlib.import_module("lq_reference.lightning_qubit_ops")
    except ImportError:
        return None


def _suffix(dtype):
    return "C64" if np.dtype(dtype) == np.complex64 else "C128"


def run_circuit(m, n, ops, dtype=np.complex128, state=None):
    """Apply ops (name, wires, inverse, params[, matrix]) with the reference's StateVector."""
    st = np.zeros(1 << n, dtype=dtype) if state is None else np.array(state, dtype=dtype)
    if state is None:
        st[0] = 1
    sv = getattr(m, "StateVector" + _suffix(dtype))(st)
    for op in ops:
        name, wires, inv, params = op[:4]
        if len(op) > 4 and op[4] is not None:
            sv.applyMatrix(np.ascontiguousarray(np.asarray(op[4], dtype=dtype).reshape(-1)), list(wires), inv)
        elif name in ("QubitStateVector", "BasisState", "StatePrep"):
            continue
        else:
            getattr(sv, name)(list(wires), inv, list(params))
    return st


def make_obs(m, terms, dtype=np.complex128):
    """Observable object from [(coeff, [(name, wires) | ("Hermitian", wires, matrix)])]."""
    s = _suffix(dtype)
    o = m.observables
    rdt = np.float32 if s == "C64" else np.float64

    def factor(f):
        if f[0] == "Hermitian":
            return getattr(o, "HermitianObs" + s)(np.ascontiguousarray(np.asarray(f[2], dtype=dtype).reshape(-1)),
                                                  list(f[1]))
        return getattr(o, "NamedObs" + s)(f[0], list(f[1]))

    def term(factors):
        if len(factors) == 1:
            return factor(factors[0])
        return getattr(o, "TensorProdObs" + s)([factor(f) for f in factors])

    if len(terms) == 1 and terms[0][0] == 1.0:
        return term(terms[0][1])
    return getattr(o, "Hamiltonian" + s)(np.array([t[0] for t in terms], dtype=rdt), [term(t[1]) for t in terms])


def expval(m, state, terms):
    dtype = state.dtype
    sv = getattr(m, "StateVector" + _suffix(dtype))(state)
    M = getattr(m, "Measurements" + _suffix(dtype))(sv)
    return float(M.expval(make_obs(m, terms, dtype)))


def var(m, state, terms):
    dtype = state.dtype
    sv = getattr(m, "StateVector" + _suffix(dtype))(state)
    M = getattr(m, "Measurements" + _suffix(dtype))(sv)
    return float(M.var(make_obs(m, terms, dtype)))


def probs(m, state, wires=None):
    dtype = state.dtype
    sv = getattr(m, "StateVector" + _suffix(dtype))(state)
    M = getattr(m, "Measurements" + _suffix(dtype))(sv)
    return np.asarray(M.probs() if wires is None else M.probs(list(wires)))


def adjoint_jacobian(m, state, ops, observables, trainable):
    dtype = state.dtype
    s = _suffix(dtype)
    sv = getattr(m, "StateVector" + s)(state)
    names = [op[0] for op in ops]
    params = [list(op[3]) for op in ops]
    wires = [list(op[1]) for op in ops]
    invs = [bool(op[2]) for op in ops]
    mats = [np.asarray(op[4], dtype=dtype).reshape(-1) if len(op) > 4 and op[4] is not None
            else np.zeros(0, dtype=dtype) for op in ops]
    opsd = getattr(m.algorithms, "create_ops_list" + s)(names, params, wires, invs, mats)
    obs = [make_obs(m, t, dtype) for t in observables]
    adj = getattr(m.algorithms, "AdjointJacobian" + s)()
    jac = np.asarray(adj(sv, obs, opsd, list(trainable)))
    return jac.reshape(len(observables), len(trainable))


def vjp_state(m, state, ops, dy, trainable):
    """VectorJacobianProductC*()(sv, ops, dy, tp) of the reference (LQ/bindings/LQubitBindings.hpp:186-246)."""
    dtype = state.dtype
    s = _suffix(dtype)
    sv = getattr(m, "StateVector" + s)(state)
    names = [op[0] for op in ops]
    params = [list(op[3]) for op in ops]
    wires = [list(op[1]) for op in ops]
    invs = [bool(op[2]) for op in ops]
    mats = [np.zeros(0, dtype=dtype) for _ in ops]
    opsd = getattr(m.algorithms, "create_ops_list" + s)(names, params, wires, invs, mats)
    vjp = getattr(m.algorithms, "VectorJacobianProduct" + s)()
    return np.asarray(vjp(sv, opsd, np.ascontiguousarray(np.asarray(dy, dtype=dtype)), list(trainable)))


def _sparse(m, state, indptr, indices, data, what):
    """MeasurementsC*.expval/var(row_map, entries, values) (LQ/bindings/LQubitBindings.hpp:127-161)."""
    dtype = state.dtype
    sv = getattr(m, "StateVector" + _suffix(dtype))(state)
    M = getattr(m, "Measurements" + _suffix(dtype))(sv)
    return float(getattr(M, what)(np.asarray(indptr, dtype=np.uint64), np.asarray(indices, dtype=np.uint64),
                                  np.asarray(data, dtype=dtype)))


def sparse_expval(m, state, indptr, indices, data):
    return _sparse(m, state, indptr, indices, data, "expval")


def sparse_var(m, state, indptr, indices, data):
    return _sparse(m, state, indptr, indices, data, "var")
