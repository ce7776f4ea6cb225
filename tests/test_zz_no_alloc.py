"""The allocation-free entry point, b200sv_expval_pauli_noalloc, called through
the C ABI on a caller-owned state and output buffer.

It serves callers that cannot call cudaMalloc when they need a result (device
memory owned by another allocator, allocation-free serving loops).  Its values
must equal those of the allocating entry point, b200sv_expval_pauli, within the
tolerances the other tests use, on two calls in a row (the static scratch array
keeps the previous call's contents).  This file is collected last so that a run
stopping at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from conftest import random_state

pytestmark = pytest.mark.gpu


def _pack(words):
    offs, wires, letters = [0], [], []
    for s, w in words:
        wires += list(w)
        letters += list(s)
        offs.append(len(wires))
    o = np.ascontiguousarray(np.asarray(offs, dtype=np.uint32))
    w = np.ascontiguousarray(np.asarray(wires if wires else [0], dtype=np.uint32))
    return o, w, ("".join(letters)).encode() + b"\0"


def _noalloc(capi, sv, words):
    import torch
    o, w, pl = _pack(words)
    out = torch.full((len(words),), float("nan"), dtype=torch.float64, device="cuda")
    capi.check(capi.lib().b200sv_expval_pauli_noalloc(
        C.c_void_p(sv.device_ptr()), sv.num_qubits, sv.code, len(words),
        o.ctypes.data_as(C.POINTER(C.c_uint32)), w.ctypes.data_as(C.POINTER(C.c_uint32)), pl,
        C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_noalloc_matches_allocating_entry_point(dtype):
    from lightning_b200 import capi
    rng = np.random.default_rng(2718)
    tol = 1e-12 if dtype == np.complex128 else 1e-6
    calls = [
        (11, [("Z", [0]), ("ZZ", [1, 2]), ("X", [3]), ("XX", [3, 7]), ("Y", [10]), ("XYZ", [0, 5, 9]),
              ("IZ", [4, 6]), ("ZX", [2, 8])]),
        (9, [("X", [8]), ("X", [8]), ("YY", [0, 4]), ("Z", [5]), ("ZZZ", [1, 3, 7]), ("I", [2])]),
    ]
    for n, words in calls:  # two calls in a row on different states and words
        sv = capi.StateVector(n, dtype)
        sv.upload(random_state(rng, n, dtype))
        want, _ = sv.expval_pauli(words)
        got = _noalloc(capi, sv, words)
        assert np.abs(got - want).max() < tol


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_noalloc_wide_state_full_word_budget(dtype):
    """22 qubits: the first pass runs on the capped grid (1184 blocks) with grid-stride loops.
    Exactly 32 words per call: 20 diagonal words in one pass, then a run of 12 words sharing
    one X mask (the 9..32-word kernel).  Two calls in a row on the same state with different
    words, each against the allocating entry point."""
    from lightning_b200 import capi
    rng = np.random.default_rng(22)
    n = 22
    tol = 1e-12 if dtype == np.complex128 else 1e-6
    sv = capi.StateVector(n, dtype)
    sv.upload(random_state(rng, n, dtype))
    diag = [("".join(rng.choice(["Z", "I"], 2)), [int(w) for w in rng.choice(n, 2, replace=False)])
            for _ in range(20)]
    xrun = [("X" + ("Z" if q % 2 else "I"), [3, q]) for q in range(4, 16)]
    yrun = [("YX" + ("Z" if q % 3 else "I"), [n - 1, 0, q]) for q in range(5, 17)]
    for words in (diag + xrun, yrun + diag):
        assert len(words) == 32
        want, _ = sv.expval_pauli(words)
        got = _noalloc(capi, sv, words)
        assert np.abs(got - want).max() < tol


def test_noalloc_rejects_host_output():
    """The output must be device memory of the current device; a host buffer is refused
    before anything is queued."""
    import torch
    from lightning_b200 import capi
    sv = capi.StateVector(4)
    o, w, pl = _pack([("Z", [0])])
    host = np.zeros(1)
    with pytest.raises(capi.B200Error, match="must be device memory"):
        capi.check(capi.lib().b200sv_expval_pauli_noalloc(
            C.c_void_p(sv.device_ptr()), sv.num_qubits, sv.code, 1,
            o.ctypes.data_as(C.POINTER(C.c_uint32)), w.ctypes.data_as(C.POINTER(C.c_uint32)), pl,
            C.c_void_p(host.ctypes.data), C.c_void_p(torch.cuda.current_stream().cuda_stream)))


def test_noalloc_rejects_too_many_words():
    from lightning_b200 import capi
    sv = capi.StateVector(4)
    words = [("Z", [q % 4]) for q in range(33)]
    with pytest.raises(capi.B200Error, match="at most 32 Pauli words"):
        _noalloc(capi, sv, words)
