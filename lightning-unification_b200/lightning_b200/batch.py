"""Batched engine: many independent circuits in one persistent launch.

Python view of ``b200sv_batch_*`` (include/b200sv.h).  Parameters, outputs and
gradients are torch CUDA tensors (float64); torch provides the device memory
and the stream, the work itself runs in libb200sv's kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi


class BatchedCircuits:
    """A packed pool of circuits ``{"num_qubits", "ops", "param_index", "observables"}``.

    ``ops`` are ``(name, wires, inverse, params)``; ``param_index[i] >= 0`` makes op i
    read slot ``param_index[i]`` of the batch parameter vector; ``observables`` is a
    list of Pauli sums ``[(coeff, "XZ", [w0, w1]), ...]`` (one output each)."""

    def __init__(self, circuits, nparams: int, dtype=np.complex64, use_graphs: bool = True):
        self.dtype = np.dtype(dtype)
        self.code = capi.B200SV_C64 if self.dtype == np.complex64 else capi.B200SV_C128
        self.nparams = int(nparams)
        self.ncirc = len(circuits)
        self._keep = []
        arr = (capi.BatchCircuit * self.ncirc)()
        self.nobs = []
        self.param_ops = [sum(1 for p in c.get("param_index", []) if p >= 0) for c in circuits]
        for i, c in enumerate(circuits):
            ol = capi.OpList([tuple(op) for op in c["ops"]], self.dtype)
            pidx = np.ascontiguousarray(np.asarray(c.get("param_index", [-1] * len(c["ops"])), dtype=np.int64))
            obs = c.get("observables", [])
            nterms, coeffs, offs, wires, letters = [], [], [0], [], []
            for ob in obs:
                nterms.append(len(ob))
                for coeff, word, ws in ob:
                    assert len(word) == len(ws)
                    coeffs.append(float(coeff))
                    wires += list(ws)
                    letters += list(word)
                    offs.append(len(wires))
            nt = np.ascontiguousarray(np.asarray(nterms, dtype=np.uint32))
            co = np.ascontiguousarray(np.asarray(coeffs, dtype=np.float64))
            of = np.ascontiguousarray(np.asarray(offs, dtype=np.uint32))
            wi = np.ascontiguousarray(np.asarray(wires if wires else [0], dtype=np.uint32))
            pl = C.create_string_buffer(("".join(letters)).encode() + b"\0")
            self._keep += [ol, pidx, nt, co, of, wi, pl]
            rec = arr[i]
            rec.num_qubits = int(c["num_qubits"])
            rec.nops = ol.n
            rec.ops = ol.arr
            rec.param_index = pidx.ctypes.data_as(C.POINTER(C.c_int64))
            rec.nobs = len(obs)
            rec.obs_nterms = nt.ctypes.data_as(C.POINTER(C.c_uint32))
            rec.obs_coeffs = co.ctypes.data_as(C.POINTER(C.c_double))
            rec.obs_offsets = of.ctypes.data_as(C.POINTER(C.c_uint32))
            rec.obs_wires = wi.ctypes.data_as(C.POINTER(C.c_uint32))
            rec.obs_paulis = C.cast(pl, C.c_char_p)
            self.nobs.append(len(obs))
        h = C.c_void_p()
        capi.check(capi.lib().b200sv_batch_create(self.code, arr, self.ncirc, self.nparams, C.byref(h)))
        self.h = h
        self._keep = []  # the engine copied everything it needs
        self.total_obs = int(sum(self.nobs))
        self.out_offsets = np.concatenate([[0], np.cumsum(self.nobs)]).astype(np.int64)
        capi.check(capi.lib().b200sv_batch_use_graphs(self.h, 1 if use_graphs else 0))

    def close(self):
        if getattr(self, "h", None):
            capi.lib().b200sv_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _bind_stream(self):
        import torch
        capi.check(capi.lib().b200sv_batch_set_stream(self.h, C.c_void_p(torch.cuda.current_stream().cuda_stream)))

    @staticmethod
    def _ptr(t):
        import torch
        assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
        return C.c_void_p(t.data_ptr())

    def forward(self, params):
        """params: float64 CUDA tensor [nparams] -> outputs [total_obs] (circuit-major)."""
        import torch
        self._bind_stream()
        out = torch.empty(self.total_obs, dtype=torch.float64, device=params.device)
        capi.check(capi.lib().b200sv_batch_forward(self.h, self._ptr(params), self._ptr(out)))
        return out

    def vjp(self, params, dy):
        """sum_c sum_o dy[c,o] d<O_co>/dparams -> float64 CUDA tensor [nparams]."""
        import torch
        self._bind_stream()
        grad = torch.empty(self.nparams, dtype=torch.float64, device=params.device)
        dyc = dy.contiguous().to(torch.float64)
        capi.check(capi.lib().b200sv_batch_vjp(self.h, self._ptr(params), self._ptr(dyc), self._ptr(grad)))
        return grad

    def jacobian(self, params):
        """Per circuit, [nobs_c x nparamops_c] blocks concatenated (float64 CUDA tensor)."""
        import torch
        self._bind_stream()
        total = sum(n * c for n, c in zip(self.nobs, self.param_ops))
        jac = torch.zeros(max(1, total), dtype=torch.float64, device=params.device)
        capi.check(capi.lib().b200sv_batch_jacobian(self.h, self._ptr(params), self._ptr(jac)))
        return jac[:total]

    def autotune(self, params) -> int:
        self._bind_stream()
        ch = C.c_int(0)
        capi.check(capi.lib().b200sv_batch_autotune(self.h, self._ptr(params), C.byref(ch)))
        return ch.value

    def last_launches(self) -> int:
        n = C.c_uint32(0)
        capi.check(capi.lib().b200sv_batch_last_launches(self.h, C.byref(n)))
        return n.value

