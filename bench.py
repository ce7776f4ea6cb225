#!/usr/bin/env python
"""Benchmark: batched adjoint circuits/s vs the plain path, and 30-qubit gate HBM GB/s.

Headline (``value``): the batched adjoint workload — 1024 circuits of 16 qubits,
8 layers of Rot(phi, theta, omega) on every qubit (serialised RZ RY RZ) plus a
CNOT ring of layer-dependent range, 16 PauliZ observables per circuit,
complex64 with FP64 reductions — one step = batched forward expectation values
plus the adjoint vector-Jacobian product through torch.autograd, inputs resident
in HBM.  Reported beside it: the plain per-circuit complex128 path (one gate per
launch, the drop-in C ABI), the max gradient error against FP64, the 30-qubit
complex128 gate sweep with the dense-gate roofline, the end-to-end number
through the public API with host buffers, and the reference CPU path timed on
this host.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
(N > 1 runs N independent replicas under torchrun, one per GPU; weak scaling.)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT / "lightning-unification_b200"), str(ROOT / "oracle")]

METRIC = "batched adjoint circuits/s vs plain on B200 @1e-5; 30q gate HBM GB/s %peak"
WORKLOAD = dict(ncirc=1024, n=16, layers=8, seed=5)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------------------------
class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during a timed region."""

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()

    def summary(self):
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], 0.0, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
def reference_cpu(circuits, params, dy, nsample, dtype=np.complex64):
    """The reference's own CPU path on a bounded sample: forward with its StateVector,
    16 expectation values, and the adjoint VJP as one Hamiltonian observable
    (lightning_qubit.py:747-772).  Falls back to the NumPy port when oracle/_ref is absent."""
    import ref
    from lightning_b200.workloads import bind
    m = ref.load()
    kind = "reference" if m is not None else "port"
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    for ci in range(nsample):
        c = circuits[ci]
        ops = bind(c, params)
        nobs = len(c["observables"])
        w = dy[ci * nobs:(ci + 1) * nobs]
        ham = [[(float(w[o]), [("PauliZ", [o])]) for o in range(nobs)]]
        npo = sum(1 for p in c["param_index"] if p >= 0)
        if m is not None:
            st = ref.run_circuit(m, c["num_qubits"], ops, dtype)
            sv = getattr(m, "StateVector" + ("C64" if dtype == np.complex64 else "C128"))(st)
            M = getattr(m, "Measurements" + ("C64" if dtype == np.complex64 else "C128"))(sv)
            _ = [M.expval("PauliZ", [o]) for o in range(nobs)]
            ref.adjoint_jacobian(m, st, ops, ham, list(range(npo)))
        else:
            import lq_oracle as O
            st = O.run_circuit(c["num_qubits"], ops, dtype)
            _ = [O.expval(st, [(1.0, [("PauliZ", [o])])]) for o in range(nobs)]
            O.adjoint_jacobian(st, ops, ham, list(range(npo)))
    dt = time.perf_counter() - t0
    return {"value": nsample / dt, "unit": "circuits/s", "cores": threads if kind == "reference" else 1,
            "kind": kind, "sample": f"{nsample} of {len(circuits)} circuits, forward + 16 expvals + adjoint VJP, "
            f"complex64, OMP_NUM_THREADS={os.environ.get('OMP_NUM_THREADS', 'unset')}", "seconds": dt}


def run_reference_arm(args):
    from lightning_b200.workloads import rot_ring_batch
    circuits, params = rot_ring_batch(**WORKLOAD)
    rng = np.random.default_rng(0)
    dy = rng.normal(size=len(circuits) * WORKLOAD["n"])
    nsample = 4
    for _ in range(args.warmup):
        reference_cpu(circuits, params, dy, 1)
    t0 = time.perf_counter()
    res = None
    for _ in range(args.steps):
        res = reference_cpu(circuits, params, dy, nsample)
    dt = (time.perf_counter() - t0) / args.steps
    v = nsample / dt
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "circuits/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded)",
            "config": {"workload": "batched adjoint, 1024 circuits x 16 qubits x 8 Rot layers + CNOT rings, "
                       "16 PauliZ observables, complex64", "sample_per_step": nsample},
            "cpu_baseline": {k: res[k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "circuits/s"},
            "e2e": {"value": v, "unit": "circuits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
def max_over_ranks(value: float, dist=None) -> float:
    """The largest per-rank value (step times are reported as the max over ranks); every
    rank must call it.  Works with NCCL (a CUDA tensor) and gloo (a CPU tensor)."""
    if dist is None:
        return value
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: int, ms_per_step: float) -> float:
    """Whole-job throughput of `world` replicas each processing `units_per_rank` per step."""
    return world * units_per_rank / (ms_per_step / 1e3)


def timed(fn, steps, warmup, stream=None):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps  # ms


SWEEP_TOUCHED = {"Hadamard": 1.0, "RX": 1.0, "RY": 1.0, "RZ": 1.0, "CNOT": 0.5, "CZ": 0.25, "SWAP": 0.5,
                 "Toffoli": 0.25, "U2": 1.0, "U3": 1.0}  # fraction of the amplitudes each gate can change


def _sweep_call(target, kind, wires, mat):
    """One gate of the sweep set on `target` (this engine's StateVector or the reference's StateVectorC128)."""
    if kind in ("U2", "U3"):
        if hasattr(target, "apply_matrix"):
            return lambda: target.apply_matrix(mat, wires)
        flat = np.ascontiguousarray(mat.reshape(-1))
        return lambda: target.applyMatrix(flat, wires, False)
    params = [0.3] if kind in ("RX", "RY", "RZ") else []
    if hasattr(target, "apply"):
        return lambda: target.apply(kind, wires, False, params)
    return lambda: getattr(target, kind)(wires, False, params)


def gate_sweep(nq: int, hbm_peak: float, cpu: bool, draws: int = 6):
    """The gate-throughput configuration at nq qubits, complex128: for each gate kind of the sweep
    set, `draws` launches on uniformly drawn distinct wires (seeded), each timed alone with CUDA
    events (the state is larger than L2 from 26 qubits); GB/s of the amplitudes the gate can
    change (2 x 16 B each) and of the whole state.  Then the 200-gate random sequence per gate
    and fused.  Beside each gate, when the reference module is built and the host has the
    memory, the reference's own lightning.qubit on the same wires (fewer draws: its gate
    kernels are single-threaded), host clock around each call."""
    import torch
    from lightning_b200 import capi
    from lightning_b200.workloads import gate_sweep as sweep_ops, random_unitary
    sv = capi.StateVector(nq, np.complex128)
    stream = torch.cuda.current_stream()
    sv.set_stream(stream.cuda_stream)
    N = 1 << nq
    state_bytes = 16 * N
    rng = np.random.default_rng(100 + nq)
    plan = {}
    for kind in SWEEP_TOUCHED:
        k = {"CNOT": 2, "CZ": 2, "SWAP": 2, "Toffoli": 3, "U2": 2, "U3": 3}.get(kind, 1)
        plan[kind] = [([int(w) for w in rng.choice(nq, k, replace=False)],
                       random_unitary(rng, k) if kind in ("U2", "U3") else None) for _ in range(draws)]
    per = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for kind, draws_k in plan.items():
        for wires, mat in draws_k[:1]:
            f = _sweep_call(sv, kind, wires, mat)
            f(); f()
        ms = []
        for wires, mat in draws_k:
            f = _sweep_call(sv, kind, wires, mat)
            torch.cuda.synchronize()
            e0.record(stream)
            f()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        touched = 2 * 16 * N * SWEEP_TOUCHED[kind]
        g = [touched / (m * 1e6) for m in ms]
        per[kind] = {"ms_mean": float(np.mean(ms)), "gbs_touched_mean": float(np.mean(g)),
                     "gbs_touched_min": float(min(g)), "gbs_touched_max": float(max(g)),
                     "hbm_frac_mean": float(np.mean(g)) / hbm_peak,
                     "gbs_state_mean": float(np.mean([2 * state_bytes / (m * 1e6) for m in ms])),
                     "wires": [w for w, _ in draws_k]}
    ops = sweep_ops(nq, 200, seed=7)
    sweep = {}
    ol = capi.OpList(ops, np.complex128)
    for label, fn in (("unfused", sv.apply_ops), ("fused", sv.apply_ops_fused)):
        fn(capi.OpList(ops[:10], np.complex128))  # warm
        sv.synchronize()
        e0.record(stream)
        fn(ol)
        e1.record(stream)
        torch.cuda.synchronize()
        sweep[label] = e0.elapsed_time(e1)
    sv.close()
    out = {"qubits": nq, "dtype": "c128", "per_gate": per, "sweep_200_gates_ms": sweep,
           "fused_speedup": sweep["unfused"] / sweep["fused"]}
    if cpu and nq <= 30:
        import psutil
        import ref  # the reference module built from its sources: the CPU baseline only
        m = ref.load()
        if m is None:
            out["reference_cpu"] = "not timed: reference module not built"
        elif psutil.virtual_memory().available < 3 * state_bytes:
            out["reference_cpu"] = f"not timed: the host has less than {3 * state_bytes / 2**30:.0f} GiB free"
        else:
            host = np.full(N, 1 / np.sqrt(N), dtype=np.complex128)
            svr = m.StateVectorC128(host)
            nref = {26: 3, 28: 2}.get(nq, 1)
            for kind, draws_k in plan.items():
                ts = []
                for wires, mat in draws_k[:nref]:
                    f = _sweep_call(svr, kind, wires, mat)
                    t0 = time.perf_counter()
                    f()
                    ts.append(time.perf_counter() - t0)
                per[kind]["reference_cpu_gbs"] = float(np.mean([2 * 16 * N * SWEEP_TOUCHED[kind] / (t * 1e9)
                                                                for t in ts]))
            out["reference_cpu"] = {"draws_per_gate": nref, "threads": os.environ.get(
                "OMP_NUM_THREADS", f"unset ({os.cpu_count()} cores; the gate kernels are single-threaded)")}
            del svr, host
    elif cpu:
        out["reference_cpu"] = f"not timed: {nq} qubits ({state_bytes / 2**30:.0f} GiB) is beyond the host-timed sizes"
    return out


def sweep_roofline(sw30: dict, hbm_peak: float):
    """Roofline of the dense one-wire kernel (RX, k_dense<double,1> or k_dense1_low on bit 0)
    from the 30-qubit sweep's RX draws; traffic from one ncu capture of an RX launch on a
    26-qubit complex128 state, scaled by the state size."""
    nq = sw30["qubits"]
    rx = sw30["per_gate"]["RX"]
    return {"bound": "hbm", "kernel": f"k_dense<double,1> (RX on random wires, {nq} qubits complex128)",
            "achieved": rx["gbs_touched_mean"], "peak": hbm_peak, "unit": "GB/s",
            "frac": rx["gbs_touched_mean"] / hbm_peak,
            "traffic": RX_DRAM_BYTES_26Q * float(1 << (nq - 26)),
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one RX launch on a "
                              "26-qubit complex128 state, scaled by the state size",
            "algorithmic_bytes_per_launch": 2 * 16 * (1 << nq)}


def rows_30q(nq: int, hbm_peak: float, cpu: bool, cpu_qubits: int = 26, steps: int = 3):
    """The remaining single-state rows on an nq-qubit complex128 random state: state copy and
    reset, the gates outside the sweep (MultiRZ, excitations, Ising, controlled rotations),
    generators, probs, expval and var.  Per op: ms (CUDA events), algorithmic bytes (gates:
    2 x 16 B x the amplitudes the op can change; reductions: 16 B per amplitude read; probs
    adds 8 B per output), GB/s and the fraction of the measured copy peak; beside it, when the
    reference module is built, the same op timed once with the reference's own lightning.qubit
    on a cpu_qubits-qubit state on the host cores (GB/s of the same algorithmic bytes)."""
    import torch
    from lightning_b200 import capi
    from lightning_b200.workloads import random_unitary
    N = 1 << nq
    S = 16
    st = torch.cuda.current_stream()
    sv = capi.StateVector(nq, np.complex128)
    sv.set_stream(st.cuda_stream)
    other = capi.StateVector(nq, np.complex128)
    other.set_stream(st.cuda_stream)
    rng = np.random.default_rng(5)
    sv.apply_ops([("Hadamard", [q], False, []) for q in range(nq)] +
                 [("RY", [q], False, [float(rng.uniform(0, 6.28))]) for q in range(nq)])
    probs_out = torch.empty(N, dtype=torch.float64, device="cuda")
    probs_small = torch.empty(1 << 10, dtype=torch.float64, device="cuda")
    h2 = random_unitary(rng, 2)
    h2 = (h2 + h2.conj().T) / 2
    ham = [("ZZ", [q, (q + 1) % nq]) for q in range(nq)] + [("ZZ", [q, (q + 2) % nq]) for q in range(nq)] + \
          [("X", [q]) for q in range(nq)]
    from lightning_b200.workloads import jordan_wigner_words
    jw = jordan_wigner_words(np.random.default_rng(5), nq, 400)
    # (label, call, algorithmic bytes, reference op or None)
    rows = [
        ("copy (A1)", lambda: other.copy_from(sv), 2 * S * N, None),
        ("set_basis_state (A1)", lambda: other.set_basis_state(0), S * N, None),
        ("MultiRZ 5 wires (A11)", lambda: sv.apply("MultiRZ", [0, 3, 7, 12, nq - 1], False, [0.3]), 2 * S * N,
         ("MultiRZ", [0, 3, 7, 12, -1], [0.3])),
        ("IsingXX (A11)", lambda: sv.apply("IsingXX", [4, nq - 3], False, [0.3]), 2 * S * N,
         ("IsingXX", [4, -3], [0.3])),
        ("CRX (A8)", lambda: sv.apply("CRX", [2, nq - 4], False, [0.3]), 2 * S * N // 2, ("CRX", [2, -4], [0.3])),
        ("ControlledPhaseShift (A8)", lambda: sv.apply("ControlledPhaseShift", [6, 9], False, [0.3]),
         2 * S * N // 4, ("ControlledPhaseShift", [6, 9], [0.3])),
        ("SingleExcitation (A11)", lambda: sv.apply("SingleExcitation", [3, nq - 6], False, [0.3]), 2 * S * N // 2,
         ("SingleExcitation", [3, -6], [0.3])),
        ("DoubleExcitation (A11)", lambda: sv.apply("DoubleExcitation", [0, 5, 11, nq - 2], False, [0.3]),
         2 * S * N // 8, ("DoubleExcitation", [0, 5, 11, -2], [0.3])),
        ("generator RX (A12)", lambda: sv.apply_generator("RX", [8]), 2 * S * N, None),
        ("generator CRY (A12)", lambda: sv.apply_generator("CRY", [1, 10]), 2 * S * N, None),
        ("generator MultiRZ (A12)", lambda: sv.apply_generator("MultiRZ", [2, 4, 6]), 2 * S * N, None),
        ("probs all wires, device output (A13)", lambda: sv.probs_device(probs_out.data_ptr()), S * N + 8 * N, None),
        ("probs 10 wires (A13)", lambda: sv.probs_device(probs_small.data_ptr(), list(range(5, 15))), S * N, None),
        ("expval Z0 X5 (A14)", lambda: sv.expval([(1.0, [("PauliZ", [0]), ("PauliX", [5])])]), S * N,
         ("expval", [(1.0, [("PauliZ", [0]), ("PauliX", [5])])])),
        ("expval Hermitian 2 wires (A14)", lambda: sv.expval([(1.0, [("Hermitian", [3, 17], h2)])]), S * N,
         ("expval", [(1.0, [("Hermitian", [3, 17], h2)])])),
        (f"expval_pauli {3 * nq}-term ZZ/X Hamiltonian (A14)", lambda: sv.expval_pauli(ham), S * N, None),
        ("expval_pauli 400-word Jordan-Wigner sum (A14)", lambda: sv.expval_pauli(jw), S * N, None),
        ("var Y7 (A15)", lambda: sv.var([(1.0, [("PauliY", [7])])]), S * N, ("var", [(1.0, [("PauliY", [7])])])),
    ]
    out = {}
    for label, fn, nbytes, _ in rows:
        ms = timed(fn, steps, 2, st)
        out[label] = {"ms": ms, "algorithmic_bytes": nbytes, "gbs": nbytes / (ms * 1e6),
                      "hbm_frac": nbytes / (ms * 1e6) / hbm_peak}
    sv.close()
    other.close()
    del probs_out
    if cpu:
        import ref  # the reference module built from its sources: the CPU baseline only
        m = ref.load()
        if m is not None:
            n2 = cpu_qubits
            N2 = 1 << n2
            st_np = (rng.normal(size=N2) + 1j * rng.normal(size=N2)).astype(np.complex128)
            st_np /= np.linalg.norm(st_np)
            svr = m.StateVectorC128(st_np)
            scale = N2 / N
            for label, _, nbytes, spec in rows:
                if spec is None:
                    continue
                t0 = time.perf_counter()
                if spec[0] in ("expval", "var"):
                    getattr(ref, spec[0])(m, st_np, spec[1])
                else:
                    wires = [w if w >= 0 else n2 + w for w in spec[1]]
                    getattr(svr, spec[0])(wires, False, list(spec[2]))
                dt = time.perf_counter() - t0
                out[label]["reference_cpu_gbs"] = nbytes * scale / (dt * 1e9)
            out["reference_cpu"] = {"qubits": n2, "threads": os.environ.get("OMP_NUM_THREADS",
                                                                            f"unset ({os.cpu_count()} cores)"),
                                    "note": "one call per op, same algorithmic bytes scaled to the state size"}
    return out


def next_rows(cpu: bool, reps: int = 7):
    """The rows beside the core path, complex128: the state-return VJP (20 qubits, 2 layers of
    RX RY RZ + CNOT ladder, 120 parameters), a sparse Hamiltonian expectation value (22 qubits,
    the periodic tridiagonal CSR matrix of the reference's tests, 3 entries per row) and
    Metropolis sampling (20 qubits, local proposal, 4096 chains).  GPU calls through the C ABI
    (median of `reps`, host clock around the call, results back on the host); beside them the
    reference module compiled from its sources, once, on the host cores."""
    from lightning_b200 import capi
    from lightning_b200.workloads import layered_rotations
    rng = np.random.default_rng(17)
    out = {}

    def med(fn):
        fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t0) * 1e3)
        return float(np.median(ts))

    # state-return VJP
    n = 20
    ops, _, _ = layered_rotations(n=n, layers=2, seed=3)
    tp = list(range(sum(1 for op in ops if op[3])))
    sv = capi.StateVector(n, np.complex128)
    sv.apply_ops(ops)
    psi = sv.download()
    dy = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    dy /= np.linalg.norm(dy)
    vjp = sv.vjp_state(ops, dy, tp)
    out["vjp_state"] = {"qubits": n, "params": len(tp), "ms": med(lambda: sv.vjp_state(ops, dy, tp))}
    sv.close()
    # sparse Hamiltonian
    ns = 22
    N = 1 << ns
    r = np.arange(N, dtype=np.uint64)
    indptr = np.arange(N + 1, dtype=np.uint64) * 3
    cols = np.stack([(r + N - 1) % N, r, (r + 1) % N], axis=1)
    vals = np.tile(np.array([-1.0, 1.0, -1.0], dtype=np.complex128), (N, 1))
    order = np.argsort(cols, axis=1, kind="stable")  # columns ascending within a row
    indices = np.take_along_axis(cols, order, axis=1).reshape(-1).astype(np.uint64)
    data = np.take_along_axis(vals, order, axis=1).reshape(-1)
    st = (rng.normal(size=N) + 1j * rng.normal(size=N)).astype(np.complex128)
    st /= np.linalg.norm(st)
    sv = capi.StateVector(ns, np.complex128)
    sv.upload(st)
    ev = sv.expval_sparse(indptr, indices, data)
    out["sparse_expval"] = {"qubits": ns, "nnz": int(3 * N), "ms": med(lambda: sv.expval_sparse(indptr, indices, data))}
    import torch
    dp = torch.tensor(indptr.astype(np.int64), device="cuda")
    di = torch.tensor(indices.astype(np.int64), device="cuda")
    dv = torch.tensor(data, device="cuda")
    out["sparse_expval"]["device_arrays_ms"] = med(
        lambda: sv.expval_sparse_device(dp.data_ptr(), di.data_ptr(), dv.data_ptr(), int(3 * N)))
    del dp, di, dv
    sv.close()
    # Metropolis sampling
    nm = 20
    sm = (rng.normal(size=1 << nm) + 1j * rng.normal(size=1 << nm)).astype(np.complex128)
    sm /= np.linalg.norm(sm)
    sv = capi.StateVector(nm, np.complex128)
    sv.upload(sm)
    shots = 1_000_000
    ms = med(lambda: sv.sample_mcmc(capi.MCMC_LOCAL, 100, shots, 4096, seed=1))
    out["mcmc_local"] = {"qubits": nm, "shots": shots, "burnin": 100, "chains": 4096, "ms": ms,
                         "shots_per_s": shots / (ms / 1e3)}
    sv.close()
    if cpu:
        import ref  # the reference module built from its sources: the CPU baseline only
        m = ref.load()
        if m is not None:
            t0 = time.perf_counter()
            want = ref.vjp_state(m, psi.copy(), ops, dy, tp)
            out["vjp_state"]["reference_cpu_ms"] = (time.perf_counter() - t0) * 1e3
            out["vjp_state"]["max_abs_diff"] = float(np.abs(vjp - want).max())
            t0 = time.perf_counter()
            ev_ref = ref.sparse_expval(m, st.copy(), indptr, indices, data)
            out["sparse_expval"]["reference_cpu_ms"] = (time.perf_counter() - t0) * 1e3
            out["sparse_expval"]["abs_diff"] = abs(ev - ev_ref)
            svr = m.StateVectorC128(sm.copy())
            rshots = 100_000
            t0 = time.perf_counter()
            m.MeasurementsC128(svr).generate_mcmc_samples(nm, "Local", 100, rshots)
            dt = time.perf_counter() - t0
            out["mcmc_local"]["reference_cpu_shots_per_s"] = rshots / dt
            out["reference_cpu"] = {"threads": os.environ.get("OMP_NUM_THREADS", f"unset ({os.cpu_count()} cores)"),
                                    "note": "one call each; the reference's Metropolis run takes 1e5 shots"}
    return out


def matrix_sweep(nq: int, hbm_peak: float, kmax: int = 8, steps: int = 3):
    """applyMatrix of random k-wire unitaries (k = 1..kmax, seeded wires) on an nq-qubit state,
    complex128 and complex64: ms per launch, HBM GB/s (2 x bytes of the state) and the matrix
    arithmetic in TFLOP/s (8 * 2^k real flops per amplitude).  Dense blocks cross from the
    HBM roofline to the FP64 (complex128) or compensated-FP32 (complex64) one near k = 4."""
    import torch
    from lightning_b200 import capi
    from lightning_b200.workloads import random_unitary
    rng = np.random.default_rng(11)
    st = torch.cuda.current_stream()
    out = {}
    for dt, label, S in ((np.complex128, "c128", 16), (np.complex64, "c64", 8)):
        sv = capi.StateVector(nq, dt)
        sv.set_stream(st.cuda_stream)
        N = 1 << nq
        rows = {}
        for k in range(1, kmax + 1):
            u = random_unitary(rng, k).astype(dt)
            wires = [int(w) for w in rng.choice(nq, size=k, replace=False)]
            ms = timed(lambda: sv.apply_matrix(u, wires), steps, 2, st)
            rows[str(k)] = {"wires": wires, "ms": ms, "gbs": 2 * S * N / (ms * 1e6),
                            "hbm_frac": 2 * S * N / (ms * 1e6) / hbm_peak,
                            "tflops": 8 * (1 << k) * N / (ms * 1e9)}
        sv.close()
        out[label] = rows
    return {"qubits": nq, "per_k": out}


# DRAM bytes (read + write) of one k_dense<double,1> launch (RX) on a 26-qubit complex128
# state, from an ncu capture; the kernel streams each amplitude once, so the traffic
# grows in proportion to the state.
RX_DRAM_BYTES_26Q = 1.0738e9 + 1.0144e9

# DRAM bytes (read + write) of the forward and VJP launches of the batched kernel on 148
# circuits of the batched-adjoint workload, from an ncu capture of `bench.py --case batch`;
# circuits are independent, so a step's traffic scales with the number of circuits.
BATCH_DRAM_BYTES_148 = (0.0397e9 + 0.9832e9) + (3.1324e9 + 3.5031e9)
BATCH_ISSUE_ACTIVE = 0.47  # scheduler cycles issuing, same capture (forward 52 %, VJP 45 %, time-weighted)


def run_case(args):
    """Small single-kernel cases for profiling: `gate` applies RX to a complex128 state of
    --qubits qubits; `batch` runs forward + VJP of --ncirc circuits of the batched workload."""
    import torch
    from lightning_b200 import capi
    torch.cuda.set_device(0)
    if args.case == "gate":
        # --gate on --wires (negative wires count from the last qubit), complex128
        sv = capi.StateVector(args.qubits, np.complex128)
        st = torch.cuda.current_stream()
        sv.set_stream(st.cuda_stream)
        wires = [w % args.qubits for w in (int(x) for x in args.wires.split(","))]
        par = [0.3] if args.gate in capi.GENERATOR_IDS else [0.1, 0.2, 0.3] if args.gate in ("Rot", "CRot") else []
        ms = timed(lambda: sv.apply(args.gate, wires, False, par), args.steps, args.warmup, st)
        gbs = 2 * 16 * (1 << args.qubits) / (ms * 1e6)
        print(json.dumps({"case": "gate", "gate": args.gate, "wires": wires, "qubits": args.qubits, "ms": ms,
                          "gbs_full_state": gbs}))
        return
    if args.case == "matrix":
        # one random --k-wire unitary per step on a --qubits-qubit state (profiling)
        from lightning_b200.workloads import random_unitary
        dt = np.complex64 if args.dtype == "c64" else np.complex128
        sv = capi.StateVector(args.qubits, dt)
        st = torch.cuda.current_stream()
        sv.set_stream(st.cuda_stream)
        rng = np.random.default_rng(11)
        u = random_unitary(rng, args.k).astype(dt)
        wires = [int(w) for w in rng.choice(args.qubits, size=args.k, replace=False)]
        ms = timed(lambda: sv.apply_matrix(u, wires), args.steps, args.warmup, st)
        print(json.dumps({"case": "matrix", "qubits": args.qubits, "k": args.k, "dtype": args.dtype, "wires": wires,
                          "ms": ms, "tflops": 8 * (1 << args.k) * (1 << args.qubits) / (ms * 1e9)}))
        return
    if args.case == "pauli":
        # Pauli sums on a --qubits state (--dtype): the 3n-term ZZ/X Hamiltonian and 400
        # Jordan-Wigner words, one expval_pauli call each per step (profiling of the Pauli passes)
        from lightning_b200.workloads import jordan_wigner_words
        dt = np.complex64 if args.dtype == "c64" else np.complex128
        n = args.qubits
        sv = capi.StateVector(n, dt)
        st = torch.cuda.current_stream()
        sv.set_stream(st.cuda_stream)
        sv.apply_ops([("RY", [q], False, [0.1 + 0.07 * q]) for q in range(n)] +
                     [("CNOT", [q, q + 1], False, []) for q in range(n - 1)] +
                     [("RX", [q], False, [0.3 - 0.01 * q]) for q in range(n)])
        zzx = [("ZZ", [q, (q + 1) % n]) for q in range(n)] + [("ZZ", [q, (q + 2) % n]) for q in range(n)] + \
              [("X", [q]) for q in range(n)]
        jw = jordan_wigner_words(np.random.default_rng(5), n, 400)
        res = {"case": "pauli", "qubits": n, "dtype": args.dtype}
        for name, words in (("zzx_ms", zzx), ("jw400_ms", jw)):
            res[name] = timed(lambda: sv.expval_pauli(words), args.steps, args.warmup, st)
        print(json.dumps(res))
        return
    if args.case == "plain":
        print(json.dumps({"case": "plain", **plain_layered(not args.no_cpu)}))
        return
    if args.case == "next":
        print(json.dumps({"case": "next", **next_rows(not args.no_cpu)}))
        return
    if args.case == "rows":
        print(json.dumps({"case": "rows", **rows_30q(args.qubits, peaks()[0], not args.no_cpu)}))
        return
    if args.case == "precision":
        res = {"case": "precision",
               "c64_33q": precision_case(33, np.complex64),
               "c128_32q": precision_case(32, np.complex128),
               "c64_vs_c128_32q": precision_compare(32)}
        print(json.dumps(res))
        return
    if args.case == "fused":
        from lightning_b200.workloads import gate_sweep, random_state
        ops = gate_sweep(args.qubits, 200, seed=7)
        dt = np.complex64 if args.dtype == "c64" else np.complex128
        sv = capi.StateVector(args.qubits, dt)
        sv.upload(random_state(args.qubits, seed=3, dtype=dt))
        st = torch.cuda.current_stream()
        sv.set_stream(st.cuda_stream)
        ol = capi.OpList(ops, dt)
        res = {"case": "fused", "qubits": args.qubits, "dtype": args.dtype, "gates": len(ops)}
        for name, fn in (("fused", sv.apply_ops_fused), ("unfused", sv.apply_ops)):
            res[name + "_ms"] = timed(lambda: fn(ol), args.steps, args.warmup, st)
        print(json.dumps(res))
        return
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.autograd import batched_expval
    from lightning_b200.workloads import rot_ring_batch
    circuits, params_np = rot_ring_batch(**(WORKLOAD | {"ncirc": args.ncirc}))
    eng = BatchedCircuits(circuits, len(params_np), dtype=np.complex64, use_graphs=False)
    params = torch.tensor(params_np, dtype=torch.float64, device="cuda", requires_grad=True)
    dy = torch.ones(eng.total_obs, dtype=torch.float64, device="cuda")

    def step():
        out = batched_expval(params, eng)
        torch.autograd.grad(out, params, dy)
    ms = timed(step, args.steps, args.warmup)
    print(json.dumps({"case": "batch", "ncirc": args.ncirc, "ms": ms, "circuits_per_s": args.ncirc / (ms / 1e3)}))


def hea_forward(steps: int, warmup: int, ncirc: int = 4096, dtype=np.complex64, cpu: bool = False):
    """Batched hardware-efficient-ansatz forward (n ~ U[10, 20], depth ~ U[4, 16], 3n-term
    Hamiltonian) in `dtype`, one persistent launch replayed as a CUDA graph, vs a per-circuit
    loop through the plain C ABI on a sample (after one untimed circuit per width).  With
    `cpu`, the reference's own lightning.qubit on the host cores over a seeded subset (the
    first 16 circuits: forward, then the Hamiltonian's expectation value as one observable),
    extrapolated to the whole batch and labelled as such."""
    import torch
    from lightning_b200 import capi
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.workloads import hea_batch, bind
    circuits, params_np = hea_batch(ncirc=ncirc, seed=11)
    eng = BatchedCircuits(circuits, len(params_np), dtype=dtype, use_graphs=True)
    params = torch.tensor(params_np, dtype=torch.float64, device="cuda")
    ms = timed(lambda: eng.forward(params), steps, warmup)
    out = eng.forward(params).cpu().numpy()
    nsample = 16
    handles = {}

    def one(c):
        n = c["num_qubits"]
        if n not in handles:
            handles[n] = capi.StateVector(n, dtype)
        sv = handles[n]
        sv.set_basis_state(0)
        sv.apply_ops(bind(c, params_np))
        words = [(w, ws) for _, w, ws in c["observables"][0]]
        coeffs = [cf for cf, _, _ in c["observables"][0]]
        return sv.expval_pauli(words, coeffs)[1]
    for c in circuits[:nsample]:
        one(c)  # warm-up: handles created, kernels loaded
    t0 = time.perf_counter()
    plain = [one(c) for c in circuits[:nsample]]
    plain_s = time.perf_counter() - t0
    for sv in handles.values():
        sv.close()
    err = float(np.abs(np.array(plain) - out[:nsample]).max())
    res = {"circuits": ncirc, "dtype": "c64" if np.dtype(dtype) == np.complex64 else "c128",
           "value": ncirc / (ms / 1e3), "unit": "circuits/s",
           "ms_per_step": ms, "per_circuit_loop": nsample / plain_s, "ratio": (ncirc / (ms / 1e3)) / (nsample / plain_s),
           "max_abs_diff_vs_loop": err}
    if cpu:
        import ref  # the reference module built from its sources: the CPU baseline only
        from lightning_b200.workloads import obs_terms
        m = ref.load()
        if m is not None:
            rdt = np.complex64 if np.dtype(dtype) == np.complex64 else np.complex128
            t0 = time.perf_counter()
            vals = []
            for c in circuits[:nsample]:
                st_ = ref.run_circuit(m, c["num_qubits"], bind(c, params_np), rdt)
                vals.append(ref.expval(m, st_, obs_terms(c["observables"][0])))
            dt = time.perf_counter() - t0
            res["reference_cpu"] = {"sample_circuits": nsample, "circuits_per_s": nsample / dt,
                                    "extrapolated_batch_s": dt / nsample * ncirc,
                                    "max_abs_diff_vs_batch": float(np.abs(np.array(vals) - out[:nsample]).max()),
                                    "note": "seeded subset, extrapolated to the whole batch by circuit count",
                                    "threads": os.environ.get("OMP_NUM_THREADS", f"unset ({os.cpu_count()} cores)")}
            res["ratio_vs_reference_cpu"] = res["value"] / (nsample / dt)
    return res


def plain_layered(cpu: bool, reps: int = 7):
    """The plain single-circuit configuration: 20 qubits complex128, 10 layers of RX RY RZ on
    every qubit + CNOT ladder (790 gates), <Z0> and the 600-parameter adjoint Jacobian, through
    the C ABI (one launch per gate), timed as the host sees each call (median of `reps`);
    beside it the reference module compiled from its sources, when present, on the host cores."""
    from lightning_b200 import capi
    from lightning_b200.workloads import layered_rotations
    ops, obs, tp = layered_rotations()
    sv = capi.StateVector(20, np.complex128)

    def fwd():
        sv.set_basis_state(0)
        sv.apply_ops(ops)
        return sv.expval(obs[0])

    def fused():
        sv.set_basis_state(0)
        sv.apply_ops_fused(ops)
        return sv.expval(obs[0])

    res = {"qubits": 20, "dtype": "c128", "gates": len(ops), "params": len(tp)}
    for label, fn in (("forward_expval_ms", fwd), ("forward_fused_expval_ms", fused),
                      ("adjoint_ms", lambda: sv.adjoint_jacobian(ops, obs, tp))):
        fwd()
        fn()
        ts = []
        for _ in range(reps):
            if label == "adjoint_ms":
                fwd()
            t0 = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t0) * 1e3)
        res[label] = float(np.median(ts))
    jac = sv.adjoint_jacobian(ops, obs, tp)
    sv.close()
    if cpu:
        import ref  # the reference module built from its sources: the CPU baseline only
        m = ref.load()
        if m is not None:
            t0 = time.perf_counter()
            psi = ref.run_circuit(m, 20, ops)
            ez = ref.expval(m, psi.copy(), obs[0])
            t1 = time.perf_counter()
            want = ref.adjoint_jacobian(m, psi, ops, obs, tp)
            t2 = time.perf_counter()
            res["reference_cpu"] = {"forward_expval_ms": (t1 - t0) * 1e3, "adjoint_ms": (t2 - t1) * 1e3,
                                    "threads": os.environ.get("OMP_NUM_THREADS", f"unset ({os.cpu_count()} cores)"),
                                    "max_abs_jac_diff": float(np.abs(jac - want).max()), "expval": ez}
    return res


def sampling_case(nq: int, shots: int = 10_000_000):
    """RY layer + QFT-style ladder applied with the fused path, then `shots` samples by the
    fixed-order inverse CDF (device Philox draws); chi-squared of the sampled top-10-wire marginal."""
    import torch
    from lightning_b200 import capi
    from lightning_b200.workloads import qft_circuit
    sv = capi.StateVector(nq, np.complex128)
    st = torch.cuda.current_stream()
    sv.set_stream(st.cuda_stream)
    ops = qft_circuit(nq, seed=9)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sv.apply_ops_fused(ops)
    sv.synchronize()
    t_gates = time.perf_counter() - t0
    t0 = time.perf_counter()
    idx = sv.sample(shots, seed=2024)
    t_sample = time.perf_counter() - t0
    k = min(10, nq)
    marg = sv.probs(list(range(k)))
    hist = np.bincount((idx >> np.uint64(nq - k)).astype(np.int64), minlength=1 << k)
    expct = marg * shots
    mask = expct > 5
    chi2 = float(((hist[mask] - expct[mask]) ** 2 / expct[mask]).sum())
    dof = int(mask.sum()) - 1
    sv.close()
    return {"qubits": nq, "dtype": "c128", "gates": len(ops), "gates_fused_s": t_gates, "shots": shots,
            "sample_s": t_sample, "shots_per_s": shots / t_sample, "chi2": chi2, "chi2_dof": dof,
            "chi2_per_dof": chi2 / max(dof, 1)}


def product_marginal(thetas, wires):
    """probs(wires) of the product state RY(theta_q)|0> on every wire, in FP64 (closed form)."""
    out = np.ones(1)
    for w in wires:
        out = np.kron(out, [np.cos(thetas[w] / 2) ** 2, np.sin(thetas[w] / 2) ** 2])
    return out


def precision_case(nq: int, dtype, shots: int = 10_000_000):
    """Full-size precision and sampling run: RY layer + QFT ladder (fused) on an nq-qubit
    state, probs over every wire into device memory (2^nq doubles), then `shots` samples by
    the fixed-order inverse CDF.  Size-independent checks: |norm^2 - 1|, |sum(probs) - 1|,
    chi-squared of the sampled top-10-wire marginal.  Then the inverse QFT (fused) returns
    the RY product state, whose <Z_q> = cos(theta_q) and marginals are known in FP64: the
    errors of the engine's expectation values and marginals against that FP64 answer."""
    import torch
    from lightning_b200 import capi
    from lightning_b200.workloads import qft_circuit
    sv = capi.StateVector(nq, dtype)
    st = torch.cuda.current_stream()
    sv.set_stream(st.cuda_stream)
    ops = qft_circuit(nq, seed=9)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sv.apply_ops_fused(ops)
    e1.record(st)
    torch.cuda.synchronize()
    t_gates = e0.elapsed_time(e1) / 1e3
    norm_err = abs(sv.norm2() - 1.0)
    probs = torch.empty(1 << nq, dtype=torch.float64, device="cuda")
    e0.record(st)
    sv.probs_device(probs.data_ptr())
    e1.record(st)
    torch.cuda.synchronize()
    t_probs = e0.elapsed_time(e1) / 1e3
    psum_err = abs(float(probs.sum().item()) - 1.0)
    del probs
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    idx = sv.sample(shots, seed=2024)
    t_sample = time.perf_counter() - t0
    k = 10
    marg = sv.probs(list(range(k)))
    hist = np.bincount((idx >> np.uint64(nq - k)).astype(np.int64), minlength=1 << k)
    expct = marg * shots
    mask = expct > 5
    chi2 = float(((hist[mask] - expct[mask]) ** 2 / expct[mask]).sum())
    dof = int(mask.sum()) - 1
    amp = np.dtype(dtype).itemsize
    # known answer: the inverse QFT brings back the RY product state
    thetas = [op[3][0] for op in ops[:nq]]
    undo = [(name, wires, not inv, params) for name, wires, inv, params in reversed(ops[nq:])]
    e0.record(st)
    sv.apply_ops_fused(undo)
    e1.record(st)
    torch.cuda.synchronize()
    t_undo = e0.elapsed_time(e1) / 1e3
    z, _ = sv.expval_pauli([("Z", [q]) for q in range(nq)])
    marg_err = 0.0
    for wires in (list(range(10)), list(range(nq - 10, nq)), [0, 15, 16, 30, nq - 1]):
        marg_err = max(marg_err, float(np.abs(sv.probs(wires) - product_marginal(thetas, wires)).max()))
    known = {"circuit": "RY layer + QFT + inverse QFT = RY product state", "inverse_qft_s": t_undo,
             "max_abs_err_expval_z": float(np.abs(z - np.cos(thetas)).max()),
             "max_abs_err_marginals": marg_err, "norm2_err": abs(sv.norm2() - 1.0),
             "marginals": "wires 0-9, the last 10, and (0, 15, 16, 30, n-1)"}
    sv.close()
    return {"qubits": nq, "dtype": "c64" if np.dtype(dtype) == np.complex64 else "c128",
            "state_gib": (amp << nq) / 2**30, "gates": len(ops), "gates_fused_s": t_gates,
            "norm2_err": norm_err, "probs_s": t_probs, "probs_gbs": ((amp + 8) << nq) / t_probs / 1e9,
            "probs_sum_err": psum_err, "shots": shots, "sample_s": t_sample, "shots_per_s": shots / t_sample,
            "chi2_per_dof": chi2 / max(dof, 1), "chi2_dof": dof, "vs_fp64_closed_form": known}


def precision_vs_reference(nq: int = 24):
    """The same circuit family at nq qubits against the reference's own complex128 lightning.qubit
    on the host (FP64): max |probs difference| over every basis state, a 10-wire marginal and a
    four-term Pauli Hamiltonian, for the complex128 and complex64 engines."""
    import ref  # the reference module built from its sources: the FP64 answer only
    from lightning_b200 import capi
    from lightning_b200.workloads import qft_circuit
    m = ref.load()
    if m is None:
        return {"unavailable": "reference module not built"}
    ops = qft_circuit(nq, seed=9)
    t0 = time.perf_counter()
    psi = ref.run_circuit(m, nq, ops)
    t_ref = time.perf_counter() - t0
    ham = [(0.7, [("PauliZ", [0]), ("PauliX", [5])]), (-1.3, [("PauliY", [nq - 1])]),
           (0.4, [("PauliX", [11]), ("PauliX", [12])]), (2.1, [("PauliZ", [17])])]
    ev_ref = ref.expval(m, psi.copy(), ham)
    marg_ref = ref.probs(m, psi.copy(), list(range(10)))
    p_ref = np.abs(psi) ** 2
    out = {"qubits": nq, "gates": len(ops), "reference_cpu_s": t_ref}
    for dt, label in ((np.complex128, "c128"), (np.complex64, "c64")):
        sv = capi.StateVector(nq, dt)
        sv.apply_ops_fused(ops)
        out[label] = {"max_abs_err_probs": float(np.abs(sv.probs() - p_ref).max()),
                      "max_abs_err_marginal_10": float(np.abs(sv.probs(list(range(10))) - marg_ref).max()),
                      "abs_err_expval": abs(sv.expval(ham) - ev_ref)}
        sv.close()
    return out


def precision_compare(nq: int = 32, k: int = 16):
    """complex64 vs complex128 on the same nq-qubit circuit: max |difference| of the top-k-wire
    marginal probabilities (the complex128 path is pinned to the FP64 oracle at small sizes)."""
    from lightning_b200 import capi
    from lightning_b200.workloads import qft_circuit
    ops = qft_circuit(nq, seed=9)
    out = {}
    for dt in (np.complex128, np.complex64):
        sv = capi.StateVector(nq, dt)
        sv.apply_ops_fused(ops)
        out[np.dtype(dt).name] = sv.probs(list(range(k)))
        sv.close()
    return {"qubits": nq, "marginal_wires": k,
            "max_abs_diff_c64_vs_c128": float(np.abs(out["complex64"] - out["complex128"]).max())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--sweep-qubits", type=int, default=30)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--case", default="full", choices=["full", "gate", "batch", "fused", "precision", "plain", "matrix", "rows", "next", "pauli"],
                    help="gate / batch: one kernel family on a small case (profiling)")
    ap.add_argument("--qubits", type=int, default=28, help="--case gate: state width (complex128)")
    ap.add_argument("--gate", default="RX", help="--case gate: gate name")
    ap.add_argument("--wires", default="3", help="--case gate: comma-separated wires (negative: from the last)")
    ap.add_argument("--ncirc", type=int, default=148, help="--case batch: number of circuits")
    ap.add_argument("--dtype", default="c128", choices=["c64", "c128"], help="--case fused / matrix / pauli: state precision")
    ap.add_argument("--k", type=int, default=5, help="--case matrix: wires of the unitary")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.case != "full":
        run_case(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference_arm(args)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from lightning_b200 import capi
    from lightning_b200.batch import BatchedCircuits
    from lightning_b200.autograd import batched_expval
    from lightning_b200.workloads import rot_ring_batch, bind

    hbm_peak, peak_kind = peaks()
    circuits, params_np = rot_ring_batch(**WORKLOAD)
    ncirc, n = WORKLOAD["ncirc"], WORKLOAD["n"]
    eng = BatchedCircuits(circuits, len(params_np), dtype=np.complex64, use_graphs=True)
    params = torch.tensor(params_np, dtype=torch.float64, device="cuda", requires_grad=True)
    rng = np.random.default_rng(0)
    dy_np = rng.normal(size=eng.total_obs)
    dy = torch.tensor(dy_np, dtype=torch.float64, device="cuda")
    tuned = eng.autotune(params.detach())

    def step():
        out = batched_expval(params, eng)
        (g,) = torch.autograd.grad(out, params, dy)
        return out, g

    for _ in range(args.warmup):
        step()
    # the engine's own kernel launches per step, read back from the engine (untimed step)
    out_l = batched_expval(params, eng)
    launches_fwd = eng.last_launches()
    torch.autograd.grad(out_l, params, dy)
    launches_vjp = eng.last_launches()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = Clocks(local)
    with clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            out, g = step()
        e1.record()
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist)
    if dist:
        dist.barrier()
    value = aggregate_rate(world, ncirc, ms)

    # end to end through the public API: params from pinned host memory, results back to the host
    params_host = torch.tensor(params_np, dtype=torch.float64).pin_memory()
    dy_host = torch.tensor(dy_np, dtype=torch.float64).pin_memory()
    out_host = torch.empty(eng.total_obs, dtype=torch.float64).pin_memory()
    grad_host = torch.empty(len(params_np), dtype=torch.float64).pin_memory()

    def e2e_step():
        p = params_host.to("cuda", non_blocking=True).requires_grad_(True)
        d = dy_host.to("cuda", non_blocking=True)
        o = batched_expval(p, eng)
        (gg,) = torch.autograd.grad(o, p, d)
        out_host.copy_(o.detach(), non_blocking=True)
        grad_host.copy_(gg, non_blocking=True)
    e2e_ms = max_over_ranks(timed(e2e_step, args.steps, args.warmup), dist)
    h2d = (params_host.numel() + dy_host.numel()) * 8
    d2h = (out_host.numel() + grad_host.numel()) * 8

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    # plain per-circuit complex128 GPU path: one gate per launch through the C ABI
    nplain = 8
    sv = capi.StateVector(n, np.complex128)
    grads_plain = []

    def plain_circuit(ci):
        c = circuits[ci]
        ops = bind(c, params_np)
        sv.set_basis_state(0)
        sv.apply_ops(ops)
        sv.expval_pauli([("Z", [q]) for q in range(n)])
        w = dy_np[ci * n:(ci + 1) * n]
        ham = [[(float(w[q]), [("PauliZ", [q])]) for q in range(n)]]
        npo = sum(1 for p in c["param_index"] if p >= 0)
        return sv.adjoint_jacobian(ops, ham, list(range(npo)))[0]
    plain_circuit(nplain)  # warm-up: loads every kernel the plain path uses
    t0 = time.perf_counter()
    for ci in range(nplain):
        grads_plain.append(plain_circuit(ci))
    plain_s = time.perf_counter() - t0
    plain_value = nplain / plain_s
    # gradient accuracy of the batched complex64 path against FP64 (plain complex128, oracle-checked)
    g_np = g.detach().cpu().numpy()
    err = 0.0
    for ci in range(nplain):
        slots = [p for p in circuits[ci]["param_index"] if p >= 0]
        err = max(err, float(np.abs(g_np[slots] - grads_plain[ci]).max()))
    sv.close()

    sweeps = {str(q): gate_sweep(q, hbm_peak, not args.no_cpu) for q in (26, 28, 30, 32)}
    roof = sweep_roofline(sweeps["30"], hbm_peak)
    roof["peak_kind"] = peak_kind
    msweep = matrix_sweep(args.sweep_qubits, hbm_peak)
    rows = rows_30q(args.sweep_qubits, hbm_peak, not args.no_cpu)
    nxt = next_rows(not args.no_cpu)

    cpu = None if args.no_cpu else reference_cpu(circuits, params_np, dy_np, 4)
    del eng
    torch.cuda.empty_cache()
    hea = hea_forward(3, 3, cpu=not args.no_cpu)
    hea128 = hea_forward(3, 3, dtype=np.complex128, cpu=not args.no_cpu)
    samp = sampling_case(28)
    plain20 = plain_layered(not args.no_cpu)
    precision = {"c64_33q": precision_case(33, np.complex64), "c128_32q": precision_case(32, np.complex128),
                 "c64_vs_c128_32q": precision_compare(32)}
    if not args.no_cpu:
        precision["vs_reference_24q"] = precision_vs_reference(24)
    line = {
        "metric": METRIC, "value": value, "unit": "circuits/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 (fp32-pair compensated gates, fp64 reductions)",
        "data": "synthetic (seeded)",
        "config": {"workload": "batched adjoint: 1024 circuits x 16 qubits x 8 layers Rot(RZ RY RZ) + CNOT ring "
                               "(range (l mod 15)+1), 16 PauliZ observables, forward + VJP per step",
                   "circuits_per_gpu": ncirc, "qubits": n, "params_per_circuit": 3 * n * WORKLOAD["layers"],
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (1 GiB of live states per step)",
                   "autotuned_config": tuned},
        "plain": {"value": plain_value, "unit": "circuits/s", "dtype": "c128", "sample_circuits": nplain,
                  "path": "C ABI, one gate per launch: apply_ops + 16 Pauli expvals + adjoint VJP"},
        "ratio_vs_plain": value / world / plain_value,
        "max_grad_err_vs_fp64": err,
        "gate_sweep": sweeps,
        "matrix_sweep": msweep,
        "rows_single_state": rows,
        "rows_next": nxt,
        "hea_batch_forward": hea,
        "hea_batch_forward_c128": hea128,
        "sampling": samp,
        "plain_20q_layered": plain20,
        "precision_sampling": precision,
        "roofline": roof,
        "roofline_batch": {
            "kernel": "k_batch<float,0|1,false> (forward + VJP launch of the headline step)",
            "bound": "issue", "hbm_traffic_per_step": BATCH_DRAM_BYTES_148 * ncirc / 148,
            "hbm_achieved_gbs": BATCH_DRAM_BYTES_148 * ncirc / 148 / (ms * 1e6),
            "hbm_frac": BATCH_DRAM_BYTES_148 * ncirc / 148 / (ms * 1e6) / hbm_peak, "peak_kind": peak_kind,
            "issue_active_frac": BATCH_ISSUE_ACTIVE,
            "note": "per-circuit states stay in shared memory within a segment; the kernel is bound by "
                    "instruction issue and latency (ncu: FMA pipe 20-23 %, shared memory 42-49 %), not by HBM"},
        "cpu_baseline": cpu,
        "e2e": {"value": aggregate_rate(world, ncirc, e2e_ms), "unit": "circuits/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": (launches_fwd + launches_vjp) * args.steps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
