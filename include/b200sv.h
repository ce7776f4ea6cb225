/*
 * b200sv.h — C ABI of the B200 state-vector engine (libb200sv.so).
 *
 * This is the drop-in boundary for the hot path of lightning.qubit: state-vector
 * gate application, measurements and adjoint differentiation.  Every entry point
 * is `extern "C"`, takes plain pointers and sizes, returns an int status
 * (B200SV_OK == 0) and leaves a thread-local message for b200sv_last_error().
 *
 * Conventions kept from the reference (paths relative to the reference project,
 * pennylane_lightning/core/src = CS/, CS/simulators/lightning_qubit = LQ/):
 *   - wire 0 is the most significant bit of the basis index
 *     (rev_wire = n - 1 - wire, LQ/gates/cpu_kernels/GateImplementationsLM.hpp:210);
 *   - matrices are row-major complex<T>, wires[0] is the most significant bit of
 *     the matrix index; `inverse` means conjugate transpose
 *     (GateImplementationsLM.hpp:204-387);
 *   - gate and generator ids are the enum values of CS/gates/GateOperation.hpp:27-111;
 *   - Jacobians are laid out [observable][trainable parameter]
 *     (LQ/algorithms/AdjointJacobianLQubit.hpp:331-334).
 *
 * All device work of a handle runs on that handle's CUDA stream and is ordered
 * there; calls that return host data synchronise that stream.  No call falls back
 * to the CPU: when no CUDA device is usable, b200sv_create fails.
 */
#ifndef B200SV_H
#define B200SV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum b200sv_status {
    B200SV_OK = 0,
    B200SV_ERR_ARGUMENT = 1,    /* bad wires, sizes, ids, parameter counts   */
    B200SV_ERR_CUDA = 2,        /* a CUDA runtime call failed                */
    B200SV_ERR_ALLOC = 3,       /* device or pinned allocation failed        */
    B200SV_ERR_UNSUPPORTED = 4, /* valid request this build does not handle  */
    B200SV_ERR_TIMEOUT = 5,     /* a bounded device wait ran out             */
    B200SV_ERR_CANCELLED = 6    /* a batch was cancelled before completion   */
};

/* ---- precisions -------------------------------------------------------- */
enum b200sv_dtype {
    B200SV_C64 = 0,  /* complex<float>  amplitudes, FP64 reductions          */
    B200SV_C128 = 1  /* complex<double> amplitudes                           */
};

/* ---- gate ids: CS/gates/GateOperation.hpp:27-70 (same numeric values) --- */
enum b200sv_gate {
    B200SV_Identity = 0, B200SV_PauliX, B200SV_PauliY, B200SV_PauliZ,
    B200SV_Hadamard, B200SV_S, B200SV_T, B200SV_PhaseShift, B200SV_RX,
    B200SV_RY, B200SV_RZ, B200SV_Rot,
    B200SV_CNOT, B200SV_CY, B200SV_CZ, B200SV_SWAP, B200SV_IsingXX,
    B200SV_IsingXY, B200SV_IsingYY, B200SV_IsingZZ,
    B200SV_ControlledPhaseShift, B200SV_CRX, B200SV_CRY, B200SV_CRZ,
    B200SV_CRot, B200SV_SingleExcitation, B200SV_SingleExcitationMinus,
    B200SV_SingleExcitationPlus,
    B200SV_Toffoli, B200SV_CSWAP,
    B200SV_DoubleExcitation, B200SV_DoubleExcitationMinus,
    B200SV_DoubleExcitationPlus,
    B200SV_MultiRZ,
    B200SV_GATE_END,
    /* ids outside the reference enum used in operation lists */
    B200SV_OP_MATRIX = 1000, /* dense matrix given in b200sv_op.matrix       */
    B200SV_OP_SKIP = 1001    /* state-preparation ops the adjoint ignores
                                ("QubitStateVector", "BasisState":
                                AdjointJacobianLQubit.hpp:287-290)          */
};

/* ---- generator ids: CS/gates/GateOperation.hpp:75-98 -------------------- */
enum b200sv_generator {
    B200SV_GEN_PhaseShift = 0, B200SV_GEN_RX, B200SV_GEN_RY, B200SV_GEN_RZ,
    B200SV_GEN_IsingXX, B200SV_GEN_IsingXY, B200SV_GEN_IsingYY,
    B200SV_GEN_IsingZZ, B200SV_GEN_CRX, B200SV_GEN_CRY, B200SV_GEN_CRZ,
    B200SV_GEN_ControlledPhaseShift, B200SV_GEN_SingleExcitation,
    B200SV_GEN_SingleExcitationMinus, B200SV_GEN_SingleExcitationPlus,
    B200SV_GEN_DoubleExcitation, B200SV_GEN_DoubleExcitationMinus,
    B200SV_GEN_DoubleExcitationPlus, B200SV_GEN_MultiRZ,
    B200SV_GEN_END
};

typedef struct b200sv_state *b200sv_handle;

/* One operation of a gate list (CS/algorithms/JacobianData.hpp:40-197 OpsData:
 * name, params, wires, inverse, matrix).  `matrix` is complex<T> row-major of
 * size 4^nwires, read only when gate == B200SV_OP_MATRIX. */
typedef struct b200sv_op {
    uint32_t gate;
    uint32_t nwires;
    const uint32_t *wires;
    int32_t inverse;
    uint32_t nparams;
    const double *params;
    const void *matrix;
} b200sv_op;

/* One factor of an observable term: a named operator (a gate id applied as an
 * operator, e.g. PauliX/Y/Z, Hadamard, Identity — CS/observables/Observables.hpp:101-143)
 * or a Hermitian matrix (Observables.hpp:151-198). */
enum b200sv_factor_kind { B200SV_FACTOR_NAMED = 0, B200SV_FACTOR_MATRIX = 1 };
typedef struct b200sv_factor {
    uint32_t kind;
    uint32_t gate;          /* for B200SV_FACTOR_NAMED                       */
    uint32_t nwires;
    const uint32_t *wires;
    const void *matrix;     /* for B200SV_FACTOR_MATRIX: complex<T>[4^nwires] */
} b200sv_factor;

/* A term: coeff * (tensor product of factors on disjoint wires). */
typedef struct b200sv_term {
    double coeff;
    uint32_t nfactors;
    const b200sv_factor *factors;
} b200sv_term;

/* An observable: NamedObs / HermitianObs / TensorProdObs are one term with
 * coeff 1; a Hamiltonian is a list of terms (Observables.hpp:325-416). */
typedef struct b200sv_observable {
    uint32_t nterms;
    const b200sv_term *terms;
} b200sv_observable;

/* ---- library ----------------------------------------------------------- */
/* Last error message of the calling thread ("" when none). */
const char *b200sv_last_error(void);
/* ABI version (major*10000 + minor*100 + patch). */
int b200sv_version(void);
/* Number of CUDA devices usable by the library (0 when none). */
int b200sv_device_count(int *count);

/* ---- state lifecycle: LQ/StateVectorLQubitManaged.hpp:72-129 ------------ */
/* Allocate 2^num_qubits amplitudes on the current device, set to |0...0>. */
int b200sv_create(uint32_t num_qubits, int dtype, b200sv_handle *out);
int b200sv_destroy(b200sv_handle h);
int b200sv_num_qubits(b200sv_handle h, uint32_t *out);
int b200sv_dtype(b200sv_handle h, int *out);
/* Run the handle's work on `cuda_stream` from now on (e.g. torch's current
 * stream).  NULL selects the legacy default stream, which torch uses unless told
 * otherwise.  Until the first call the handle runs on a private stream.  When the
 * stream changes, the call waits for the work already issued on the previous one. */
int b200sv_set_stream(b200sv_handle h, void *cuda_stream);
int b200sv_synchronize(b200sv_handle h);
/* Device address of the amplitudes (complex<T>[2^n]) for zero-copy interop. */
int b200sv_device_ptr(b200sv_handle h, void **out);
/* Copy 2^n complex<T> host amplitudes in / out (updateData, getData). */
int b200sv_upload(b200sv_handle h, const void *host, uint64_t length);
int b200sv_download(b200sv_handle h, void *host, uint64_t length);
/* dst <- src (same size and dtype): the copy constructor. */
int b200sv_copy(b200sv_handle dst, b200sv_handle src);
/* |index> (index 0 = |0...0>): setBasisState. */
int b200sv_set_basis_state(b200sv_handle h, uint64_t index);

/* ---- gates: CS/simulators/base/StateVectorBase.hpp:99-194 ---------------- */
/* applyOperation(name, wires, inverse, params) with the name resolved to an id
 * (LQ/StateVectorLQubit.hpp:231-240).  Parameter counts follow
 * CS/gates/Constant.hpp:234-269; wire counts Constant.hpp:163-197 (MultiRZ: any). */
int b200sv_apply_gate(b200sv_handle h, uint32_t gate, const uint32_t *wires,
                      uint32_t nwires, int inverse, const double *params,
                      uint32_t nparams);
/* applyMatrix (LQ/StateVectorLQubit.hpp:329-365): complex<T> row-major 4^nwires. */
int b200sv_apply_matrix(b200sv_handle h, const void *matrix,
                        const uint32_t *wires, uint32_t nwires, int inverse);
/* applyOperations: a list applied in order on the handle's stream. */
int b200sv_apply_ops(b200sv_handle h, const b200sv_op *ops, uint32_t nops);
/* applyOperations with gate fusion: the list is cut into segments whose wires
 * fit in a shared-memory tile (2^12 complex128 / 2^13 complex64 amplitudes, the
 * lowest wires filling the rest so loads coalesce), and each segment is one
 * pass over HBM instead of one pass per gate.  Same results as
 * b200sv_apply_ops to rounding (complex128: 1e-12).  Gates outside the tile
 * forms (more than three wires, dense matrices on three wires) run as their own
 * pass in order.  States narrower than the tile plus 8 wires use the per-gate
 * path. */
int b200sv_apply_ops_fused(b200sv_handle h, const b200sv_op *ops, uint32_t nops);
/* applyGenerator (LQ/StateVectorLQubit.hpp:250-275): G applied in place (it is
 * not unitary for projector-type generators); *scale receives the factor of
 * GateImplementationsLM.hpp:1355-1639 / PauliGenerator.hpp:34-56. */
int b200sv_apply_generator(b200sv_handle h, uint32_t generator,
                           const uint32_t *wires, uint32_t nwires, int adj,
                           double *scale);

/* ---- measurements: LQ/measurements/MeasurementsLQubit.hpp:79-558 --------- */
/* probs() (nwires == 0 means all wires in order 0..n-1) and probs(wires):
 * out receives 2^nwires FP64 values, wires[0] the most significant bit. */
int b200sv_probs(b200sv_handle h, const uint32_t *wires, uint32_t nwires,
                 double *out);
/* Device-side variant: writes 2^nwires doubles to a device buffer. */
int b200sv_probs_device(b200sv_handle h, const uint32_t *wires,
                        uint32_t nwires, double *out_device);
/* psi <- O psi in place (Observable::applyInPlace, CS/observables/Observables.hpp:63-73;
 * Hamiltonian::applyInPlace, LQ/observables/ObservablesLQubit.hpp:156-305: the sum of
 * coeff * term applied to copies of psi).  O need not be unitary, so psi is not renormalised. */
int b200sv_apply_observable(b200sv_handle h, const b200sv_observable *obs);
/* <psi|O|psi> for an observable (expval(Observable), :248-265). */
int b200sv_expval(b200sv_handle h, const b200sv_observable *obs, double *out);
/* <O^2> - <O>^2 as ||O psi||^2 - <psi|O psi>^2 (var(Observable), :273-372). */
int b200sv_var(b200sv_handle h, const b200sv_observable *obs, double *out);
/* Pauli-word sums evaluated as read-only fused reductions.  Term t acts with
 * paulis[off[t]..off[t+1]) ('I','X','Y','Z') on wires[off[t]..off[t+1]).
 * out_terms (nterms doubles, may be NULL) receives each <P_t>; out_sum (may
 * be NULL) receives sum_t coeffs[t] <P_t>. */
int b200sv_expval_pauli(b200sv_handle h, uint32_t nterms, const double *coeffs,
                        const uint32_t *offsets, const uint32_t *wires,
                        const char *paulis, double *out_terms, double *out_sum);
/* Re/Im of <bra|ket> in FP64 (innerProdC, LQ/utils/LinearAlgebra.hpp:190-213). */
int b200sv_inner_product(b200sv_handle bra, b200sv_handle ket, double *re,
                         double *im);
/* ||psi||^2 in FP64. */
int b200sv_norm2(b200sv_handle h, double *out);
/* Sparse Hamiltonian H in CSR form (host arrays): row i holds the non-zeros
 * [row_map[i] - row_map[0], row_map[i+1] - row_map[0]) of entries (column
 * indices) and values (complex in the handle's dtype).  row_map_size must be
 * 2^n + 1 ("Statevector and Hamiltonian have incompatible sizes." otherwise).
 * expval = Re<psi|H psi>  (expval(row_map, ..., numNNZ),
 * LQ/measurements/MeasurementsLQubit.hpp:197-214; binding
 * LQ/bindings/LQubitBindings.hpp:127-138);
 * var = <H psi|H psi> - Re<H psi|psi>^2  (var(row_map, ...), :451-472;
 * binding LQubitBindings.hpp:150-161).  Accumulated in FP64. */
int b200sv_expval_sparse(b200sv_handle h, const uint64_t *row_map,
                         uint64_t row_map_size, const uint64_t *entries,
                         const void *values, uint64_t nnz, double *out);
int b200sv_var_sparse(b200sv_handle h, const uint64_t *row_map,
                      uint64_t row_map_size, const uint64_t *entries,
                      const void *values, uint64_t nnz, double *out);
/* The same with the CSR arrays already in device memory (a Hamiltonian kept resident
 * across calls): row_map holds 2^n + 1 entries, entries and values nnz each; nothing
 * crosses from the host.  Row bounds and column indices are checked on the device, with
 * the messages of the host-array forms. */
int b200sv_expval_sparse_device(b200sv_handle h, const uint64_t *row_map_device,
                                const uint64_t *entries_device,
                                const void *values_device, uint64_t nnz,
                                double *out);
int b200sv_var_sparse_device(b200sv_handle h, const uint64_t *row_map_device,
                             const uint64_t *entries_device,
                             const void *values_device, uint64_t nnz,
                             double *out);

/* Sampling by inverse CDF (the lightning.kokkos rule,
 * LK/measurements/MeasuresFunctors.hpp:70-103 over an exclusive scan,
 * LK/measurements/MeasurementsKokkos.hpp:713-722).  p_i = re*re + im*im in FP64
 * without contraction; the scan order is fixed (runs of 32 summed in sequence,
 * recursively, offsets added top-down), so the indices
 * are a deterministic function of the state and the uniforms.
 * uniforms: nshots doubles in [0,1) on the host, or NULL to draw them on the
 * device from Philox4x32-10 with `seed`.  idx_out: nshots basis indices. */
int b200sv_sample(b200sv_handle h, uint64_t nshots, const double *uniforms,
                  uint64_t seed, uint64_t *idx_out);
/* generate_samples layout: nshots x n bits, MSB (wire 0) first, as uint64. */
int b200sv_sample_bits(b200sv_handle h, uint64_t nshots, const double *uniforms,
                       uint64_t seed, uint64_t *bits_out);

/* Metropolis-Hastings sampling (generate_samples_metropolis,
 * LQ/measurements/MeasurementsLQubit.hpp:387-434; metropolis_step :612-640;
 * proposals LQ/measurements/TransitionKernels.hpp:56-160).  nchains independent
 * chains start at basis index 0, take num_burnin steps, then chain c gives
 * samples c, c + nchains, ... from consecutive steps; nchains = 1 is the
 * reference's single chain.  A step accepts the proposal t from i when
 * p_i == 0 or U * p_i < p_t (p = |amplitude|^2 in FP64), i.e.
 * U < min(1, p_t / p_i).  Random numbers: Philox4x32-10, counter
 * (step_lo, step_hi, chain, 0x4D434D43), key seed; the indices are a
 * deterministic function of state, seed and nchains.
 * proposal: B200SV_MCMC_LOCAL sets a uniformly chosen bit to a uniformly chosen
 * value (LocalTransitionKernel); B200SV_MCMC_NONZERO draws uniformly among the
 * basis states with |amplitude| > machine epsilon of the state's precision
 * (NonZeroRandomTransitionKernel).  The reference binds its kernel names the
 * other way round (kernel_factory, TransitionKernels.hpp:147-159): its "Local"
 * name runs the non-zero proposal and "NonZeroRandom" the local one.
 * idx_out: nshots basis indices. */
enum b200sv_mcmc_proposal { B200SV_MCMC_LOCAL = 0, B200SV_MCMC_NONZERO = 1 };
int b200sv_sample_mcmc(b200sv_handle h, int proposal, uint64_t num_burnin,
                       uint64_t nshots, uint32_t nchains, uint64_t seed,
                       uint64_t *idx_out);

/* Allocation-free Pauli-word expectation values.  No counterpart in the
 * reference: this entry point exists for callers that cannot call cudaMalloc
 * when they need the result (device memory owned by another allocator such as
 * PyTorch's caching allocator, serving loops that must not hit cudaMalloc's
 * implicit synchronisation, hosts that forbid allocation after start-up).
 * state_device: 2^num_qubits amplitudes of `dtype` owned by the caller;
 * out_device: nterms doubles owned by the caller, receiving <psi|P_t|psi>;
 * words as in b200sv_expval_pauli.  At most B200SV_NOALLOC_MAX_TERMS words per
 * call (more is rejected with an error).  state_device, out_device and
 * cuda_stream must belong to the current CUDA device (pointers of another device
 * are rejected with an error).  Work is queued on cuda_stream (NULL = legacy
 * default stream) and not synchronised.  Scratch is one static device
 * array shared by all calls: calls that overlap on the GPU race, so serialise
 * them; the first call on a device sets up the array's address and should come
 * before any stream capture. */
#define B200SV_NOALLOC_MAX_TERMS 32
int b200sv_expval_pauli_noalloc(const void *state_device, uint32_t num_qubits,
                                int dtype, uint32_t nterms,
                                const uint32_t *offsets, const uint32_t *wires,
                                const char *paulis, double *out_device,
                                void *cuda_stream);

/* ---- adjoint Jacobian: LQ/algorithms/AdjointJacobianLQubit.hpp:212-335 ---- */
/* jac (nobs x ntp doubles, [obs][param]) for the state in `psi` (unchanged).
 * With apply_operations != 0 the ops are applied to a copy of psi first.
 * trainable holds sorted indices into the list of parametric operations. */
int b200sv_adjoint_jacobian(b200sv_handle psi, const b200sv_op *ops,
                            uint32_t nops, const b200sv_observable *obs,
                            uint32_t nobs, const uint64_t *trainable,
                            uint32_t ntrainable, int apply_operations,
                            double *jac);

/* State-return vector-Jacobian product (LQ/algorithms/VectorJacobianProduct.hpp:60-156):
 * vjp[j] = i * scale_p * <G_p mu | lambda> for trainable parameter p = trainable[j],
 * where lambda starts from psi (after the ops when apply_operations != 0) and mu
 * from the cotangent state dy (2^n complex<T> on the host); both are swept
 * backwards through the ops.  out: ntrainable complex<double> as (re, im) pairs. */
int b200sv_vjp_state(b200sv_handle psi, const b200sv_op *ops, uint32_t nops,
                     const void *dy, uint64_t dy_length, const uint64_t *trainable,
                     uint32_t ntrainable, int apply_operations, double *out);

/* ---- batched engine ------------------------------------------------------ */
/* A batch is a packed pool of independent circuits of uneven width, run by one
 * persistent kernel per step (optionally replayed as a CUDA graph).  Each circuit
 * is an op list over its own wires 0..n_c-1 starting from |0...0>, followed by
 * an observable given as a Pauli-word sum.  Parameters live in one device array
 * so steps can change angles without rebuilding the batch.  Ops: every gate with at
 * most one parameter (the double excitations included) and B200SV_OP_MATRIX on 1 to 4
 * wires; Rot and CRot are given as their RZ RY RZ decomposition. */
typedef struct b200sv_batch *b200sv_batch_handle;

typedef struct b200sv_batch_circuit {
    uint32_t num_qubits;
    uint32_t nops;
    const b200sv_op *ops;           /* params of ops index param_index below */
    const int64_t *param_index;     /* per op: first slot in the batch param
                                       array (-1: op.params used as constants) */
    uint32_t nobs;                  /* Pauli-word observables (outputs)        */
    const uint32_t *obs_nterms;     /* per observable: number of terms        */
    const double *obs_coeffs;       /* all terms, observable-major             */
    const uint32_t *obs_offsets;    /* per term: offsets into wires/paulis     */
    const uint32_t *obs_wires;
    const char *obs_paulis;
} b200sv_batch_circuit;

int b200sv_batch_create(int dtype, const b200sv_batch_circuit *circuits,
                        uint32_t ncircuits, uint64_t nparams,
                        b200sv_batch_handle *out);
int b200sv_batch_destroy(b200sv_batch_handle b);
/* Same stream rule as b200sv_set_stream (NULL = legacy default stream). */
int b200sv_batch_set_stream(b200sv_batch_handle b, void *cuda_stream);
/* Forward: params_device (nparams doubles on the device) -> out_device
 * (sum over circuits of nobs doubles, circuit-major). */
int b200sv_batch_forward(b200sv_batch_handle b, const double *params_device,
                         double *out_device);
/* Adjoint VJP: given dy_device (same layout as the forward outputs), writes
 * grad_device[p] = sum_c sum_o dy[c,o] d<O_{c,o}>/d param[p] (nparams doubles;
 * parameters not referenced by any circuit receive 0). */
int b200sv_batch_vjp(b200sv_batch_handle b, const double *params_device,
                     const double *dy_device, double *grad_device);
/* Full Jacobian per circuit: jac_device[c] block of nobs_c x nparams_c
 * (the circuit's own referenced params in op order), circuit-major. */
int b200sv_batch_jacobian(b200sv_batch_handle b, const double *params_device,
                          double *jac_device);
/* Record the forward / vjp of this batch as CUDA graphs on first use and
 * replay them afterwards (0 = launch directly). */
int b200sv_batch_use_graphs(b200sv_batch_handle b, int enable);
/* Autotuner: times a forward + VJP step (best of three) for each candidate
 * launch shape (threads per CTA x tile width) and keeps the fastest; *chosen
 * receives threads * 100 + tile bits. */
int b200sv_batch_autotune(b200sv_batch_handle b, const double *params_device,
                          int *chosen);
/* Number of kernels the last forward / vjp call launched. */
int b200sv_batch_last_launches(b200sv_batch_handle b, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif /* B200SV_H */
