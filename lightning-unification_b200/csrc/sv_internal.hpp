// sv_internal.hpp — declarations shared by the .cu files of libb200sv (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "../../include/b200sv.h"
#include "gate_compiler.hpp"

namespace b200sv {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct AllocError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, const char *what);

// Runs f, maps exceptions to a b200sv_status code and records the message for
// b200sv_last_error() (defined in sv_capi.cu, shared by every entry point).
int run_guarded(const std::function<void()> &f);
#define B200SV_CUDA(x) ::b200sv::cuda_check((x), #x)

// Number of SMs of the current device (cached per device).
int sm_count();

constexpr int kMaxStatesPerLaunch = 32;

// Apply a compiled gate to `nstates` states of 2^nq amplitudes of precision R
// (R = float or double).  `dev_scratch` must hold 4^k complex<R> when the
// descriptor is Dense with k >= 4 (used for the matrix); it is written with a
// stream-ordered copy before the launch.
template <typename R>
void launch_gate(void *const *states, int nstates, uint32_t nq, const GateDesc &g,
                 void *dev_matrix_scratch, cudaStream_t st);

// complex64 dense matrices on 3..5 wires on the tensor cores (sv_tensor.cu): applies when
// the descriptor has no controls and the state holds at least one 128-group tile;
// `scratch` must hold dense_tc_scratch_bytes(k) bytes (the split real-embedded matrix).
bool dense_tc_applies(uint32_t nq, const GateDesc &g);
size_t dense_tc_scratch_bytes(int k);
void launch_dense_tc(void *const *states, int ns, uint32_t nq, const GateDesc &g, void *scratch, cudaStream_t st);
// MMA-completion waits that gave up since the library was loaded (0 in a healthy run)
unsigned int dense_tc_timeouts();

// ---- reductions (sv_reduce.cu) -------------------------------------------
// All reductions are two-pass and deterministic: per-block partials into
// `partials` (kPartialsCapacity doubles), then one block finalises into a
// device array.  Results stay on the device unless noted.
constexpr int kMaxRedBlocks = 1184;     // 148 SMs x 8
constexpr size_t kPartialsCapacity = size_t(kMaxRedBlocks) * 64;

// out_dev[0] = ||a||^2
template <typename R>
void reduce_norm2(const void *a, uint32_t nq, double *partials, double *out_dev, cudaStream_t st);
// out_dev[0..1] = <bra|ket> (re, im)
template <typename R>
void reduce_inner(const void *bra, const void *ket, uint32_t nq, double *partials, double *out_dev,
                  cudaStream_t st);
// A Pauli word: P|i> = i^ny (-1)^popcount(i & zmask) |i ^ xmask> (zmask covers Z and Y factors).
struct PauliWord {
    uint64_t xmask = 0, zmask = 0;
    int ny = 0;  // number of Y factors (phase i^ny)
};
// out_dev[t] = <psi|P_t|psi> for up to 32 words sharing one X mask, in one pass over the
// amplitude pairs; with_norm: out_dev[nterms] = <psi|psi> from the same pass.
template <typename R>
void reduce_pauli_group(const void *psi, uint32_t nq, const PauliWord *terms, int nterms,
                        double *partials, double *out_dev, cudaStream_t st, bool with_norm = false);
// out_dev[t] = <psi|Z_(zmask_dev[t])|psi> for up to 256 diagonal words (device masks), one
// pass over a state of at least 12 qubits.
template <typename R>
void reduce_pauli_diag(const void *psi, uint32_t nq, const uint64_t *zmask_dev, int nwords, double *partials,
                       size_t partials_cap, double *out_dev, cudaStream_t st);
// out_dev[t] = <psi|P_t|psi> for up to 32 words of any X masks, sorted by X mask, in one pass
// (each amplitude and its partners read; for partners within L2 reach).
template <typename R>
void reduce_pauli_multi(const void *psi, uint32_t nq, const PauliWord *terms, int nterms,
                        double *partials, double *out_dev, cudaStream_t st);
// tile bits (state positions) of a tiled Pauli pass over words whose X masks OR to xunion:
// those bits, the lowest 3 (complex128) or 4 (complex64) state bits, then the lowest others up
// to 12 (complex128) or 13 (complex64) bits; 0 when they do not fit
uint64_t pauli_tile_bits(uint64_t xunion, uint32_t nq, size_t amp_bytes);
// words with X factors, sorted by X mask, whose X masks fit one tile (pauli_tile_bits): one
// read of the state for the group (<= 32 words)
template <typename R>
void reduce_pauli_tiled(const void *psi, uint32_t nq, const PauliWord *terms, int nterms, double *partials,
                        double *out, cudaStream_t st);
// out_dev[0] = Re <psi| M |psi> for a dense Hermitian M on k <= 4 bits (matrix on device).
template <typename R>
void reduce_dense_expval(const void *psi, uint32_t nq, const GateDesc &g, void *dev_matrix,
                         double *partials, double *out_dev, cudaStream_t st);
// One adjoint step of a one-wire gate on state bit `bit`: out_dev[o * out_stride] = alpha *
// Im <bra_o| G |lambda> (G the 2x2 generator), then lambda and every bra <- U lambda, U bra
// (U the 2x2 inverse gate), in one pass; `arrival` as for reduce_generator_inner.
template <typename R>
void adjoint_rot_step(void *lambda, void *const *bras, int nbra, uint32_t nq, uint32_t bit, const cd (&g)[4],
                      const cd (&u)[4], double alpha, double *partials, double *out_dev, int out_stride,
                      unsigned int *arrival, cudaStream_t st);
// out_dev[o * out_stride] = alpha * Im <bra_o| G |ket>, o < nbra (<= 16).  With `arrival`
// (a device counter that is zero, and is left zero) the kernel's last block forms the results
// and no finalize launch follows.
template <typename R>
void reduce_generator_inner(void *const *bras, int nbra, const void *ket, uint32_t nq,
                            const GateDesc &g, double alpha, double *partials, double *out_dev,
                            int out_stride, cudaStream_t st, unsigned int *arrival = nullptr);
// out2_dev[0..1] = (Re, Im) <bra| G |ket>.
template <typename R>
void reduce_generator_inner_complex(const void *bra, const void *ket, uint32_t nq, const GateDesc &g,
                                    double *partials, double *out2_dev, cudaStream_t st);
// out_dev[0] = Re<psi|H psi>, out_dev[1] = |H psi|^2 for H in CSR form (device arrays,
// row i owning [row_map[i] - row_map[0], row_map[i+1] - row_map[0]), nnz the entries row_map
// addresses); sv_sparse.cu.  *bad_dev (zero before the call) gets bit 0 for decreasing row
// bounds, bit 2 for a row ending past nnz and bit 1 for a column index outside the state.
template <typename R>
void reduce_sparse(const void *psi, uint32_t nq, const uint64_t *row_map_dev, const uint64_t *cols_dev,
                   const void *vals_dev, uint64_t nnz, double *partials, double *out_dev, unsigned int *bad_dev,
                   cudaStream_t st);
int sparse_lanes(uint64_t nrows, uint64_t nnz);
// Metropolis-Hastings chains (sv_mcmc.cu): nshots indices into a device buffer.
void sample_mcmc(const void *state, uint32_t nq, int dtype, int proposal, uint64_t burnin, uint64_t nshots,
                 uint64_t nchains, uint64_t seed, uint64_t *idx_dev, cudaStream_t st);
// Fused application of compiled gates to one state (sv_fused.cu): runs of gates that
// fit a shared-memory tile of 2^fused_tile_bits amplitudes share one pass over the
// state; other gates go through apply_single, in order.
int fused_tile_bits(int dtype, uint32_t nq);
bool fused_worthwhile(int dtype, uint32_t nq);
// One step of the adjoint reverse sweep: the inverse of an op and, when the op is
// differentiated, its generator G with alpha = -2 * scale, and the Jacobian column.
struct AdjItem {
    GateDesc adj;
    bool diff = false;
    GateDesc G;
    double alpha = 0.0;
    int64_t col = -1;
};
// The sweep over lambda and one bra in fused passes; items without a register form run
// through exec_single(i) in order.  Products land in d_jac[col].
bool fused_adjoint_worthwhile(int dtype, uint32_t nq);
void apply_fused_adjoint(void *lambda, void *bra, uint32_t nq, int dtype, const std::vector<AdjItem> &items,
                         const std::function<void(size_t)> &exec_single, double *d_jac, cudaStream_t st);
void apply_fused(void *state, uint32_t nq, int dtype, const std::vector<GateDesc> &descs,
                 const std::function<void(const GateDesc &)> &apply_single, cudaStream_t st);
// Marginal probabilities over `bits` (bits[0] = MSB of the output index).
template <typename R>
void reduce_probs(const void *psi, uint32_t nq, const std::vector<uint32_t> &bits, double *partials,
                  size_t partials_cap, double *out_dev, cudaStream_t st);

// ---- elementwise helpers (sv_reduce.cu) ----------------------------------
template <typename R> void set_basis(void *psi, uint32_t nq, uint64_t index, cudaStream_t st);
// acc += c * P psi for one Pauli word (no aliasing between acc and psi)
template <typename R>
void axpy_pauli(void *acc, const void *psi, uint32_t nq, const PauliWord &w, double c,
                cudaStream_t st);
// acc += c * x
template <typename R> void axpy(void *acc, const void *x, uint32_t nq, double c, cudaStream_t st);

// ---- sampling (sv_sample.cu) ---------------------------------------------
// Doubles of workspace for the run offsets of the fixed-order CDF (about N / 31).
size_t run_offsets_doubles(uint64_t N);
// O_1 (the CDF at every 32nd index) into the start of work
template <typename R> void build_run_offsets(const void *psi, uint32_t nq, double *work, cudaStream_t st);
void philox_uniforms(double *u, uint64_t n, uint64_t seed, cudaStream_t st);
// inverse-CDF indices for nshots uniforms, CDF entries formed from O_1 and the state
template <typename R>
void sample_runs(const void *psi, uint32_t nq, const double *o1, const double *u, uint64_t nshots, uint64_t *idx,
                 cudaStream_t st);

}  // namespace b200sv
